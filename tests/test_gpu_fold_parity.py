"""Parity on the benchmarked configuration: the 256x256 self-contact fold.

Every test here starts from the benchmark's own fold-phase state
(tests/golden/sheet256_fold_state.npz: config 1, 65,536 vertices, ~95k
retained contact terms) or steps config 1 itself, and compares the CUDA
library (through the C ABI) with the oracle, the FP64 restatement of the
reference CPU path (src/vbd.rs:250-422, src/ogc/world.rs:308-420,
src/ogc/candidates.rs:23-68):

  (c) contact lists (kind, vertices, count, epsilon bits, radii, incidence,
      minimum distance) bit for bit, and fresh candidate pair lists equal;
  (a) one step with the benchmark's settings - residual target 1e-3 checked
      every 2 iterations, stall refresh 2, cap 200, with and without the
      Chebyshev acceleration, plain and learned initial guess, and the
      reference's fixed 30 iterations - within 1e-5 m per vertex, with the
      oracle's iteration and detection counts;
  trajectory: steps 197-200 of the fold generator's run (tests/golden/
      make_fold_state.py) on both sides, each within 1e-5 m.

The learned step is compared by giving the oracle the correction the
library's tcgen05 network computed for that step (the network's own
numerics are checked in test_gpu_learned.py); the oracle then restates
everything the step does with it.
"""
import os

import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.abi import cc_ogc_settings
from clothcraft_b200.learned import Mlp
from clothcraft_b200.vbd import OgcWorld, VbdSolver

pytestmark = pytest.mark.gpu

POSITION_TOL_M = 1e-5  # bar (a)
RESIDUAL_RTOL = 1e-6   # FP64 on both sides; summation order differs
LANES = 8 | 4 << 8     # the lane variant the benchmark's autotuner keeps on a B200
HERE = os.path.dirname(os.path.abspath(__file__))
FOLD = os.path.join(HERE, "golden", "sheet256_fold_state.npz")
MLP = os.path.join(os.path.dirname(HERE), "clothcraft_b200", "data", "fold_init_mlp.npz")
THREADS = os.cpu_count() or 1


def fold_state():
    z = np.load(FOLD)
    return z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])


def assert_same_contacts(a, b, ctx=""):
    assert len(a["kinds"]) == len(b["kinds"]), (ctx, len(a["kinds"]), len(b["kinds"]))
    for key in ("kinds", "vertices", "counts", "incident_offsets", "incident"):
        assert np.array_equal(a[key], b[key]), (ctx, key)
    for key in ("epsilon", "radii"):
        assert np.array_equal(a[key].view(np.uint64), b[key].view(np.uint64)), (ctx, key)
    for k in ("active_contacts", "vertex_face_candidates", "edge_edge_candidates", "broad_phase_rebuilt"):
        assert a[k] == b[k], (ctx, k, a[k], b[k])
    assert np.float64(a["minimum_distance"]).view(np.uint64) == np.float64(b["minimum_distance"]).view(np.uint64)


def test_fold_detection_and_candidate_lists_match_oracle_bit_for_bit():
    sc = scenes.config1()
    x, _, _ = fold_state()
    obs = sc.obstacle
    x_all = np.ascontiguousarray(np.concatenate([x, obs.vertices]))
    tris = np.ascontiguousarray(np.concatenate([sc.mesh.triangles, obs.triangles + sc.n]))
    g = OgcWorld(x_all, tris, sc.n)
    o = oracle.World(x_all, tris, sc.n)
    r = sc.settings.radius
    st = cc_ogc_settings(r, sc.settings.stiffness, 0.45, 0.01)
    # the step's query radius lies in [2r, 4r]; a cache miss, two reuses, a
    # grown radius that rebuilds
    for rq in (2.5 * r, 2.0 * r, 2.2 * r, 4.0 * r):
        a, b = g.detect(x_all, rq, st), o.detect(x_all, rq, st)
        assert len(a["kinds"]) > 5000
        assert_same_contacts(a, b, rq)
        assert a["candidate_pairs"] == b["candidate_pairs"] and a["aabb_rejections"] == b["aabb_rejections"]
    for search in (2.0 * r, 4.0 * r + 1e-4):
        vf_g, ee_g = g.candidates(x_all, search)
        vf_o, ee_o = o.candidates(x_all, search)
        assert len(vf_o) > 10000 and len(ee_o) > 10000
        assert np.array_equal(vf_g, vf_o) and np.array_equal(ee_g, ee_o)


def bench_settings(sc, acceleration, init_mode=0, fixed=None):
    s = sc.settings
    if fixed:
        s.iterations, s.residual_tolerance, s.residual_check_every = fixed, 0.0, fixed
        s.stall_refresh, s.acceleration = 0, 0.0
    else:
        s.iterations, s.residual_tolerance, s.residual_check_every = 200, 1e-3, 2
        s.stall_refresh, s.acceleration = 2, acceleration
    s.init_mode = init_mode
    return s.to_c()


def compare_step(mg, mo, xg, xo):
    err = float(np.linalg.norm(xg - xo, axis=1).max())
    assert err <= POSITION_TOL_M, err
    for key in ("iterations", "detection_updates", "broad_phase_rebuilds", "contact_terms", "colors",
                "truncated_vertices"):
        assert mg[key] == mo[key], (key, mg[key], mo[key])
    for key in ("relative_residual", "initial_relative_residual", "relative_force_residual"):
        assert abs(mg[key] - mo[key]) <= RESIDUAL_RTOL * mo[key], (key, mg[key], mo[key])
    return err


@pytest.mark.parametrize("leg", ["plain_accelerated", "plain", "fixed_30"])
def test_fold_step_with_benchmark_settings_matches_oracle(leg):
    """Plain adaptive init at the benchmark's residual target with and without
    acceleration, and the reference's fixed 30-iteration step."""
    sc = scenes.config1()
    x, v, t = fold_state()
    st = {"plain_accelerated": lambda: bench_settings(sc, 0.95),
          "plain": lambda: bench_settings(sc, 0.0),
          "fixed_30": lambda: bench_settings(sc, 0.0, fixed=30)}[leg]()
    g = VbdSolver(sc).set_lanes(LANES)
    xg, _, tg, mg = g.step(x, v, t, st)
    o = oracle.Solver(sc, threads=THREADS)
    xo, _, to, mo = o.step(x, v, t, st)
    assert tg == to
    compare_step(mg, mo, xg, xo)
    if leg != "fixed_30":
        assert mg["relative_residual"] <= 1e-3 or mg["iterations"] == 200


def test_fold_learned_step_with_benchmark_settings_matches_oracle():
    """The benchmark's `value` leg: shipped network on the tensor cores,
    acceleration 0.95, residual target 1e-3. The oracle gets the network
    output of this very step (features of a sample step from the same state,
    through the same tcgen05 inference) and restates the rest."""
    import torch

    sc = scenes.config1()
    x, v, t = fold_state()
    st = bench_settings(sc, 0.95, init_mode=1)
    net = Mlp.load(MLP)
    probe = VbdSolver(sc).set_lanes(LANES)
    probe.set_state(x, v, t)
    rows = probe.free_vertices
    feats = torch.zeros((rows, 24), dtype=torch.float32, device="cuda")
    targs = torch.zeros((rows, 3), dtype=torch.float32, device="cuda")
    probe.step_sample(bench_settings(sc, 0.95), feats, targs)
    corr = net.forward(feats, precision=1).cpu().numpy()
    assert np.abs(corr).max() > 0.0
    g = VbdSolver(sc).set_lanes(LANES)
    g.set_mlp(net, 1)
    xg, _, _, mg = g.step(x, v, t, st)
    o = oracle.Solver(sc, threads=THREADS)
    o.set_learned_correction(corr)
    xo, _, _, mo = o.step(x, v, t, st)
    assert mg["init_used"] == mo["init_used"]
    compare_step(mg, mo, xg, xo)


def test_fold_generator_steps_match_oracle():
    """Steps 197-200 of the fold generator's run: the GPU advances config 1
    from its initial state, and from each of its states 196-199 a fresh GPU
    solver and a fresh oracle take the next step (no adaptive-init history on
    either side), within bar (a) with the oracle's detection and colour
    counts. (Along two separate trajectories the last-bit differences of the
    contact-rich fold grow from step to step, ~3e-5 m after three steps, so
    each step is checked from the same state.)"""
    sc = scenes.config1()
    st = sc.settings.to_c()
    run = VbdSolver(sc).set_lanes(LANES)
    run.set_state(sc.x0, sc.v0, 0.0)
    for _ in range(196):
        run.step_resident(st)
    contact_terms = 0
    for k in range(4):
        x, v, t = run.get_state()
        xg, _, _, mg = VbdSolver(sc).set_lanes(LANES).step(x, v, t, st)
        xo, _, _, mo = oracle.Solver(sc, threads=THREADS).step(x, v, t, st)
        err = float(np.linalg.norm(xg - xo, axis=1).max())
        assert err <= POSITION_TOL_M, (k, err)
        for key in ("detection_updates", "contact_terms", "colors"):
            assert mg[key] == mo[key], (k, key, mg[key], mo[key])
        contact_terms = mg["contact_terms"]
        run.step_resident(st)
    assert contact_terms > 5000  # folded onto itself by then
