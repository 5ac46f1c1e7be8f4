"""GPU VBD step parity against the oracle, through the C ABI.

Bars (from the hot-path contract):
  (a) per-vertex positions after one step within 1e-5 m of the CPU path;
  (b) energy and force residual within 1 % after many steps;
  plus the reference's own VBD known-answer tests run on the GPU backend.
Local blocks (energy, gradient, Hessian) and colourings are compared at
identical positions: colours exactly, blocks to 1e-9 relative.
"""
import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.vbd import VbdError, VbdSolver

pytestmark = pytest.mark.gpu

POSITION_TOL_M = 1e-5      # (a)
RELATIVE_TOL = 0.01        # (b)
BLOCK_RTOL = 1e-9


def contact_scene(n=16, seed=0):
    """Small sheet 4 mm above a sphere so contacts appear within a few steps."""
    return scenes.small_sheet(n, seed=seed, height=0.104, side=0.2, pins=(), radius=0.002)


def run_both(sc, steps, settings=None):
    st = (settings or sc.settings).to_c()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    xg, vg, tg = sc.x0.copy(), sc.v0.copy(), 0.0
    xo, vo, to = sc.x0.copy(), sc.v0.copy(), 0.0
    out = []
    for _ in range(steps):
        xg, vg, tg, mg = g.step(xg, vg, tg, st)
        xo, vo, to, mo = o.step(xo, vo, to, st)
        out.append((xg.copy(), xo.copy(), mg, mo))
    return out, g, o


def test_local_blocks_match_oracle_jet_ad():
    sc = contact_scene()
    g = VbdSolver(sc)
    o = oracle.Solver(sc)
    rng = np.random.default_rng(0)
    st = sc.settings.to_c()
    x = sc.x0.copy()
    x[:, 1] -= 0.0035
    x += rng.uniform(-3e-4, 3e-4, x.shape)
    x_all = g.positions(x)
    targets = x + rng.uniform(-1e-3, 1e-3, x.shape)
    inertia = sc.mesh.masses * (1 + 1.5 / 60) * 3600
    eg, gg, hg = g.local_blocks(x_all, 0.008, st, targets=targets, inertia=inertia)
    eo, go, ho = o.local_blocks(x_all, 0.008, st, targets=targets, inertia=inertia)
    assert np.all(np.abs(eg - eo) <= BLOCK_RTOL * np.maximum(np.abs(eo), 1e-12))
    gscale = np.linalg.norm(go, axis=1, keepdims=True) + 1e-12
    assert np.all(np.abs(gg - go) <= BLOCK_RTOL * gscale + 1e-15)
    hscale = np.abs(ho).max(axis=(1, 2), keepdims=True) + 1e-12
    assert np.all(np.abs(hg - ho) <= BLOCK_RTOL * hscale)


def test_local_blocks_with_grab_and_default_fabric():
    sc = scenes.demo_left_panel(3, 4)
    g = VbdSolver(sc)
    o = oracle.Solver(sc)
    rng = np.random.default_rng(1)
    x = sc.x0 + rng.uniform(-0.01, 0.01, sc.x0.shape)
    grab = dict(vertices=[0, 5, 6], weights=[0.2, 0.3, 0.5], target=[0.0, 0.9, 0.05], stiffness=100.0)
    st = sc.settings.to_c()
    eg, gg, hg = g.local_blocks(x, 0.01, st, grab=grab)
    eo, go, ho = o.local_blocks(x, 0.01, st, grab=grab)
    assert np.allclose(eg, eo, rtol=BLOCK_RTOL, atol=1e-15)
    assert np.allclose(gg, go, rtol=1e-8, atol=1e-12 * np.abs(go).max())
    assert np.allclose(hg, ho, rtol=1e-8, atol=1e-12 * np.abs(ho).max())


def test_coloring_matches_sequential_greedy():
    sc = contact_scene(20)
    g = VbdSolver(sc)
    o = oracle.Solver(sc)
    x = sc.x0.copy()
    x[:, 1] -= 0.0037
    x_all = g.positions(x)
    grab = dict(vertices=[0, 21, 22], weights=[0.2, 0.3, 0.5], target=[0.0, 0.2, 0.0], stiffness=100.0)
    for gr in (None, grab):
        cg, ng = g.colors(x_all, 0.008, sc.settings, grab=gr)
        co, no = o.colors(x_all, 0.008, sc.settings.ogc_c(), grab=gr)
        assert ng == no
        assert np.array_equal(cg, co)


def test_coloring_matches_sequential_greedy_above_the_shared_memory_size():
    """102,400 vertices (more than the 92,160 colours the walk keeps in shared
    memory, so colours stay in global memory) folded into two layers 1 mm
    apart: ~10^5 contact co-vertex edges between the layers."""
    sc = scenes.small_sheet(320, seed=1, obstacle=False, side=1.0, radius=0.0005, pins=())
    x = sc.x0.copy()
    right = x[:, 0] > 0.0
    x[right, 0] = -x[right, 0]
    x[right, 1] += 0.001
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    x_all = g.positions(x)
    cg, ng = g.colors(x_all, 0.002, sc.settings)
    co, no = o.colors(x_all, 0.002, sc.settings.ogc_c())
    assert ng == no and ng > 4
    assert np.array_equal(cg, co)
    # again from the previous colouring, after a small displacement
    x[::7, 1] += 2e-4
    x_all = g.positions(x)
    cg, ng = g.colors(x_all, 0.002, sc.settings)
    co, no = o.colors(x_all, 0.002, sc.settings.ogc_c())
    assert ng == no and np.array_equal(cg, co)


@pytest.mark.parametrize("maker", [lambda: scenes.small_sheet(16, seed=2),
                                   lambda: contact_scene(16, seed=4)])
def test_one_step_positions_within_1e5_m(maker):
    sc = maker()
    # advance a state with the oracle so contact is exercised, then step it
    # once with two fresh solvers (neither has adaptive-init history)
    o = oracle.Solver(sc, threads=8)
    st = sc.settings.to_c()
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(3):
        x, v, t, _ = o.step(x, v, t, st)
    g = VbdSolver(sc)
    o2 = oracle.Solver(sc, threads=8)
    xg, vg, tg, mg = g.step(x, v, t, st)
    xo, vo, to, mo = o2.step(x, v, t, st)
    err = np.linalg.norm(xg - xo, axis=1).max()
    assert err <= POSITION_TOL_M, err
    assert tg == to
    assert mg["contact_terms"] == mo["contact_terms"]
    assert mg["detection_updates"] == mo["detection_updates"]


def test_stepping_with_history_stays_within_1e5_m():
    """Both solvers advance their own trajectories (adaptive-init history
    active from step 2 on); per-step deviation stays within bar (a)."""
    sc = contact_scene(16, seed=9)
    out, _, _ = run_both(sc, 8)
    for k, (xg, xo, mg, mo) in enumerate(out):
        err = np.linalg.norm(xg - xo, axis=1).max()
        assert err <= POSITION_TOL_M, (k, err)


def test_config0_one_step_parity():
    sc = scenes.config0()
    out, _, _ = run_both(sc, 1)
    xg, xo, mg, mo = out[0]
    err = np.linalg.norm(xg - xo, axis=1).max()
    assert err <= POSITION_TOL_M, err
    assert mg["contact_terms"] == mo["contact_terms"]
    assert mg["colors"] == mo["colors"]


def test_many_steps_energy_and_residual_within_one_percent():
    sc = contact_scene(16, seed=6)
    out, g, o = run_both(sc, 40)
    xg, xo, mg, mo = out[-1]
    for key in ("residual_rms_n",):
        assert abs(mg[key] - mo[key]) <= RELATIVE_TOL * abs(mo[key]) + 1e-12, (mg[key], mo[key])
    # total potential (membrane + bending + contact) via the oracle's blocks at each final state
    st = sc.settings.to_c()
    eg = o.local_blocks(o.positions(xg), 0.008, st)[0].sum()
    eo = o.local_blocks(o.positions(xo), 0.008, st)[0].sum()
    assert abs(eg - eo) <= RELATIVE_TOL * abs(eo), (eg, eo)


def test_config0_hundred_steps_energy_and_residual_within_one_percent():
    """Bar (b) on config 0 (64x64 sheet, two pinned corners, r = 0.1 m
    icosphere, 20 iterations): after 100 steps of each side's own trajectory
    the potential energy, the reference's residual_rms_n and the relative
    force residual agree within 1 %. The residual is evaluated once, after the
    last iteration of every step, which does not change the iterates."""
    sc = scenes.config0()
    s = sc.settings
    s.residual_check_every = s.iterations
    out, g, o = run_both(sc, 100, s)
    xg, xo, mg, mo = out[-1]
    assert mg["contact_terms"] > 0 and mo["contact_terms"] > 0  # draped over the sphere by then
    for key in ("residual_rms_n", "relative_force_residual", "relative_residual"):
        assert abs(mg[key] - mo[key]) <= RELATIVE_TOL * abs(mo[key]), (key, mg[key], mo[key])
    st = s.to_c()
    grav = np.array(st.gravity)

    def potential(x):  # elastic + contact (oracle blocks, each term per incident vertex) + gravity
        blocks = o.local_blocks(o.positions(x), 4 * st.contact.radius, st)[0].sum()
        return blocks - float((sc.mesh.masses[:, None] * x * grav).sum())

    eg, eo = potential(xg), potential(xo)
    assert abs(eg - eo) <= RELATIVE_TOL * abs(eo), (eg, eo)


# ---------------------------------------------------- reference known answers
def test_resting_contact_settles_without_sawtooth_on_gpu():  # tests/vbd.rs:10-34
    for offset in ((0.0, 0.0, 0.0), (100.0, 101.4, -100.0)):
        sc = scenes.resting_patch(offset)
        s = VbdSolver(sc)
        st = sc.settings.to_c()
        x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
        max_delta = 0.0
        for i in range(60):
            old = x.copy()
            x, v, t, _ = s.step(x, v, t, st)
            assert np.all(np.abs(x[:, 1] - offset[1] - st.contact.radius) < 1e-5), (i, x[:, 1])
            if i > 10:
                max_delta = max(max_delta, float(np.abs(x[:, 1] - old[:, 1]).max()))
        assert max_delta < 1e-6


def test_free_fall_matches_backward_euler_on_gpu():  # tests/vbd.rs:44-61
    sc = scenes.demo_left_panel()
    s = VbdSolver(sc)
    st = scenes.StepSettings(dt=0.005, damping=0.0, iterations=3).to_c()
    x, v, t, _ = s.step(sc.x0, sc.v0, 0.0, st)
    g = np.array([0.0, -9.81, 0.0])
    assert np.all(np.linalg.norm(v - g * 0.005, axis=1) < 1e-9)
    assert np.all(np.linalg.norm(x - sc.x0 - g * 0.005 ** 2, axis=1) < 1e-12)


def test_grab_pulls_and_invalid_input_is_transactional_on_gpu():  # tests/vbd.rs:62-91
    sc = scenes.demo_left_panel()
    s = VbdSolver(sc)
    tri = sc.mesh.triangles[0]
    center = sum(sc.x0[i] / 3.0 for i in tri)
    grab = dict(vertices=tri, weights=[1 / 3] * 3, target=center + np.array([0, 0, 0.01]), stiffness=100.0)
    st = scenes.StepSettings(gravity=(0.0, 0.0, 0.0), iterations=6).to_c()
    x, v, t, _ = s.step(sc.x0, sc.v0, 0.0, st, grab)
    assert sum(x[i] / 3.0 for i in tri)[2] > center[2]
    x_before, t_before = x.copy(), t
    with pytest.raises(VbdError):
        s.step(x, v, t, st, dict(grab, target=np.array([np.nan, 0, 0])))
    # the caller's arrays are untouched and the solver still steps
    assert np.array_equal(x, x_before) and t == t_before
    s.step(x, v, t, st, grab)


def test_invalid_settings_and_state_are_rejected_on_gpu():
    sc = scenes.demo_left_panel()
    s = VbdSolver(sc)
    with pytest.raises(VbdError):
        s.step(sc.x0, sc.v0, 0.0, scenes.StepSettings(dt=0.1).to_c())
    v = sc.v0.copy()
    v[0, 0] = np.inf
    with pytest.raises(VbdError):
        s.step(sc.x0, v, 0.0, scenes.StepSettings().to_c())


def test_resident_stepping_equals_host_stepping():
    sc = contact_scene(12, seed=8)
    st = sc.settings.to_c()
    a = VbdSolver(sc).set_lanes(4)  # bitwise comparison: same lanes in both solvers
    b = VbdSolver(sc).set_lanes(4)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    b.set_state(x, v, t)
    for _ in range(5):
        x, v, t, _ = a.step(x, v, t, st)
        b.step_resident(st)
    xb, vb, tb = b.get_state()
    assert np.array_equal(x, xb) and np.array_equal(v, vb) and t == tb


@pytest.mark.parametrize("lanes", [4, 8, 16])
def test_register_caps_give_identical_steps(lanes):
    """The register cap (resident blocks per SM, with local-memory spills above
    3) changes only the schedule: every cap gives the bits of cap 3."""
    sc = contact_scene(12, seed=8)
    st = sc.settings.to_c()
    ref = VbdSolver(sc).set_lanes(lanes | 3 << 8)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    ref.set_state(x, v, t)
    for _ in range(3):
        ref.step_resident(st)
    xr, vr, _ = ref.get_state()
    for cap in (4, 5, 6, 8):
        s = VbdSolver(sc).set_lanes(lanes | cap << 8)
        s.set_state(x, v, t)
        for _ in range(3):
            s.step_resident(st)
        xs, vs, _ = s.get_state()
        assert np.array_equal(xs, xr) and np.array_equal(vs, vr), cap


def test_invalid_register_cap_is_rejected():
    s = VbdSolver(contact_scene(8, seed=1))
    for bad in (4 | 7 << 8, 4 | 2 << 8, 4 | 9 << 8, 3, 0 | 4 << 8):
        with pytest.raises(VbdError):
            s.set_lanes(bad)


def test_step_into_pinned_arrays_equals_step():
    """In-place stepping on pinned host arrays (the caller's memory is copied
    as it is and converted on the GPU) gives the bits of `step`, and a failed
    step leaves the caller's arrays untouched."""
    import torch

    sc = contact_scene(12, seed=8)
    st = sc.settings.to_c()
    a = VbdSolver(sc).set_lanes(4)
    b = VbdSolver(sc).set_lanes(4)
    xh = torch.empty((sc.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    vh = torch.empty((sc.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    xh[:], vh[:] = sc.x0, sc.v0
    x, v, ta, tb = sc.x0.copy(), sc.v0.copy(), 0.0, 0.0
    for _ in range(4):
        x, v, ta, _ = a.step(x, v, ta, st)
        tb, _ = b.step_into(xh, vh, tb, st)
    assert np.array_equal(x, xh) and np.array_equal(v, vh) and ta == tb
    before = (xh.copy(), vh.copy())
    with pytest.raises(VbdError):
        b.step_into(xh, vh, tb, scenes.StepSettings(dt=0.1).to_c())
    assert np.array_equal(xh, before[0]) and np.array_equal(vh, before[1])
    with pytest.raises(ValueError):
        b.step_into(xh[:, :2], vh, tb, st)


PERSISTENT, B64, B256 = 1 << 16, 1 << 17, 2 << 17


@pytest.mark.parametrize("fp32,lanes", [(False, 4), (False, 8), (True, 8), (True, 16)])
def test_persistent_grids_and_block_sizes_give_identical_steps(fp32, lanes):
    """A persistent grid (each block looping over the colour's vertices) and
    blocks of 64 or 256 threads change only the schedule: on the fold state,
    where a colour has ~16k vertices and the persistent grid loops, every
    variant gives the bits of the 128-thread one-pass grid."""
    import os

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sheet256_fold_state.npz"))
    x, v, t = z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])
    sc = scenes.config1()
    s = sc.settings
    s.iterations = 6
    s.sweep_precision = 1 if fp32 else 0
    st = s.to_c()

    def run(variant):
        g = VbdSolver(sc)
        (g.set_lanes32 if fp32 else g.set_lanes)(variant)
        g.set_state(x, v, t)
        for _ in range(2):
            g.step_resident(st)
        return g.get_state()

    xr, vr, _ = run(lanes | 4 << 8)
    for extra in (PERSISTENT, B64, B256, B64 | PERSISTENT):
        xs, vs, _ = run(lanes | 4 << 8 | extra)
        assert np.array_equal(xs, xr) and np.array_equal(vs, vr), extra


def test_invalid_block_variants_are_rejected():
    s = VbdSolver(contact_scene(8, seed=1))
    for bad in (16 | 4 << 8 | B64, 2 | 4 << 8 | B256, 8 | 5 << 8 | B64, 8 | 4 << 8 | 3 << 17, 8 | 4 << 8 | 1 << 19):
        with pytest.raises(VbdError):
            s.set_lanes(bad)
    for bad in (4 | 4 << 8 | B64, 32 | 4 << 8 | B256):
        with pytest.raises(VbdError):
            s.set_lanes32(bad)


@pytest.mark.parametrize("target", [False, True])
def test_graph_launches_give_the_bits_of_direct_launches(target):
    """CUDA-graph chunks (captured, updated in place or re-instantiated when
    a colouring changes the topology) against direct launches on the fold
    state: fixed iterations, and the residual target with acceleration,
    stall refreshes and the chunked look-ahead."""
    import os

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sheet256_fold_state.npz"))
    x, v, t = z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])
    sc = scenes.config1()
    s = sc.settings
    if target:
        s.iterations, s.residual_tolerance, s.residual_check_every, s.stall_refresh = 200, 1e-3, 2, 2
        s.acceleration = 0.95
    st = s.to_c()
    out = []
    for graphs in (False, True):
        g = VbdSolver(sc).set_lanes(8 | 4 << 8).set_graphs(graphs)
        g.set_state(x, v, t)
        its = [g.step_resident(st)["iterations"] for _ in range(3)]
        out.append((g.get_state(), its))
    (xa, va, _), ia = out[0]
    (xb, vb, _), ib = out[1]
    assert ia == ib
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
