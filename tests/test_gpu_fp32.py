"""The FP32-assembly sweep (cc_vbd_settings.sweep_precision = CC_SWEEP_FP32)
against the oracle, the FP64 restatement of the reference CPU path.

The FP32 form rounds every element's edge vectors once to FP32 and assembles
membrane and bending derivatives in FP32, so its iterates are not the CPU
path's bits; the bars are the contract's tolerances instead:
  (a) per-vertex positions after one step within 1e-5 m (fixed iteration
      counts, so both sides run the same number of sweeps);
  (b) energy and residual_rms_n within 1 % after 100 steps of each side's
      own trajectory (config 0), and the relative force residual inside the
      spread of FP64 runs from starts 1e-12..1e-8 m apart (that quantity is
      chaotic in the trajectory);
  and on the benchmarked fold the residual target (1e-3, evaluated in FP64)
  is reached in about as many iterations as the FP64 form needs.
"""
import os

import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.abi import CC_SWEEP_FP32
from clothcraft_b200.vbd import VbdSolver

pytestmark = pytest.mark.gpu

POSITION_TOL_M = 1e-5  # bar (a)
RELATIVE_TOL = 0.01    # bar (b)
THREADS = os.cpu_count() or 1
FOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sheet256_fold_state.npz")


def fp32(settings):
    settings.sweep_precision = CC_SWEEP_FP32
    return settings


def contact_scene(n=16, seed=0):
    return scenes.small_sheet(n, seed=seed, height=0.104, side=0.2, pins=(), radius=0.002)


@pytest.mark.parametrize("lanes", [4 | 3 << 8, 8 | 4 << 8, 16 | 3 << 8, 32 | 3 << 8])
def test_fp32_step_within_1e5_m_of_oracle_in_contact(lanes):
    sc = contact_scene(16, seed=4)
    o = oracle.Solver(sc, threads=THREADS)
    st = sc.settings.to_c()
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(4):
        x, v, t, _ = o.step(x, v, t, st)
    g = VbdSolver(sc).set_lanes32(lanes)
    xg, _, _, mg = g.step(x, v, t, fp32(sc.settings).to_c())
    xo, _, _, mo = oracle.Solver(sc, threads=THREADS).step(x, v, t, st)
    assert mo["contact_terms"] > 0
    err = float(np.linalg.norm(xg - xo, axis=1).max())
    assert err <= POSITION_TOL_M, err
    assert mg["detection_updates"] == mo["detection_updates"]


def test_fp32_config0_step_within_1e5_m_of_oracle():
    sc = scenes.config0()
    xg, _, _, mg = VbdSolver(sc).step(sc.x0, sc.v0, 0.0, fp32(sc.settings).to_c())
    xo, _, _, mo = oracle.Solver(sc, threads=THREADS).step(sc.x0, sc.v0, 0.0, scenes.config0().settings.to_c())
    err = float(np.linalg.norm(xg - xo, axis=1).max())
    assert err <= POSITION_TOL_M, err
    assert mg["colors"] == mo["colors"]


def fp64_ensemble_residuals(sc, steps, perturbations, seed=7):
    """Relative force residual of the last step after `steps` FP64 steps from
    the scene's start with every free vertex displaced by `eps` times a seeded
    standard normal (one run per eps; eps = 0 is the unperturbed run)."""
    s = sc.settings
    s.residual_check_every = s.iterations
    s.sweep_precision = 0
    st = s.to_c()
    free = sc.mesh.pinned[:, None] == 0
    out = []
    for eps in perturbations:
        rng = np.random.default_rng(seed)
        x = sc.x0 + eps * rng.standard_normal(sc.x0.shape) * free
        v, t = sc.v0.copy(), 0.0
        g = VbdSolver(sc)
        for _ in range(steps):
            x, v, t, m = g.step(x, v, t, st)
        out.append(m["relative_force_residual"])
    return out


def test_fp32_config0_hundred_steps_energy_and_residual():
    """Bar (b) for the FP32 form: after 100 steps of each side's own
    trajectory the potential energy and the reference's residual_rms_n agree
    with the FP64 CPU path within 1 %.

    The relative force residual of a 20-iteration step is not a quantity two
    trajectories can agree on to 1 % unless they are the same to the last
    bits: the sheet's contact with the sphere makes the trajectory chaotic, so
    FP64 runs whose starts differ by 1e-12 m end 100 steps later several
    millimetres apart, with relative force residuals from 0.005 to 0.1
    (measured on a B200: 0.068, 0.067, 0.0046 and 0.097 for displacements of
    0, 1e-12, 1e-10 and 1e-8 m), while the FP32 run gave 0.059. The test
    therefore pins that spread and checks that the FP32 value lies inside the
    range of the FP64 runs (widened by 25 %)."""
    sc = scenes.config0()
    s = sc.settings
    s.residual_check_every = s.iterations
    st64 = s.to_c()
    st32 = fp32(s).to_c()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=THREADS)
    xg, vg, tg = sc.x0.copy(), sc.v0.copy(), 0.0
    xo, vo, to = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(100):
        xg, vg, tg, mg = g.step(xg, vg, tg, st32)
        xo, vo, to, mo = o.step(xo, vo, to, st64)
    assert mo["contact_terms"] > 0
    assert abs(mg["residual_rms_n"] - mo["residual_rms_n"]) <= RELATIVE_TOL * abs(mo["residual_rms_n"])
    grav = np.array(st64.gravity)

    def potential(x):
        blocks = o.local_blocks(o.positions(x), 4 * st64.contact.radius, st64)[0].sum()
        return blocks - float((sc.mesh.masses[:, None] * x * grav).sum())

    eg, eo = potential(xg), potential(xo)
    assert abs(eg - eo) <= RELATIVE_TOL * abs(eo), (eg, eo)
    # the spread of the FP64 path itself under starts 1e-12..1e-8 m apart
    ens = fp64_ensemble_residuals(scenes.config0(), 100, (0.0, 1e-12, 1e-10, 1e-8))
    print("relative force residual after 100 steps: fp32 %.4g, fp64 oracle %.4g, fp64 ensemble %s" % (
        mg["relative_force_residual"], mo["relative_force_residual"], ["%.4g" % r for r in ens]))
    assert abs(ens[0] - mo["relative_force_residual"]) <= RELATIVE_TOL * mo["relative_force_residual"]
    assert max(ens) > 1.1 * min(ens), ens  # the quantity does not survive a 1e-12 m change of the start
    assert 0.8 * min(ens) <= mg["relative_force_residual"] <= 1.25 * max(ens), (mg["relative_force_residual"], ens)


def fold_state():
    z = np.load(FOLD)
    return z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])


def test_fp32_fold_fixed_iterations_within_1e5_m_of_oracle():
    """The reference's fixed 30-iteration step on the fold state (~95k
    contact terms): FP32 assembly against the FP64 CPU path."""
    sc = scenes.config1()
    x, v, t = fold_state()
    st = sc.settings.to_c()
    xg, _, _, mg = VbdSolver(sc).step(x, v, t, fp32(scenes.config1().settings).to_c())
    xo, _, _, mo = oracle.Solver(sc, threads=THREADS).step(x, v, t, st)
    err = float(np.linalg.norm(xg - xo, axis=1).max())
    assert err <= POSITION_TOL_M, err
    # refresh detections run at iterates ~1e-7 m apart, so terms right at the
    # query radius may differ by a few; the detection count may not
    assert mg["detection_updates"] == mo["detection_updates"]
    assert abs(mg["contact_terms"] - mo["contact_terms"]) <= 1e-3 * mo["contact_terms"]


def test_fp32_fold_reaches_the_residual_target_like_fp64():
    """At the benchmark's target (1e-3 relative residual, FP64 evaluation,
    acceleration 0.95, stall refresh 2) the FP32 form converges on each of
    three fold steps, in iteration counts close to the FP64 form's."""
    sc = scenes.config1()
    x, v, t = fold_state()
    s = sc.settings
    s.iterations, s.residual_tolerance, s.residual_check_every, s.stall_refresh = 200, 1e-3, 2, 2
    s.acceleration = 0.95
    st64 = s.to_c()
    st32 = fp32(s).to_c()
    a, b = VbdSolver(sc), VbdSolver(sc)
    a.set_state(x, v, t)
    b.set_state(x, v, t)
    its32, its64 = [], []
    for _ in range(3):
        m32 = a.step_resident(st32)
        m64 = b.step_resident(st64)
        assert m32["relative_residual"] <= 1e-3 and m64["relative_residual"] <= 1e-3
        its32.append(m32["iterations"])
        its64.append(m64["iterations"])
    assert sum(its32) <= 1.25 * sum(its64) + 4, (its32, its64)
