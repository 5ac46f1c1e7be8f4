"""Relative residual and the residual-target iteration mode, on the GPU.

relative residual = ||P grad E(x)|| / ||grad E(y)|| over free vertices (E the
step objective with the step's OGC terms, y the inertial target, P the
projection that drops the outward normal part of the gradient at vertices on
the boundary of their OGC ball). The GPU value is compared with the oracle's
FP64 evaluation of the same rule, and the residual-target mode is
checked against fixed-iteration runs: it must stop exactly at the first
evaluation that meets the target and give the same bits as a fixed run of
that many iterations.
"""
import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.vbd import VbdSolver

pytestmark = pytest.mark.gpu

RESIDUAL_RTOL = 1e-9  # FP64 on both sides; only summation order differs


def contact_scene(n=16, seed=0):
    return scenes.small_sheet(n, seed=seed, height=0.104, side=0.2, pins=(), radius=0.002)


def settings(sc, iterations, check=1, tol=0.0):
    s = sc.settings
    s.iterations = iterations
    s.residual_check_every = check
    s.residual_tolerance = tol
    return s


def advance(sc, steps):
    """State after `steps` plain steps (contacts present in the contact scene)."""
    g = VbdSolver(sc)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(steps):
        x, v, t, _ = g.step(x, v, t, sc.settings.to_c())
    return x, v, t


@pytest.mark.parametrize("steps_before", [0, 12])
def test_relative_residual_matches_oracle(steps_before):
    """GPU residual = the oracle's restatement of the same rule (projected
    gradient over the OGC balls), and never above the unprojected force norm
    of the FP64 Newton oracle's objective."""
    sc = contact_scene()
    x0, v0, t0 = advance(sc, steps_before)
    st = settings(sc, 12, check=4)
    g = VbdSolver(sc)
    x, v, t, m = g.step(x0, v0, t0, st.to_c())
    assert m["relative_residual"] is not None
    o = oracle.Solver(sc, threads=8)
    xo, _, _, mo = o.step(x0, v0, t0, st.to_c())
    assert np.abs(x - xo).max() <= 1e-12
    for key in ("relative_residual", "initial_relative_residual"):
        assert abs(m[key] - mo[key]) <= RESIDUAL_RTOL * mo[key]
    if m["detection_updates"] == 1:  # the Newton oracle evaluates with the step-start contacts
        o2 = oracle.Solver(sc, threads=8)
        unprojected = o2.relative_residual(x0, v0, st.to_c(), x)
        assert m["relative_residual"] <= unprojected * (1 + 1e-9)
    # the residual falls with iterations
    assert m["relative_residual"] < m["initial_relative_residual"]


def test_no_residual_unless_requested():
    sc = contact_scene()
    g = VbdSolver(sc)
    _, _, _, m = g.step(sc.x0, sc.v0, 0.0, sc.settings.to_c())
    assert m["relative_residual"] is None


def test_residual_target_stops_at_first_evaluation_below_it():
    sc = contact_scene()
    x0, v0, t0 = advance(sc, 3)
    # residuals of fixed runs of k iterations
    res = {}
    for k in (2, 4, 6, 8, 10):
        g = VbdSolver(sc)
        _, _, _, m = g.step(x0, v0, t0, settings(sc, k, check=2).to_c())
        res[k] = m["relative_residual"]
    tol = 0.5 * (res[6] + res[8])  # met first at k = 8
    assert res[6] > tol >= res[8]
    g = VbdSolver(sc).set_lanes(4)  # bitwise comparison: same lanes in both solvers
    xa, va, _, ma = g.step(x0, v0, t0, settings(sc, 60, check=2, tol=tol).to_c())
    assert ma["iterations"] == 8
    assert ma["relative_residual"] <= tol
    g2 = VbdSolver(sc).set_lanes(4)
    xb, vb, _, mb = g2.step(x0, v0, t0, settings(sc, 8, check=2).to_c())
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert ma["relative_residual"] == mb["relative_residual"]
    assert ma["vertex_solves"] == mb["vertex_solves"]


def test_residual_target_on_the_fold_state_with_refreshes():
    """Fold-phase 256x256 state: the target mode with refresh detections
    running ahead on the device gives the bits of the fixed run."""
    sc = scenes.config1()
    z = np.load(scenes_fold_state())
    x0, v0 = z["x"].astype(np.float64), z["v"].astype(np.float64)
    t0 = 200 / 60
    g = VbdSolver(sc).set_lanes(4)  # bitwise comparison: same lanes in both solvers
    g.set_state(x0, v0, t0)
    ma = g.step_resident(settings(sc, 120, check=5, tol=2e-3).to_c())
    xa, va, _ = g.get_state()
    k = ma["iterations"]
    assert k % 5 == 0 and ma["relative_residual"] <= 2e-3 or k == 120
    g2 = VbdSolver(sc).set_lanes(4)
    g2.set_state(x0, v0, t0)
    mb = g2.step_resident(settings(sc, k, check=5).to_c())
    xb, vb, _ = g2.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert ma["detection_updates"] == mb["detection_updates"]


def scenes_fold_state():
    import os

    return os.path.join(os.path.dirname(__file__), "golden", "sheet256_fold_state.npz")


@pytest.mark.parametrize("tol,stall,rho", [(2e-2, 0, 0.0), (1e-4, 0, 0.0), (1e-4, 2, 0.0), (1e-4, 2, 0.5),
                                          (1e-4, 2, 0.8), (2e-2, 0, 0.95), (1e-4, 2, 0.95), (1e-4, 0, 0.95)])
def test_residual_target_matches_oracle(tol, stall, rho):
    """Same stopping iteration, refresh count and positions as the oracle's
    restatement of the residual-target rule, with and without the stall
    refresh and the Chebyshev acceleration with its restarts (FP64 both;
    bar (a) on positions)."""
    sc = contact_scene()
    x0, v0, t0 = advance(sc, 3)
    s = settings(sc, 60, check=2, tol=tol)
    s.stall_refresh = stall
    s.acceleration = rho
    st = s.to_c()
    g = VbdSolver(sc).set_lanes(4)
    x, _, _, m = g.step(x0, v0, t0, st)
    o = oracle.Solver(sc, threads=8)
    xo, _, _, mo = o.step(x0, v0, t0, st)
    assert m["iterations"] == mo["iterations"]
    assert m["detection_updates"] == mo["detection_updates"]
    if tol > 1e-3:
        assert m["iterations"] < 60
    assert np.abs(x - xo).max() <= 1e-5
    assert abs(m["relative_residual"] - mo["relative_residual"]) <= 1e-6 * mo["relative_residual"]
    assert abs(m["initial_relative_residual"] - mo["initial_relative_residual"]) <= 1e-6 * mo["initial_relative_residual"]


def test_last_step_trace_records_every_evaluation():
    sc = contact_scene()
    x0, v0, t0 = advance(sc, 3)
    g = VbdSolver(sc)
    _, _, _, m = g.step(x0, v0, t0, settings(sc, 9, check=3).to_c())
    r, c = g.last_step_trace()
    assert np.isnan(r[0]) and np.isnan(r[1]) and np.isfinite(r[2]) and np.isfinite(r[5]) and np.isfinite(r[8])
    assert r[8] == m["relative_residual"] or abs(r[8] - m["relative_residual"]) <= 1e-15 * r[8]
    assert int(c[:9].sum()) == m["truncated_vertices"]


def test_acceleration_fixed_iterations_match_oracle_and_keep_the_trust_region():
    """Chebyshev acceleration over a fixed iteration count: positions within
    bar (a) of the oracle's for three steps, every vertex inside its OGC ball
    (the step fails its trust-region check otherwise), and the weights act."""
    sc = contact_scene()
    x0, v0, t0 = advance(sc, 3)
    s = settings(sc, 24)
    s.acceleration = 0.9
    st = s.to_c()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    xg, vg, tg, xo, vo, to = x0, v0, t0, x0, v0, t0
    for _ in range(3):
        xg, vg, tg, mg = g.step(xg, vg, tg, st)
        xo, vo, to, mo = o.step(xo, vo, to, st)
        assert mg["detection_updates"] == mo["detection_updates"]
        assert np.abs(xg - xo).max() <= 1e-5
    plain = settings(sc, 24)
    plain.acceleration = 0.0
    xp, _, _, _ = VbdSolver(sc).step(x0, v0, t0, plain.to_c())
    xa, _, _, _ = VbdSolver(sc).step(x0, v0, t0, st)
    assert np.abs(xa - xp).max() > 0.0


def test_acceleration_out_of_range_is_rejected():
    sc = contact_scene()
    g = VbdSolver(sc)
    for rho in (1.0, -0.1, float("nan")):
        s = settings(sc, 4)
        s.acceleration = rho
        with pytest.raises(Exception):
            g.step(sc.x0, sc.v0, 0.0, s.to_c())
