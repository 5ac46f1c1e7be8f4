"""Relative residual and the residual-target iteration mode, on the GPU.

relative residual = ||grad E(x)|| / ||grad E(y)|| over free vertices (E the
step objective with the step's OGC terms, y the inertial target). The GPU
value is compared with the oracle's FP64 evaluation at the same positions
(contacts detected at the step start, frozen), and the residual-target mode is
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


@pytest.mark.parametrize("steps_before", [0, 3])
def test_relative_residual_matches_oracle(steps_before):
    sc = contact_scene()
    x0, v0, t0 = advance(sc, steps_before)
    st = settings(sc, 12, check=4)
    g = VbdSolver(sc)
    x, v, t, m = g.step(x0, v0, t0, st.to_c())
    assert m["relative_residual"] is not None
    assert m["detection_updates"] == 1, "a refresh changes the contact set; pick a calmer state"
    o = oracle.Solver(sc, threads=8)
    ref = o.relative_residual(x0, v0, st.to_c(), x)
    assert abs(m["relative_residual"] - ref) <= RESIDUAL_RTOL * ref
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
    g = VbdSolver(sc)
    xa, va, _, ma = g.step(x0, v0, t0, settings(sc, 60, check=2, tol=tol).to_c())
    assert ma["iterations"] == 8
    assert ma["relative_residual"] <= tol
    g2 = VbdSolver(sc)
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
    g = VbdSolver(sc)
    g.set_state(x0, v0, t0)
    ma = g.step_resident(settings(sc, 120, check=5, tol=2e-3).to_c())
    xa, va, _ = g.get_state()
    k = ma["iterations"]
    assert k % 5 == 0 and ma["relative_residual"] <= 2e-3 or k == 120
    g2 = VbdSolver(sc)
    g2.set_state(x0, v0, t0)
    mb = g2.step_resident(settings(sc, k, check=5).to_c())
    xb, vb, _ = g2.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    assert ma["detection_updates"] == mb["detection_updates"]


def scenes_fold_state():
    import os

    return os.path.join(os.path.dirname(__file__), "golden", "sheet256_fold_state.npz")
