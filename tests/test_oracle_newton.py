"""The FP64 Newton-PCG oracle (src/solver.rs:422-646, extended with the
step's frozen OGC contacts) against known answers on the CPU: a free-falling
sheet lands exactly on its inertial target, and the VBD oracle converges
toward the Newton solution as its iteration count grows."""
import numpy as np

import oracle
from clothcraft_b200 import scenes


def test_free_fall_lands_on_the_inertial_target():
    mesh, x = scenes.sheet(10, 0.5, 0.3, scenes.Material.stvk_mapped())  # rest shape, no jitter
    sc = scenes.Scene("free_fall", mesh, None, x, np.zeros_like(x),
                      scenes.StepSettings(dt=1 / 60, iterations=20, damping=1.5, radius=0.002, stiffness=1e4), 1)
    st = sc.settings
    o = oracle.Solver(sc, threads=4)
    x, res, conv, its = o.newton_step(sc.x0, sc.v0, st.to_c(), abs_tol=1e-14, rel_tol=1e-8)
    y = sc.x0 + (sc.v0 * st.dt + np.array(st.gravity) * st.dt ** 2) / (1 + st.damping * st.dt)
    assert conv
    assert np.abs(x - y).max() <= 1e-9


def test_vbd_converges_toward_newton():
    sc = scenes.small_sheet(10, obstacle=False, pins=(0, 9))
    st = sc.settings
    # a stretched start so that the elastic terms matter
    x0 = sc.x0.copy()
    x0[:, 0] *= 1.02
    x0[sc.mesh.pinned.astype(bool)] = sc.mesh.pin_positions[sc.mesh.pinned.astype(bool)]
    o = oracle.Solver(sc, threads=4)
    xn, res, conv, its = o.newton_step(x0, sc.v0, st.to_c(), newton_iterations=50, pcg_iterations=500,
                                       abs_tol=1e-12, rel_tol=1e-10)
    assert conv
    errs = []
    for k in (5, 40, 200):
        s = sc.settings
        s.iterations = k
        v = oracle.Solver(sc, threads=4)
        xv, _, _, _ = v.step(x0, sc.v0, 0.0, s.to_c())
        errs.append(np.abs(xv - xn).max())
    assert errs[2] < errs[1] < errs[0]
    assert errs[2] < 0.5 * errs[0]
