"""The oracle's learned-guess pieces (CPU): the FP64 MLP gradient equals
central finite differences, and the features have the documented layout."""
import numpy as np

import oracle
from clothcraft_b200 import scenes


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(10115) * 0.1).astype(np.float32)
    f = rng.standard_normal((40, 24)).astype(np.float32)
    t = rng.standard_normal((40, 3)).astype(np.float32)
    g, loss = oracle.mlp_gradients(p, f, t)
    out = oracle.mlp_forward(p, f)
    assert abs(loss - np.mean(np.sum((out - t) ** 2, axis=1))) <= 1e-12 * loss

    def L(pp):
        return float(np.mean(np.sum((oracle.mlp_forward(pp, f) - t) ** 2, axis=1)))

    # one index per block: W1, b1, W2, b2, W3, b3, W4, b4
    for i in (0, 1540, 1700, 5700, 5800, 9990, 10000, 10113):
        e = 1e-2
        pp = p.copy()
        pp[i] += e
        hi = L(pp)
        pp[i] -= 2 * e
        lo = L(pp)
        fd = (hi - lo) / (2 * e)
        assert abs(fd - g[i]) <= 1e-3 * max(abs(g[i]), 1e-3), (i, fd, g[i])


def test_features_layout_on_a_resting_sheet():
    sc = scenes.small_sheet(12, height=0.3, pins=(0, 11))
    o = oracle.Solver(sc)
    F = o.learned_features(sc.x0, sc.v0, 0.0, sc.settings.to_c())
    assert F.shape == (sc.n - 2, 24)
    st = sc.settings
    # at rest with a fresh history: inertial displacement = guess = g dt^2 / (1 + c dt) / u
    expect = -1.0 / (1.0 + st.damping * st.dt)
    assert np.allclose(F[:, 1], expect, rtol=1e-6) and np.allclose(F[:, 4], expect, rtol=1e-6)
    assert np.allclose(F[:, 20:23], 0.0)  # no last-step correction without history
    assert np.allclose(np.abs(F[:, 13]), 1.0, atol=1e-6)  # flat sheet: normal along y
    assert np.all(F[:, 18] <= 1.0) and np.all(F[:, 18] > 0.0)
