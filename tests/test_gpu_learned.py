"""Learned initial guess on the GPU: MLP kernels against the FP64 oracle,
features against the oracle's restatement, the solver's learned mode with its
energy-checked scale search and fallback, and that a guess fitted to the
solver's own converged steps is taken and starts closer to the solution.

Tolerances: FP32 inference 1e-5 relative to the output scale (FP32 sums of 64
terms); FP16-operand tensor-core inference 1e-2 of the output scale (FP16
activations and weights, 11-bit significands, FP32 accumulation); gradients
1e-4 relative in the L2 norm (FP32 sums over hundreds of samples); features
1e-5 relative (FP64 on both sides, rounded once to float32).
"""
import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.learned import Mlp
from clothcraft_b200.vbd import VbdSolver

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

FP32_RTOL = 1e-5
TC_RTOL = 1e-2
GRAD_RTOL = 1e-4
FEATURE_RTOL = 1e-5  # identical inputs; 1e-4 where the two trajectories differ by ~1e-15 m


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def random_net(seed, scale=0.25):
    rng = np.random.default_rng(seed)
    m = Mlp(seed)
    p = m.parameters()
    p += (rng.standard_normal(p.size) * scale * 0.2).astype(np.float32)  # non-zero biases too
    m.set_parameters(p)
    return m, p


@pytest.mark.parametrize("n", [1, 127, 1000, 4099])
def test_forward_fp32_matches_oracle(n):
    m, p = random_net(1)
    f = np.random.default_rng(n).standard_normal((n, 24)).astype(np.float32)
    out = m.forward(cuda(f), precision=0).cpu().numpy()
    ref = oracle.mlp_forward(p, f)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(out - ref).max() <= FP32_RTOL * scale


@pytest.mark.parametrize("n", [1, 128, 1000, 70001])
def test_forward_tensor_cores_matches_oracle(n):
    m, p = random_net(2)
    f = np.random.default_rng(n).standard_normal((n, 24)).astype(np.float32)
    out = m.forward(cuda(f), precision=1).cpu().numpy()
    ref = oracle.mlp_forward(p, f)
    scale = max(1.0, np.abs(ref).max())
    err = np.abs(out - ref).max()
    assert err <= TC_RTOL * scale, err


def test_kernels_run_after_the_device_is_selected_again():
    """The MLP kernels raise their dynamic shared-memory limit on the device
    current at each launch (the limit is a per-device attribute): after
    cc_set_device selects the device again, tcgen05 and FP32 inference still
    run and match the oracle."""
    from clothcraft_b200 import native

    L = native.load()
    m, p = random_net(3)
    f = np.random.default_rng(5).standard_normal((777, 24)).astype(np.float32)
    ref = oracle.mlp_forward(p, f)
    scale = max(1.0, np.abs(ref).max())
    for _ in range(2):
        assert L.cc_set_device(torch.cuda.current_device()) == 0
        tc = m.forward(cuda(f), precision=1).cpu().numpy()
        f32 = m.forward(cuda(f), precision=0).cpu().numpy()
        assert np.abs(tc - ref).max() <= TC_RTOL * scale
        assert np.abs(f32 - ref).max() <= FP32_RTOL * scale


def test_gradients_match_oracle():
    m, p = random_net(3)
    rng = np.random.default_rng(7)
    f = rng.standard_normal((777, 24)).astype(np.float32)
    t = rng.standard_normal((777, 3)).astype(np.float32)
    g, loss = m.gradients(cuda(f), cuda(t))
    gr, lr = oracle.mlp_gradients(p, f, t)
    assert abs(loss - lr) <= 1e-5 * lr
    assert np.linalg.norm(g - gr) <= GRAD_RTOL * np.linalg.norm(gr)


def test_adam_step_is_the_published_update():
    m, p = random_net(4)
    rng = np.random.default_rng(8)
    f = rng.standard_normal((512, 24)).astype(np.float32)
    t = rng.standard_normal((512, 3)).astype(np.float32)
    g, _ = m.gradients(cuda(f), cuda(t))
    lr = 1e-3
    m.train(cuda(f), cuda(t), batch=512, steps=1, lr=lr, seed=0)  # one full-batch step
    # first Adam step with bias correction: m_hat = g, v_hat = g^2
    expect = p - lr * g / (np.abs(g) + 1e-8)
    got = m.parameters()
    assert np.abs(got - expect).max() <= 1e-6 + 1e-3 * lr


def test_training_fits_a_teacher_network():
    teacher, _ = random_net(5, scale=0.5)
    rng = np.random.default_rng(9)
    f = cuda(rng.standard_normal((20000, 24)))
    t = teacher.forward(f, precision=0)
    student = Mlp(11)
    losses = student.train(f, t, batch=2048, steps=600, lr=3e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-20:].mean() < 0.1 * losses[:5].mean()


def contact_scene(n=16, seed=0):
    return scenes.small_sheet(n, seed=seed, height=0.104, side=0.2, pins=(), radius=0.002)


def test_features_with_history_match_oracle():
    """With adaptive-guess history (both solvers stepped along their own
    trajectories), the last-step-correction features agree too."""
    sc = contact_scene()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    st = sc.settings.to_c()
    xg, vg, tg = sc.x0.copy(), sc.v0.copy(), 0.0
    xo, vo, to = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(5):
        xg, vg, tg, _ = g.step(xg, vg, tg, st)
        xo, vo, to, _ = o.step(xo, vo, to, st)
    rows = g.free_vertices
    feat = torch.zeros((rows, 24), dtype=torch.float32, device="cuda")
    targ = torch.zeros((rows, 3), dtype=torch.float32, device="cuda")
    g.set_state(xg, vg, tg)  # the same bits as the committed state: history stays valid
    g.step_sample(st, feat, targ)
    ref = o.learned_features(xo, vo, to, st)
    f = feat.cpu().numpy()
    assert np.abs(ref[:, 20:23]).max() > 0  # history present
    assert np.all(np.abs(f - ref) <= 1e-4 * np.maximum(1.0, np.abs(ref)))


def test_features_and_targets_match_oracle():
    sc = contact_scene()
    g = VbdSolver(sc)
    o = oracle.Solver(sc)
    # advance both a few plain steps so that contacts exist, then compare a
    # fresh-history step start (both solvers rebuilt: adaptive factor 1)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(4):
        x, v, t, _ = g.step(x, v, t, sc.settings.to_c())
    g = VbdSolver(sc)
    rows = g.free_vertices
    feat = torch.zeros((rows, 24), dtype=torch.float32, device="cuda")
    targ = torch.zeros((rows, 3), dtype=torch.float32, device="cuda")
    g.set_state(x, v, t)
    m = g.step_sample(sc.settings.to_c(), feat, targ)
    ref = o.learned_features(x, v, t, sc.settings.to_c())
    f = feat.cpu().numpy()
    scale = np.maximum(1.0, np.abs(ref))
    assert np.all(np.abs(f - ref) <= FEATURE_RTOL * scale)
    assert f[:, 19].max() > 0  # contact terms present
    # targets = (x_end - adaptive guess) / (|g| dt^2); fresh history: guess = y
    xe, _, _ = g.get_state()
    st = sc.settings
    u = 9.81 * st.dt * st.dt
    y = x + (v * st.dt + np.array(st.gravity) * st.dt * st.dt) / (1 + st.damping * st.dt)
    assert np.allclose(targ.cpu().numpy(), ((xe - y) / u).astype(np.float32), rtol=1e-5, atol=1e-6)
    assert m["iterations"] == st.iterations


def _plain_and_learned(net, precision, steps=3):
    sc = contact_scene()
    st_p = sc.settings.to_c()
    s = sc.settings
    s.init_mode = 1
    st_l = s.to_c()
    a, b = VbdSolver(sc).set_lanes(4), VbdSolver(sc).set_lanes(4)  # bitwise comparison: same lanes
    b.set_mlp(net, precision)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    xb, vb, tb = x.copy(), v.copy(), t
    out = []
    for _ in range(steps + 4):
        x, v, t, ma = a.step(x, v, t, st_p)
        xb, vb, tb, mb = b.step(xb, vb, tb, st_l)
        out.append((x.copy(), xb.copy(), ma, mb))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_zero_network_reproduces_the_adaptive_guess_bitwise(precision):
    net = Mlp(0)
    net.set_parameters(np.zeros(net.count, np.float32))
    for xa, xb, ma, mb in _plain_and_learned(net, precision):
        assert mb["init_used"] == 0  # equal energies keep the adaptive guess
        assert mb["init_energy_learned"] == mb["init_energy_adaptive"]
        assert np.array_equal(xa, xb)


def test_worse_guess_falls_back_to_the_adaptive_guess():
    net = Mlp(0)
    p = np.zeros(net.count, np.float32)
    p[-3] = 50.0  # output bias: a 50 |g| dt^2 shift in x, clipped to the OGC balls
    net.set_parameters(p)
    for xa, xb, ma, mb in _plain_and_learned(net, 1):
        assert mb["init_used"] == 0  # no scale of the shift lowers the energy
        assert mb["init_energy_learned"] > mb["init_energy_adaptive"]
        assert np.array_equal(xa, xb)


def test_better_guess_is_taken():
    """A network fitted to one step's converged corrections (a sampled step)
    must be taken on that step and must start closer to the solution."""
    sc = contact_scene()
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    g0 = VbdSolver(sc)
    for _ in range(6):
        x, v, t, _ = g0.step(x, v, t, sc.settings.to_c())
    g = VbdSolver(sc)
    rows = g.free_vertices
    feat = torch.zeros((rows, 24), dtype=torch.float32, device="cuda")
    targ = torch.zeros((rows, 3), dtype=torch.float32, device="cuda")
    s = sc.settings
    s.iterations, s.residual_tolerance, s.residual_check_every = 200, 1e-6, 1
    g.set_state(x, v, t)
    g.step_sample(s.to_c(), feat, targ)
    net = Mlp(3)
    net.train(feat, targ, batch=rows, steps=1500, lr=3e-3, seed=0)
    s.residual_tolerance, s.residual_check_every = 1e-3, 1
    runs = {}
    for mode in (0, 1):
        s.init_mode = mode
        h = VbdSolver(sc)
        h.set_mlp(net, 1)
        _, _, _, m = h.step(x, v, t, s.to_c())
        runs[mode] = m
    assert runs[1]["init_used"] == 1
    assert runs[1]["initial_relative_residual"] < runs[0]["initial_relative_residual"]
    assert runs[1]["iterations"] <= runs[0]["iterations"]


def test_step_energy_difference_matches_oracle():
    """The device step energy (all terms once each) against the oracle's FP64
    objective: E(learned guess) - E(adaptive guess) for a constant shift."""
    sc = contact_scene()
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    g0 = VbdSolver(sc)
    for _ in range(4):
        x, v, t, _ = g0.step(x, v, t, sc.settings.to_c())
    net = Mlp(0)
    p = np.zeros(net.count, np.float32)
    p[-3], p[-1] = 0.05, -0.02  # small constant correction
    net.set_parameters(p)
    s = sc.settings
    s.init_mode = 1
    g = VbdSolver(sc)  # fresh history: adaptive guess = y
    g.set_mlp(net, 0)
    _, _, _, m = g.step(x, v, t, s.to_c())
    st = sc.settings
    u = 9.81 * st.dt * st.dt
    y = x + (v * st.dt + np.array(st.gravity) * st.dt * st.dt) / (1 + st.damping * st.dt)
    o = oracle.Solver(sc, threads=8)
    rq = min(max(st.radius + np.linalg.norm(y - x, axis=1).max(), 2 * st.radius), 4 * st.radius)
    cs = o.world.detect(o.positions(x), rq, st.ogc_c())
    centers, radii = x, np.asarray(cs["radii"])[: sc.n]

    def clip(p):
        d = p - centers
        ln = np.linalg.norm(d, axis=1)
        k = ln > radii
        out = p.copy()
        out[k] = centers[k] + d[k] * (radii[k] / ln[k])[:, None]
        return out

    xp = clip(y)
    xl = clip(y + np.array([0.05, 0.0, -0.02]) * u)
    ep, _ = o.step_gradient(x, v, st.to_c(), xp)
    el, _ = o.step_gradient(x, v, st.to_c(), xl)
    d_gpu = m["init_energy_learned"] - m["init_energy_adaptive"]
    assert abs(d_gpu - (el - ep)) <= 1e-9 * abs(ep) + 1e-6 * abs(el - ep)


def test_shipped_fold_network_gains_on_held_out_fold_steps():
    """The shipped network (clothcraft_b200/data/fold_init_mlp.npz, trained on
    fold variants with seeds other than the benchmark's) on twelve steps of
    the benchmark's own seed from its fold-phase state, at the benchmark's
    target and acceleration: the energy check takes it on most steps and the
    steps need no more iterations in total than with the plain adaptive
    guess (measured: 468 against 484). The figures are printed; the initial
    relative residual is not a gain measure here (a guess that lowers the
    step energy can start with a larger barrier gradient)."""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    net = Mlp.load(os.path.join(root, "clothcraft_b200", "data", "fold_init_mlp.npz"))
    z = np.load(os.path.join(root, "tests", "golden", "sheet256_fold_state.npz"))
    x, v, t = z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])
    sc = scenes.config1()
    s = sc.settings
    s.iterations, s.residual_tolerance, s.residual_check_every, s.stall_refresh = 200, 1e-3, 2, 2
    s.acceleration = 0.95
    runs = {}
    for mode in (0, 1):
        s.init_mode = mode
        h = VbdSolver(sc).set_lanes(8 | 4 << 8)
        h.set_mlp(net, 1)
        h.set_state(x, v, t)
        runs[mode] = [h.step_resident(s.to_c()) for _ in range(12)]
    its = {k: sum(m["iterations"] for m in r) for k, r in runs.items()}
    r0 = {k: float(np.mean([m["initial_relative_residual"] for m in r])) for k, r in runs.items()}
    used = float(np.mean([m["init_used"] for m in runs[1]]))
    print("held-out fold steps: iterations plain %d learned %d; mean initial residual plain %.3g learned %.3g; "
          "learned taken on %.0f %% of steps" % (its[0], its[1], r0[0], r0[1], 100 * used))
    assert used >= 0.5
    assert its[1] <= its[0]
