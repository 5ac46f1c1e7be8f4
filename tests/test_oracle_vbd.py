"""Pins the oracle's VBD restatement against the reference's known-answer tests
(tests/vbd.rs, src/vbd/prediction.rs tests, src/vbd/coloring.rs tests,
tests/deformation.rs)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from clothcraft_b200 import abi, scenes
from clothcraft_b200.abi import cc_ogc_settings


# tests/vbd.rs:10-34
def test_contact_activates_during_the_step_and_settles_without_a_sawtooth():
    sc = scenes.resting_patch()
    s = oracle.Solver(sc)
    st = sc.settings.to_c()
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    max_delta = 0.0
    for i in range(60):
        old = x.copy()
        x, v, t, m = s.step(x, v, t, st)
        assert np.all(np.abs(x[:, 1] - st.contact.radius) < 1e-5), (i, x[:, 1])
        if i > 10:
            max_delta = max(max_delta, float(np.abs(x[:, 1] - old[:, 1]).max()))
    assert max_delta < 1e-6


# tests/vbd.rs:44-61
def test_free_fall_preserves_rest_shape_and_backward_euler_velocity():
    sc = scenes.demo_left_panel()
    s = oracle.Solver(sc)
    st = scenes.StepSettings(dt=0.005, damping=0.0, iterations=3).to_c()
    x, v, t, _ = s.step(sc.x0, sc.v0, 0.0, st)
    g = np.array([0.0, -9.81, 0.0])
    assert np.all(np.linalg.norm(v - g * 0.005, axis=1) < 1e-9)
    assert np.all(np.linalg.norm(x - sc.x0 - g * 0.005 ** 2, axis=1) < 1e-12)


# tests/vbd.rs:62-91
def test_mouse_attachment_pulls_cloth_and_invalid_input_is_transactional():
    sc = scenes.demo_left_panel()
    s = oracle.Solver(sc)
    tri = sc.mesh.triangles[0]
    center = sc.x0[tri].mean(axis=0)
    center = sum(sc.x0[i] / 3.0 for i in tri)
    grab = dict(vertices=tri, weights=[1 / 3] * 3, target=center + np.array([0, 0, 0.01]), stiffness=100.0)
    st = scenes.StepSettings(gravity=(0.0, 0.0, 0.0), iterations=6).to_c()
    x, v, t, _ = s.step(sc.x0, sc.v0, 0.0, st, grab)
    moved = sum(x[i] / 3.0 for i in tri)
    assert moved[2] > center[2]
    bad = dict(grab, target=np.array([np.nan, 0, 0]))
    with pytest.raises(oracle.OracleError):
        s.step(x, v, t, st, bad)


# src/vbd/prediction.rs:59-87
def test_adaptive_guess_preserves_damped_fall_and_supported_rest_and_invalidates_edits():
    L = oracle.lib()
    st = scenes.StepSettings(dt=1 / 60).to_c()
    p = L.or_prediction_create()
    x = np.array([[0.0, 1.0, 0.0]])
    v = np.zeros((1, 3))
    t = 0.0
    g = np.array([0.0, -9.81, 0.0])
    dt, damping = 1 / 60, 1.5
    for _ in range(5):
        nxt = np.zeros((1, 3))
        L.or_prediction_guess(p, oracle.f64p(x), oracle.f64p(v), 1, t, C.byref(st), oracle.f64p(nxt))
        expected = (v[0] * dt + g * dt ** 2) / (1 + damping * dt)
        assert np.linalg.norm(nxt[0] - x[0] - expected) < 1e-12
        old = v.copy()
        v = (nxt - x) / dt
        x = nxt
        t += dt
        L.or_prediction_record(p, oracle.f64p(old), oracle.f64p(x), oracle.f64p(v), 1, t, C.byref(st))
    v = np.zeros((1, 3))
    L.or_prediction_record(p, oracle.f64p(np.zeros((1, 3))), oracle.f64p(x), oracle.f64p(v), 1, t, C.byref(st))
    out = np.zeros((1, 3))
    L.or_prediction_guess(p, oracle.f64p(x), oracle.f64p(v), 1, t, C.byref(st), oracle.f64p(out))
    assert np.array_equal(out, x)
    x2 = x.copy()
    x2[0, 0] += 0.01
    L.or_prediction_guess(p, oracle.f64p(x2), oracle.f64p(v), 1, t, C.byref(st), oracle.f64p(out))
    assert out[0, 1] < x2[0, 1]
    L.or_prediction_destroy(p)


# src/vbd/coloring.rs:51-137
def test_incidence_coloring_matches_expanded_graph_and_has_no_conflicts():
    L = oracle.lib()
    x = np.array([[0.0, 0.0, 0.002 * i] for i in range(4) for _ in range(3)])
    for i in range(4):
        x[3 * i + 1, 0] = 1.0
        x[3 * i + 2, 1] = 1.0
    w = oracle.World(x, [[0, 1, 2], [3, 4, 5], [6, 7, 8], [9, 10, 11]], 9)
    st = cc_ogc_settings(0.003, 100000.0, 0.45, 0.01)
    contact = w.detect(x, 0.012, st)
    assert len(contact["kinds"]) > 0
    graph = [[1], [0, 2], [1], [], [6], [], [4], [], []]
    offsets = np.zeros(10, np.uint64)
    offsets[1:] = np.cumsum([len(g) for g in graph])
    adj = np.array([a for g in graph for a in g], np.uint32)
    cc = abi.cc_contacts()
    keep = [np.ascontiguousarray(contact[k]) for k in ("kinds", "vertices", "counts", "epsilon", "incident_offsets",
                                                       "incident")]
    cc.kinds = abi.ptr(keep[0], C.c_uint8)
    cc.vertices = abi.ptr(keep[1], C.c_uint32)
    cc.counts = abi.ptr(keep[2], C.c_uint8)
    cc.mollifier_epsilon = abi.ptr(keep[3], C.c_double)
    cc.incident_offsets = abi.ptr(keep[4], C.c_uint64)
    cc.incident = abi.ptr(keep[5], C.c_uint32)
    cc.n_contacts = len(contact["kinds"])
    grab = dict(vertices=[0, 4, 8], weights=[0.2, 0.3, 0.5], target=[0, 0, 0], stiffness=100.0)
    for g in (None, grab):
        out = np.zeros(9, np.uint32)
        gc = oracle.grab_c(g)
        nc = L.or_greedy_colors(9, abi.ptr(offsets, C.c_uint64), oracle.u32p(adj), C.byref(cc),
                                C.byref(gc) if gc is not None else C.cast(None, C.POINTER(abi.cc_grab)),
                                oracle.u32p(out))
        full = [list(gg) for gg in graph]

        def connect(vs):
            for a in vs:
                for b in vs:
                    if a != b and a < 9 and b < 9:
                        full[a].append(b)
        for k, vs in zip(contact["counts"], contact["vertices"]):
            connect([int(u) for u in vs[:k]])
        if g is not None:
            connect(g["vertices"])
        assigned = [None] * 9
        for vtx in range(9):
            c = 0
            while any(assigned[i] == c for i in full[vtx]):
                c += 1
            assigned[vtx] = c
        assert out.tolist() == assigned
        assert nc == max(assigned) + 1
        for vtx in range(9):
            for o in full[vtx]:
                assert out[vtx] != out[o]
    empty = abi.cc_contacts()
    z = np.zeros(10, np.uint64)
    empty.incident_offsets = abi.ptr(z, C.c_uint64)
    out = np.zeros(9, np.uint32)
    nc = L.or_greedy_colors(9, abi.ptr(np.zeros(10, np.uint64), C.c_uint64), oracle.u32p(np.zeros(1, np.uint32)),
                            C.byref(empty), C.cast(None, C.POINTER(abi.cc_grab)), oracle.u32p(out))
    assert nc == 1 and np.all(out == 0)


# tests/deformation.rs:5-19 (on the demo's left panel)
def test_extension_diagnostic_uses_material_rest_and_is_rigid_motion_invariant():
    L = oracle.lib()
    mesh = scenes.pattern_build(0.4, 0.6, 3, 4, scenes.Material())
    x = np.stack([mesh.uv[:, 0], -mesh.uv[:, 1], np.zeros(mesh.n)], axis=1) + np.array([-0.4, 1.0, 0.0])
    m, keep = mesh.to_c()
    out = np.zeros(2)
    L.or_extension_percent(C.byref(m), oracle.f64p(np.ascontiguousarray(x)), oracle.f64p(out))
    assert out[1] < 1e-10
    y = np.stack([-x[:, 1] * 1.2, x[:, 0] * 1.2, x[:, 2]], axis=1) + 2.0
    L.or_extension_percent(C.byref(m), oracle.f64p(np.ascontiguousarray(y)), oracle.f64p(out))
    assert np.all(np.abs(out - 20.0) < 1e-10)


def test_step_failures_are_transactional():
    """Invalid settings and non-finite state fail without touching the state
    (src/vbd.rs:256-274)."""
    sc = scenes.demo_left_panel()
    s = oracle.Solver(sc)
    with pytest.raises(oracle.OracleError):
        s.step(sc.x0, sc.v0, 0.0, scenes.StepSettings(dt=0.1).to_c())
    v = sc.v0.copy()
    v[0, 0] = np.inf
    with pytest.raises(oracle.OracleError):
        s.step(sc.x0, v, 0.0, scenes.StepSettings().to_c())


# Chebyshev acceleration (library extension; off by default)
def _hanging(rho, iterations=60):
    sc = scenes.small_sheet(16, seed=3, obstacle=False)
    s = sc.settings
    s.iterations, s.residual_tolerance, s.residual_check_every, s.acceleration = iterations, 0.0, iterations, rho
    return sc, s.to_c()


def test_acceleration_lowers_the_residual_of_a_slowly_converging_sheet():
    """A sheet hanging from two corners converges slowly under plain sweeps
    (low-frequency modes); the Chebyshev extrapolation reaches a lower
    relative residual in the same 60 iterations, more so for larger rho."""
    res = []
    for rho in (0.0, 0.5, 0.9):
        sc, st = _hanging(rho)
        _, _, _, m = oracle.Solver(sc, threads=4).step(sc.x0, sc.v0, 0.0, st)
        res.append(m["relative_residual"])
    assert res[2] < res[1] < res[0]
    assert res[2] < 0.8 * res[0]


def test_accelerated_contact_steps_keep_the_trust_region():
    """With rho = 0.95 in a contact scene every extrapolated position is
    clipped to its OGC ball (the step raises if any vertex leaves it) and
    the separation stays positive."""
    sc = scenes.small_sheet(16, seed=0, height=0.104, side=0.2, pins=(), radius=0.002)
    s = sc.settings
    s.iterations, s.acceleration = 30, 0.95
    st = s.to_c()
    o = oracle.Solver(sc, threads=4)
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(8):
        x, v, t, m = o.step(x, v, t, st)
    assert m["contact_terms"] > 0 and m["minimum_distance_m"] > 0.0
    assert np.all(np.isfinite(x))


def test_acceleration_outside_zero_to_one_is_rejected():
    for rho in (1.0, -0.5, float("inf")):
        sc, st = _hanging(rho, 4)
        with pytest.raises(oracle.OracleError):
            oracle.Solver(sc).step(sc.x0, sc.v0, 0.0, st)
