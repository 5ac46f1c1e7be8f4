"""Pins the oracle's OGC restatement against the reference's known-answer tests
(tests/ogc.rs, tests/ogc_bvh.rs, tests/ogc_cache.rs, src/ogc/world.rs tests)."""
import numpy as np
import pytest

import oracle
from clothcraft_b200.abi import cc_ogc_settings


def ogc(r, stiffness=100000.0, relaxation=0.45, refresh=0.01):
    return cc_ogc_settings(r, stiffness, relaxation, refresh)


def keyset(c):
    return [(int(k), tuple(int(x) for x in v)) for k, v in zip(c["kinds"], c["vertices"])]


# tests/ogc.rs:17-35
def test_two_stage_potential_is_c2_at_join_and_has_barrier():
    L = oracle.lib()
    r, k = 0.01, 1200.0
    tau, eps = r / 2, 1e-9
    a = np.zeros(3)
    b = np.zeros(3)
    L.or_activation_jet1(tau - eps, r, k, oracle.f64p(a))
    L.or_activation_jet1(tau + eps, r, k, oracle.f64p(b))
    assert abs(a[0] - b[0]) < 1e-7
    assert abs(a[1] - b[1]) < 1e-5
    assert abs(a[2] - b[2]) < 0.001
    assert L.or_activation(r, r, k) == 0.0
    assert np.isinf(L.or_activation(0.0, r, k))
    assert L.or_activation(1e-12, r, k) > L.or_activation(1e-6, r, k)
    for d in (0.001, 0.004, 0.007, 0.009):
        j = np.zeros(3)
        L.or_activation_jet1(d, r, k, oracle.f64p(j))
        fd = (L.or_activation(d + eps, r, k) - L.or_activation(d - eps, r, k)) / (2 * eps)
        assert abs(fd - j[1]) < 1e-7


# tests/ogc.rs:37-99
def test_contact_block_derivatives_and_force_balance():
    L = oracle.lib()
    cases = [
        (0, [[0.1, 0.1, 0.04], [0.1, 0.1, 0.0]], 2),
        (1, [[0.1, 0.04, 0.02], [-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]], 3),
        (2, [[0.1, 0.1, 0.04], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]], 4),
        (3, [[-1.0, 0.0, 0.04], [1.0, 0.0, 0.04], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0]], 4),
    ]

    def block(x, v):
        e = np.zeros(1)
        g = np.zeros(3)
        h = np.zeros(9)
        L.or_contact_block(kind, count, 0.01, oracle.f64p(np.ascontiguousarray(x)), v, 0.1, 20.0,
                           oracle.f64p(e), oracle.f64p(g), oracle.f64p(h))
        return e[0], g, h.reshape(3, 3)

    def value(x):
        return L.or_contact_value(kind, count, 0.01, oracle.f64p(np.ascontiguousarray(x)), 0.1, 20.0)

    for kind, p, count in cases:
        x = np.zeros((4, 3))
        x[:len(p)] = p
        eps = 1e-7
        force = np.zeros(3)
        for v in range(count):
            _, g, h = block(x, v)
            force += g
            for axis in range(3):
                a = x.copy()
                b = x.copy()
                a[v, axis] += eps
                b[v, axis] -= eps
                fd = (value(a) - value(b)) / (2 * eps)
                assert abs(fd - g[axis]) < 1e-6
                dg = (block(a, v)[1] - block(b, v)[1]) / (2 * eps)
                assert np.linalg.norm(dg - h[:, axis]) < 1e-4
        assert np.linalg.norm(force) < 1e-9
        ang = 0.64
        R = np.array([[np.cos(ang), 0, np.sin(ang)], [0, 1, 0], [-np.sin(ang), 0, np.cos(ang)]])
        rotated = x @ R.T + 2.0
        assert abs(value(x) - value(rotated)) < 1e-10


# tests/ogc.rs:101-121
def test_folded_surface_preserves_multiple_layers_and_excludes_false_edge_contact():
    x = np.array([[0.0, 0.1, 0.1], [-1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    tris = np.array([[1, 2, 3], [2, 1, 4]], np.uint32)
    assert oracle.lib().or_edge_feasible(oracle.f64p(x), 5, oracle.u32p(tris), 2,
                                         oracle.f64p(np.ascontiguousarray(x[0])), 1, 2) == 0
    w = oracle.World(x, tris, 1)
    s = w.detect(x, 0.25, ogc(0.2))
    assert int((s["kinds"] == 2).sum()) == 2


# tests/ogc.rs:123-135
def test_shared_feature_contact_is_not_duplicated():
    x = np.array([[0.0, -0.03, 0.04], [-1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, -1.0]])
    w = oracle.World(x, [[1, 2, 3], [2, 1, 4]], 1)
    s = w.detect(x, 0.2, ogc(0.1))
    assert len(s["kinds"]) == 1
    assert s["kinds"][0] == 1


def _truncate(s, i, p, centers):
    d = p - centers[i]
    n = np.linalg.norm(d)
    b = s["radii"][i]
    return (centers[i] + d * (b / n), True) if n > b else (p, False)


# tests/ogc.rs:137-177
def test_reverse_vertex_face_and_edge_edge_bounds_protect_face_interiors():
    x = np.array([[-1.0, -1.0, 0.1], [1.0, -1.0, 0.1], [0.0, 1.0, 0.1], [0.0, 0.0, 0.0], [0.01, 0.0, -1.0],
                  [0.0, 0.01, -1.0]])
    w = oracle.World(x, [[0, 1, 2], [3, 4, 5]], 3)
    s = w.detect(x, 0.2, ogc(0.15))
    assert np.all(s["radii"] <= 0.045 + 1e-12)
    for i in range(3):
        p, b = _truncate(s, i, x[i] - np.array([0, 0, 10.0]), x)
        assert b and p[2] >= 0.055 - 1e-12
    x = np.array([[-1.0, 0.0, 0.1], [1.0, 0.0, 0.1], [-1.0, -1.0, 0.1], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0],
                  [1.0, 1.0, 0.0]])
    w = oracle.World(x, [[0, 1, 2], [3, 4, 5]], 6)
    s = w.detect(x, 0.2, ogc(0.15))
    assert np.any(s["kinds"] == 3)
    assert s["radii"][0] <= 0.045 + 1e-12 and s["radii"][1] <= 0.045 + 1e-12
    moved = np.array([_truncate(s, i, x[i] + (np.array([0, 0, -10.0]) if i < 3 else np.array([0, 0, 10.0])),
                                x)[0] for i in range(6)])
    w.validate_start(moved)


# tests/ogc.rs:179-200
def test_bounds_are_cumulative_until_detection_and_settings_fail_closed():
    x = np.array([[0.0, 0.0, 0.1], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    w = oracle.World(x, [[1, 2, 3]], 1)
    s = w.detect(x, 0.2, ogc(0.15))
    p = _truncate(s, 0, x[0] - np.array([0, 0, 0.04]), x)[0]
    q = _truncate(s, 0, p - np.array([0, 0, 0.04]), x)[0]
    assert abs(q[2] - 0.055) < 1e-12
    with pytest.raises(oracle.OracleError):
        w.detect(x, 0.01, ogc(0.15))
    with pytest.raises(oracle.OracleError):
        w.detect(x, 0.2, ogc(0.003, relaxation=0.5))


# tests/ogc.rs:202-213
def test_initial_intersection_is_rejected_instead_of_claiming_a_guarantee():
    x = np.array([[0.0, 0.0, -1.0], [0.0, 0.0, 1.0], [2.0, 0.0, 0.0], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0],
                  [0.0, 1.0, 0.0]])
    w = oracle.World(x, [[0, 1, 2], [3, 4, 5]], 3)
    with pytest.raises(oracle.OracleError):
        w.validate_start(x)


# tests/ogc.rs:216-231
def test_query_radius_changes_bounds_without_activating_distant_forces():
    x = np.array([[0.0, 0.0, 0.02], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    w = oracle.World(x, [[1, 2, 3]], 1)
    s = w.detect(x, 0.03, ogc(0.01))
    assert len(s["kinds"]) == 1
    assert s["active_contacts"] == 0
    assert abs(s["radii"][0] - 0.009) < 1e-12


# tests/ogc.rs:233-255
def test_dormant_contact_activates_inside_the_same_original_trust_region():
    L = oracle.lib()
    x = np.array([[0.0, 0.0, 0.00305], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    w = oracle.World(x, [[1, 2, 3]], 1)
    st = ogc(0.003)
    s = w.detect(x, 0.006, st)
    assert s["active_contacts"] == 0
    p, clipped = _truncate(s, 0, np.array([0.0, 0.0, 0.0025]), x)
    assert not clipped
    x2 = x.copy()
    x2[0] = p
    # the single retained term is a point-face contact (0; 1,2,3)
    assert s["kinds"][0] == 2
    val = L.or_contact_value(2, 4, 0.0, oracle.f64p(np.ascontiguousarray(x2)), st.radius, st.stiffness)
    expected = 0.5 * st.stiffness * 0.0005 ** 2
    assert abs(val - expected) < 1e-12
    s2 = w.detect(x2, 0.006, st)
    assert s2["active_contacts"] == 1


# tests/ogc.rs:258-274
def test_static_edges_before_moving_edges_are_not_missed():
    x = np.array([[-1.0, 0.0, 0.1], [1.0, 0.0, 0.1], [-1.0, -1.0, 0.1], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0],
                  [1.0, 1.0, 0.0]])
    a = oracle.World(x, [[0, 1, 2], [3, 4, 5]], 3)
    b = oracle.World(x, [[3, 4, 5], [0, 1, 2]], 3)
    sa = a.detect(x, 0.2, ogc(0.15))
    sb = b.detect(x, 0.2, ogc(0.15))
    assert np.array_equal(sa["radii"], sb["radii"])
    assert sa["edge_edge_candidates"] == sb["edge_edge_candidates"]
    assert len(sa["kinds"]) == len(sb["kinds"])


# tests/ogc.rs:277-292
def test_shared_vertex_near_parallel_edges_do_not_create_false_initial_intersections():
    x = np.array([[0.194131180644, 0.943517088890, 0.091018132865],
                  [0.183311969042, 0.970439314842, 0.101929388940],
                  [0.197149559855, 0.954595983028, 0.076061360538],
                  [0.195560514927, 0.972076416016, 0.068995960057],
                  [0.188853010535, 0.980777919292, 0.085684590042]]).astype(np.float32).astype(np.float64)
    w = oracle.World(x, [[0, 1, 2], [3, 2, 4]], 5)
    w.validate_start(x)


# src/ogc/world.rs:566-633
@pytest.mark.parametrize("offset", [(0.0, 0.0, 0.0), (1e6, -2e6, 3e6)])
def test_current_boxes_preserve_exact_contacts_and_balls_during_cache_reuse(offset):
    off = np.array(offset)
    rest = []
    tris = []
    for layer in range(3):
        for y in range(5):
            for xx in range(5):
                rest.append(off + np.array([xx * 0.008, y * 0.008, layer * 0.003]))
        for y in range(4):
            for xx in range(4):
                a = layer * 25 + y * 5 + xx
                tris += [[a, a + 1, a + 5], [a + 1, a + 6, a + 5]]
    rest = np.array(rest)
    pruned = oracle.World(rest, tris, 50, [[0, 25], [1, 26]])
    reference = oracle.World(rest, tris, 50, [[0, 25], [1, 26]])
    st = ogc(0.003)
    rejections = reuse = rebuilds = 0
    for frame in range(24):
        x = rest.copy()
        for i in range(50):
            a = frame * 0.15 + i * 0.31
            x[i] += np.array([np.sin(a) * 0.0004, np.cos(a) * 0.0003, np.sin(a) * 0.0002])
            if frame >= 18:
                x[i, 0] += 0.004
        rq = 0.006 if frame <= 11 else (0.009 if frame <= 15 else 0.004)
        a = pruned.detect(x, rq, st)
        b = reference.detect(x, rq, st, prune=False)
        assert np.array_equal(a["radii"], b["radii"])
        assert a["minimum_distance"] == b["minimum_distance"]
        for k in ("active_contacts", "vertex_face_candidates", "edge_edge_candidates", "broad_phase_rebuilt"):
            assert a[k] == b[k], k
        assert np.array_equal(a["incident"], b["incident"])
        assert np.array_equal(a["incident_offsets"], b["incident_offsets"])
        assert keyset(a) == keyset(b)
        assert np.array_equal(a["epsilon"].view(np.uint64), b["epsilon"].view(np.uint64))
        rejections += a["aabb_rejections"]
        rebuilds += int(a["broad_phase_rebuilt"])
        reuse += int(not a["broad_phase_rebuilt"])
    assert rejections > 0 and reuse > 0 and rebuilds > 1


def _lcg(seed):
    s = [seed]

    def random():
        s[0] = (s[0] * 6364136223846793005 + 1) & 0xFFFFFFFFFFFFFFFF
        return (s[0] >> 32) / 4294967295.0
    return random


def _box(p, q=None):
    q = p if q is None else q
    return np.concatenate([np.minimum(p, q), np.maximum(p, q)])


def _dist2(a, b):
    d = np.maximum(np.maximum(a[:3] - b[3:], b[:3] - a[3:]), 0.0)
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2]


# tests/ogc_bvh.rs:5-67
def test_dual_tree_pairs_match_exhaustive_search_without_duplicates():
    rnd = _lcg(53)
    a = []
    for _ in range(129):
        p = np.array([rnd(), rnd(), rnd()])
        a.append(_box(p, p + 0.03))
    b = [_box(np.array([rnd(), rnd(), rnd()])) for _ in range(97)]
    a = np.array(a)
    b = np.array(b)
    da = np.array([i % 3 == 1 for i in range(len(a))])
    db = np.array([i % 2 == 1 for i in range(len(b))])
    ta = oracle.Bvh(a, da)
    tb = oracle.Bvh(b, db)
    for frame in range(4):
        if frame > 0:
            for i in range(len(a)):
                if da[i]:
                    delta = np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5])
                    a[i, :3] += delta
                    a[i, 3:] += delta
            ta.refit_dynamic(a)
        for radius in (0.0, 0.05, 0.2, 2.0):
            got = ta.pairs(tb, radius)
            pairs = set(map(tuple, got.tolist()))
            assert len(pairs) == len(got)
            expected = {(i, j) for i in range(len(a)) for j in range(len(b))
                        if (da[i] or db[j]) and _dist2(a[i], b[j]) <= radius * radius}
            assert pairs == expected
            got = ta.pairs(None, radius, same=True)
            pairs = set(map(tuple, got.tolist()))
            assert len(pairs) == len(got) and all(i < j for i, j in pairs)
            expected = {(i, j) for i in range(len(a)) for j in range(i + 1, len(a))
                        if (da[i] or da[j]) and _dist2(a[i], a[j]) <= radius * radius}
            assert pairs == expected


# tests/ogc_bvh.rs:70-96
def test_bounds_distance_never_discards_a_close_primitive_pair():
    L = oracle.lib()
    s = [19]

    def rnd():
        s[0] = (s[0] * 6364136223846793005 + 1) & 0xFFFFFFFFFFFFFFFF
        return (s[0] >> 32) / 4294967295.0 * 4.0 - 2.0
    for _ in range(2000):
        p = np.array([[rnd(), rnd(), rnd()] for _ in range(4)])
        q = np.zeros(3)
        L.or_closest_triangle(oracle.f64p(np.ascontiguousarray(p)), oracle.f64p(q))
        vf = L.or_bounds_distance_squared(oracle.f64p(_box(p[3])),
                                          oracle.f64p(np.concatenate([p[:3].min(0), p[:3].max(0)])))
        assert vf <= ((p[3] - q) ** 2).sum() + 1e-12
        st = np.zeros(2)
        L.or_closest_segments(oracle.f64p(np.ascontiguousarray(p)), oracle.f64p(st))
        ee = L.or_bounds_distance_squared(oracle.f64p(_box(p[0], p[1])), oracle.f64p(_box(p[2], p[3])))
        pa = p[0] + (p[1] - p[0]) * st[0]
        pb = p[2] + (p[3] - p[2]) * st[1]
        assert ee <= ((pa - pb) ** 2).sum() + 1e-12


# tests/ogc_bvh.rs:99-143
def test_partitioned_bvh_matches_exhaustive_queries_after_large_deformations():
    rnd = _lcg(7)
    boxes = []
    for _ in range(513):
        p = np.array([rnd(), rnd(), rnd()])
        boxes.append(_box(p, p + 0.04))
    boxes = np.array(boxes)
    dynamic = np.array([i % 3 == 0 for i in range(len(boxes))])
    bvh = oracle.Bvh(boxes, dynamic)
    for frame in range(4):
        if frame > 0:
            for i in range(len(boxes)):
                if dynamic[i]:
                    delta = np.array([rnd() - 0.5, rnd() - 0.5, rnd() - 0.5])
                    boxes[i, :3] += delta
                    boxes[i, 3:] += delta
            bvh.refit_dynamic(boxes)
        for _ in range(50):
            p = np.array([rnd(), rnd(), rnd()])
            q = np.concatenate([p - 0.15, p + 0.15])
            for only_moving in (False, True):
                expected = [i for i in range(len(boxes))
                            if np.all(q[:3] <= boxes[i, 3:]) and np.all(q[3:] >= boxes[i, :3])
                            and (not only_moving or dynamic[i])]
                actual = sorted(bvh.query(q, only_moving).tolist())
                assert actual == expected


# tests/ogc_cache.rs:5-63
def test_temporal_candidates_match_fresh_detection_through_motion_and_radius_changes():
    x = np.array([[-1.0, -1.0, 0.06], [1.0, -1.0, 0.06], [1.0, 1.0, 0.06], [-1.0, 1.0, 0.06],
                  [-1.1, -1.1, 0.0], [1.1, -1.1, 0.0], [1.1, 1.1, 0.0], [-1.1, 1.1, 0.0]])
    tris = [[0, 1, 2], [0, 2, 3], [4, 5, 6], [4, 6, 7]]
    cached = oracle.World(x, tris, 4, [[0, 1]])
    st = ogc(0.1)
    reused = rebuilt = 0
    for frame in range(50):
        for i in range(4):
            x[i, 0] += 0.3 if frame == 12 else 0.0007 * (i + 1)
            x[i, 2] += 0.0002 * (i + 1)
        rq = 0.21 if frame >= 25 else 0.16
        a = cached.detect(x, rq, st)
        b = oracle.World(np.concatenate([np.array([[-1.0, -1.0, 0.06], [1.0, -1.0, 0.06], [1.0, 1.0, 0.06],
                                                   [-1.0, 1.0, 0.06]]), x[4:]]), tris, 4, [[0, 1]]).detect(x, rq, st)
        reused += int(not a["broad_phase_rebuilt"])
        rebuilt += int(a["broad_phase_rebuilt"])
        assert np.array_equal(a["radii"], b["radii"]), frame
        assert a["minimum_distance"] == b["minimum_distance"]
        assert a["vertex_face_candidates"] == b["vertex_face_candidates"]
        assert a["edge_edge_candidates"] == b["edge_edge_candidates"]
        assert keyset(a) == keyset(b)
        assert np.array_equal(a["epsilon"], b["epsilon"])
    assert reused > 30 and rebuilt >= 3
    x[4, 0] += 0.01
    with pytest.raises(oracle.OracleError):
        cached.detect(x, 0.21, st)


# tests/ogc_cache.rs:66-88
def test_cached_broad_phase_catches_a_pair_entering_the_query_radius():
    x = np.array([[0.0, 0.0, 0.065], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    w = oracle.World(x, [[1, 2, 3]], 1)
    st = ogc(0.02)
    a = w.detect(x, 0.05, st)
    assert a["vertex_face_candidates"] == 0
    x[0, 2] = 0.047
    b = w.detect(x, 0.05, st)
    assert not b["broad_phase_rebuilt"]
    assert b["vertex_face_candidates"] == 1
    assert abs(b["radii"][0] - 0.45 * 0.047) < 1e-14
    assert len(b["kinds"]) == 1
    assert b["active_contacts"] == 0
