"""GPU OGC detection parity: the CUDA world against the oracle on identical
positions. Contact keys, mollifier epsilons, radii and minimum distances are
compared bit for bit (integer/index work and FP64 decisions made with the
same operation order); candidate pair lists are compared as sorted lists.
Runs through the C ABI (clothcraft_b200.vbd -> libclothcraft_b200.so)."""
import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.abi import cc_ogc_settings
from clothcraft_b200.vbd import OgcWorld, VbdError

pytestmark = pytest.mark.gpu


def ogc(r, stiffness=100000.0, relaxation=0.45, refresh=0.01):
    return cc_ogc_settings(r, stiffness, relaxation, refresh)


def assert_same_contacts(a, b, ctx=""):
    assert len(a["kinds"]) == len(b["kinds"]), (ctx, len(a["kinds"]), len(b["kinds"]))
    assert np.array_equal(a["kinds"], b["kinds"]), ctx
    assert np.array_equal(a["vertices"], b["vertices"]), ctx
    assert np.array_equal(a["counts"], b["counts"]), ctx
    assert np.array_equal(a["epsilon"].view(np.uint64), b["epsilon"].view(np.uint64)), ctx
    assert np.array_equal(a["radii"].view(np.uint64), b["radii"].view(np.uint64)), ctx
    assert np.array_equal(a["incident_offsets"], b["incident_offsets"]), ctx
    assert np.array_equal(a["incident"], b["incident"]), ctx
    for k in ("active_contacts", "vertex_face_candidates", "edge_edge_candidates", "broad_phase_rebuilt"):
        assert a[k] == b[k], (ctx, k, a[k], b[k])
    assert np.float64(a["minimum_distance"]).view(np.uint64) == np.float64(b["minimum_distance"]).view(np.uint64)


def both(x, tris, moving, excluded=()):
    return OgcWorld(x, tris, moving, excluded), oracle.World(x, tris, moving, excluded)


REFERENCE_CASES = [
    # (positions, triangles, moving, query radius, contact radius) from tests/ogc.rs
    ([[0.0, 0.1, 0.1], [-1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]],
     [[1, 2, 3], [2, 1, 4]], 1, 0.25, 0.2),
    ([[0.0, -0.03, 0.04], [-1.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, -1.0]],
     [[1, 2, 3], [2, 1, 4]], 1, 0.2, 0.1),
    ([[-1.0, -1.0, 0.1], [1.0, -1.0, 0.1], [0.0, 1.0, 0.1], [0.0, 0.0, 0.0], [0.01, 0.0, -1.0], [0.0, 0.01, -1.0]],
     [[0, 1, 2], [3, 4, 5]], 3, 0.2, 0.15),
    ([[-1.0, 0.0, 0.1], [1.0, 0.0, 0.1], [-1.0, -1.0, 0.1], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0], [1.0, 1.0, 0.0]],
     [[0, 1, 2], [3, 4, 5]], 6, 0.2, 0.15),
    ([[-1.0, 0.0, 0.1], [1.0, 0.0, 0.1], [-1.0, -1.0, 0.1], [0.0, -1.0, 0.0], [0.0, 1.0, 0.0], [1.0, 1.0, 0.0]],
     [[3, 4, 5], [0, 1, 2]], 3, 0.2, 0.15),
    ([[0.0, 0.0, 0.02], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]], [[1, 2, 3]], 1, 0.03, 0.01),
    ([[0.0, 0.0, 0.00305], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]], [[1, 2, 3]], 1, 0.006, 0.003),
]


@pytest.mark.parametrize("case", range(len(REFERENCE_CASES)))
def test_reference_scenes_match_oracle_bit_for_bit(case):
    x, tris, moving, rq, r = REFERENCE_CASES[case]
    x = np.array(x)
    g, o = both(x, tris, moving)
    assert_same_contacts(g.detect(x, rq, ogc(r)), o.detect(x, rq, ogc(r)), case)


def test_folded_surface_and_shared_feature_known_answers_on_gpu():
    x, tris, moving, rq, r = REFERENCE_CASES[0]
    s = OgcWorld(np.array(x), tris, moving).detect(np.array(x), rq, ogc(r))
    assert int((s["kinds"] == 2).sum()) == 2  # tests/ogc.rs:101-121
    x, tris, moving, rq, r = REFERENCE_CASES[1]
    s = OgcWorld(np.array(x), tris, moving).detect(np.array(x), rq, ogc(r))
    assert len(s["kinds"]) == 1 and s["kinds"][0] == 1  # tests/ogc.rs:123-135
    x, tris, moving, rq, r = REFERENCE_CASES[3]
    s = OgcWorld(np.array(x), tris, moving).detect(np.array(x), rq, ogc(r))
    assert np.any(s["kinds"] == 3)  # EE protects crossing edges (tests/ogc.rs:159-170)


def test_initial_intersection_and_settings_fail_closed_on_gpu():
    x = np.array([[0.0, 0.0, -1.0], [0.0, 0.0, 1.0], [2.0, 0.0, 0.0], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0],
                  [0.0, 1.0, 0.0]])
    w = OgcWorld(x, [[0, 1, 2], [3, 4, 5]], 3)
    with pytest.raises(VbdError):
        w.validate_start(x)
    x = np.array([[0.0, 0.0, 0.1], [-1.0, -1.0, 0.0], [1.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    w = OgcWorld(x, [[1, 2, 3]], 1)
    with pytest.raises(VbdError):
        w.detect(x, 0.01, ogc(0.15))  # query radius below contact radius
    with pytest.raises(VbdError):
        w.detect(x, 0.2, ogc(0.003, relaxation=0.5))
    x2 = x.copy()
    x2[1, 0] += 0.01
    with pytest.raises(VbdError):
        w.detect(x2, 0.2, ogc(0.15))  # fixed geometry moved
    # near-coplanar shared-vertex regression (tests/ogc.rs:277-292)
    y = np.array([[0.194131180644, 0.943517088890, 0.091018132865],
                  [0.183311969042, 0.970439314842, 0.101929388940],
                  [0.197149559855, 0.954595983028, 0.076061360538],
                  [0.195560514927, 0.972076416016, 0.068995960057],
                  [0.188853010535, 0.980777919292, 0.085684590042]]).astype(np.float32).astype(np.float64)
    OgcWorld(y, [[0, 1, 2], [3, 2, 4]], 5).validate_start(y)


def layered_scene(offset=(0.0, 0.0, 0.0)):
    """src/ogc/world.rs:566-633: three 5x5 layers 3 mm apart, two moving."""
    off = np.array(offset)
    rest, tris = [], []
    for layer in range(3):
        for y in range(5):
            for xx in range(5):
                rest.append(off + np.array([xx * 0.008, y * 0.008, layer * 0.003]))
        for y in range(4):
            for xx in range(4):
                a = layer * 25 + y * 5 + xx
                tris += [[a, a + 1, a + 5], [a + 1, a + 6, a + 5]]
    return np.array(rest), tris


@pytest.mark.parametrize("offset", [(0.0, 0.0, 0.0), (1e6, -2e6, 3e6)])
def test_cache_reuse_frames_match_oracle(offset):
    rest, tris = layered_scene(offset)
    g, o = both(rest, tris, 50, [[0, 25], [1, 26]])
    st = ogc(0.003)
    rebuilt = reused = 0
    for frame in range(24):
        x = rest.copy()
        for i in range(50):
            a = frame * 0.15 + i * 0.31
            x[i] += np.array([np.sin(a) * 0.0004, np.cos(a) * 0.0003, np.sin(a) * 0.0002])
            if frame >= 18:
                x[i, 0] += 0.004
        rq = 0.006 if frame <= 11 else (0.009 if frame <= 15 else 0.004)
        a, b = g.detect(x, rq, st), o.detect(x, rq, st)
        assert_same_contacts(a, b, frame)
        assert a["aabb_rejections"] == b["aabb_rejections"]
        assert a["candidate_pairs"] == b["candidate_pairs"]
        rebuilt += int(a["broad_phase_rebuilt"])
        reused += int(not a["broad_phase_rebuilt"])
    assert rebuilt > 1 and reused > 0


def folded_sheet(n=24, seed=3):
    """A sheet folded into three close layers (self contact everywhere) above
    a sphere; deterministic."""
    sc = scenes.small_sheet(n, seed=seed, radius=0.002, side=0.3, height=0.12)
    x = sc.x0.copy()
    u = (x[:, 0] + 0.15) / 0.3
    # z-fold: layers at heights separated by ~4 mm, jittered
    rng = np.random.default_rng(seed)
    x[:, 1] = 0.12 + 0.004 * np.floor(u * 2.999) + rng.uniform(-4e-4, 4e-4, len(x))
    x[:, 0] = -0.15 + 0.3 * (u * 3 % 1.0)
    return sc, x


def test_self_contact_fold_matches_oracle_and_candidate_lists_are_identical():
    sc = scenes.small_sheet(24, seed=3, radius=0.002, side=0.3, height=0.12)
    obs = sc.obstacle
    n = sc.n
    _, xf = folded_sheet(24, 3)
    x_all = np.concatenate([xf, obs.vertices])
    tris = np.concatenate([sc.mesh.triangles, obs.triangles + n])
    g, o = both(x_all, tris, n)
    for rq, r in ((0.004, 0.002), (0.008, 0.002), (0.006, 0.003)):
        a, b = g.detect(x_all, rq, ogc(r)), o.detect(x_all, rq, ogc(r))
        assert len(a["kinds"]) > 100
        assert_same_contacts(a, b, rq)
    for search in (0.004, 0.0101):
        vf_g, ee_g = g.candidates(x_all, search)
        vf_o, ee_o = o.candidates(x_all, search)
        assert len(vf_o) > 0 and len(ee_o) > 0
        assert np.array_equal(vf_g, vf_o)
        assert np.array_equal(ee_g, ee_o)
    assert np.array_equal(g.edges(), o.edges())


def test_random_displacements_against_oracle():
    rng = np.random.default_rng(11)
    sc = scenes.small_sheet(20, seed=5, radius=0.002, side=0.2, height=0.102)
    n = sc.n
    obs = sc.obstacle
    tris = np.concatenate([sc.mesh.triangles, obs.triangles + n])
    x0 = np.concatenate([sc.x0, obs.vertices])
    g, o = both(x0, tris, n)
    for k in range(6):
        x = x0.copy()
        x[:n, 1] -= 0.002 * k
        x[:n] += rng.uniform(-1e-3, 1e-3, (n, 3))
        a, b = g.detect(x, 0.008, ogc(0.002)), o.detect(x, 0.008, ogc(0.002))
        assert_same_contacts(a, b, k)


def test_tree_rebuild_period_does_not_change_detections():
    """The LBVH policy (refit the first build's trees, or rebuild them every
    k-th candidate rebuild) changes only the traversal cost: worlds created on
    the flat sheet and detected while it folds into layers give the oracle's
    contact sets and candidate lists for every period."""
    sc = scenes.small_sheet(24, seed=3, radius=0.002, side=0.3, height=0.12)
    obs = sc.obstacle
    n = sc.n
    _, xf = folded_sheet(24, 3)
    flat = np.concatenate([sc.x0, obs.vertices])
    tris = np.concatenate([sc.mesh.triangles, obs.triangles + n])
    worlds = []
    for period in (0, 1, 3):
        w = OgcWorld(flat, tris, n)
        w.set_tree_rebuild_period(period)
        worlds.append(w)
    o = oracle.World(flat, tris, n)
    with pytest.raises(VbdError):
        worlds[0].set_tree_rebuild_period(-1)
    for frame in range(8):
        s = frame / 7.0
        x = flat.copy()
        x[:n] = (1.0 - s) * sc.x0 + s * xf
        ref = o.detect(x, 0.004, ogc(0.002))
        for w in worlds:
            assert_same_contacts(w.detect(x, 0.004, ogc(0.002)), ref, frame)
    vf_o, ee_o = o.candidates(x, 0.0101)
    for w in worlds:
        vf_g, ee_g = w.candidates(x, 0.0101)
        assert np.array_equal(vf_g, vf_o) and np.array_equal(ee_g, ee_o)
