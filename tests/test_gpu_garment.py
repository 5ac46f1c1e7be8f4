"""Sewn garment proxy (two Poisson-disk/Delaunay panels around a capsule,
joined by penalty sewing springs whose vertex pairs are excluded from
contact) on the GPU against the oracle: stitch terms in the sweep, seam
exclusions in detection, seam-gap metric. A coarse variant of the scene keeps
the oracle fast; the code paths are those of the full-size scene.

Bars: per-vertex positions within 1e-5 m (bar (a)) while both solvers follow
their own trajectories; contact lists bit for bit at identical positions."""
import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes
from clothcraft_b200.vbd import VbdSolver

from test_gpu_ogc import assert_same_contacts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def garment():
    return scenes.config3(seed=5, spacing=0.012)


def test_garment_steps_match_oracle(garment):
    sc = garment
    st = sc.settings.to_c()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    xg, vg, tg = sc.x0.copy(), sc.v0.copy(), 0.0
    xo, vo, to = sc.x0.copy(), sc.v0.copy(), 0.0
    for k in range(4):
        xg, vg, tg, mg = g.step(xg, vg, tg, st)
        xo, vo, to, mo = o.step(xo, vo, to, st)
        assert np.abs(xg - xo).max() <= 1e-5, k
        assert abs(mg["max_seam_gap_m"] - mo["max_seam_gap_m"]) <= 1e-9, k
        assert mg["contact_terms"] == mo["contact_terms"], k
    # the seams pull the panels together: the gap shrinks from 0.4 m
    assert mg["max_seam_gap_m"] < 0.4


def test_garment_contacts_with_seam_exclusions_match_oracle(garment):
    sc = garment
    g = VbdSolver(sc)
    o = oracle.Solver(sc)
    x = sc.x0.copy()
    # bring the back panel to 1.5 mm behind the front one: every stitched
    # pair sits 1.5 mm apart and is excluded, other close pairs are contacts
    ids = sc.mesh.stitch_vertices.reshape(-1, 2)
    n0 = int(ids[0, 1] - ids[0, 0])
    x[n0:, 2] = x[0, 2] - 0.0015
    xa = g.positions(x)
    cg = g.world.detect(xa, 0.004, sc.settings.ogc_c())
    co = o.world.detect(xa, 0.004, sc.settings.ogc_c())
    assert_same_contacts(cg, co, "garment")
    pairs = {tuple(sorted(p)) for p in ids.tolist()}
    for kind, vs, cnt in zip(cg["kinds"], cg["vertices"], cg["counts"]):
        if kind == 0:  # point-point: never a stitched pair
            assert tuple(sorted(vs[:2].tolist())) not in pairs
    assert len(cg["kinds"]) > 0 and n0 > 0
