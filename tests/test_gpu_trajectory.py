"""metrics.jsonl rows written from GPU steps agree with the oracle's rows on
every field the two backends compute alike (counts bit for bit, distances and
residuals to the parity bars); timings and gpu_compute_ms differ by design."""
import json

import numpy as np
import pytest

import oracle
from clothcraft_b200 import scenes, trajectory
from clothcraft_b200.vbd import VbdSolver

pytestmark = pytest.mark.gpu

EXACT = ["iterations", "contacts", "contact_terms", "detection_updates", "broad_phase_rebuilds"]


def test_gpu_rows_match_oracle_rows(tmp_path):
    sc = scenes.small_sheet(16, seed=0, height=0.104, side=0.2, pins=(), radius=0.002)
    st = sc.settings.to_c()
    g = VbdSolver(sc)
    o = oracle.Solver(sc, threads=8)
    lg = trajectory.RunLog(str(tmp_path / "gpu"), sc, st, gpu=True)
    lo = trajectory.RunLog(str(tmp_path / "cpu"), sc, st, gpu=False, backend="cpu-f64-vbd-ogc")
    # each backend follows its own trajectory (as in the parity tests), so both
    # keep their adaptive-guess history
    xg, vg, tg = sc.x0.copy(), sc.v0.copy(), 0.0
    xo, vo, to = sc.x0.copy(), sc.v0.copy(), 0.0
    for _ in range(6):
        xg, vg, tg, mg = g.step(xg, vg, tg, st)
        xo, vo, to, mo = o.step(xo, vo, to, st)
        lg.record(mg)
        lo.record(mo)
    assert np.abs(xg - xo).max() <= 1e-5
    rg = lg.finish(xg)
    ro = lo.finish(xo)
    rows_g = [json.loads(s) for s in (tmp_path / "gpu" / "metrics.jsonl").read_text().splitlines()]
    rows_o = [json.loads(s) for s in (tmp_path / "cpu" / "metrics.jsonl").read_text().splitlines()]
    assert len(rows_g) == len(rows_o) == 6
    for a, b in zip(rows_g, rows_o):
        assert list(a) == list(b)
        for k in EXACT:
            assert a[k] == b[k], k
        assert a["contact_profile"]["candidate_pairs"] == b["contact_profile"]["candidate_pairs"]
        assert abs(a["minimum_distance_m"] - b["minimum_distance_m"]) <= 1e-9 * b["minimum_distance_m"]
        assert abs(a["truncated_vertices"] - b["truncated_vertices"]) <= 2
        assert abs(a["time_s"] - b["time_s"]) <= 1e-12 and a["dt_s"] == b["dt_s"]
        assert abs(a["residual_rms_n"] - b["residual_rms_n"]) <= 1e-6 * b["residual_rms_n"] + 1e-15
        assert abs(a["extension_max_percent"] - b["extension_max_percent"]) <= 1e-6
        assert a["gpu_compute_ms"] > 0 and b["gpu_compute_ms"] is None
    assert rows_g[-1]["contact_terms"] > 0
    assert rg["settings"] == ro["settings"] and rg["backend"] == trajectory.BACKEND
