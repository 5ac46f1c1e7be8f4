"""Run-directory records (metrics.jsonl, run.json) in the reference's serde
layout (src/vbd.rs:61-83, src/ogc/world.rs:14-22, src/bin/cloth-fit.rs:127-172),
written from oracle steps on the CPU."""
import json
from types import SimpleNamespace

import numpy as np

import oracle
from clothcraft_b200 import scenes, trajectory

# VbdMetrics field order (src/vbd.rs:61-83)
METRIC_KEYS = ["time_s", "dt_s", "step_ms", "detection_ms", "contact_profile", "solve_ms", "gpu_compute_ms",
               "iterations", "contacts", "contact_terms", "detection_updates", "broad_phase_rebuilds",
               "truncated_vertices", "minimum_distance_m", "max_seam_gap_m", "extension_p95_percent",
               "extension_max_percent", "residual_rms_n"]
PROFILE_KEYS = ["refit_ms", "candidates_ms", "narrow_ms", "candidate_pairs", "aabb_rejections"]
RUN_KEYS = ["backend", "steps", "settings", "vertices", "triangles", "wall_ms", "mean_step_ms", "last", "seams",
            "scope"]


def contact_scene():
    return scenes.small_sheet(8, seed=0, height=0.104, side=0.2, pins=(), radius=0.002)


def test_metrics_rows_and_run_report_follow_the_reference_layout(tmp_path):
    sc = contact_scene()
    st = sc.settings
    st.iterations = 12
    o = oracle.Solver(sc)
    log = trajectory.RunLog(str(tmp_path), sc, st, gpu=False, backend="cpu-f64-vbd-ogc")
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    mets = []
    for _ in range(4):
        x, v, t, m = o.step(x, v, t, st.to_c())
        log.record(m)
        mets.append(m)
    report = log.finish(x)
    lines = (tmp_path / "metrics.jsonl").read_text().splitlines()
    assert len(lines) == 4
    for line, m in zip(lines, mets):
        row = json.loads(line)
        assert list(row) == METRIC_KEYS
        assert list(row["contact_profile"]) == PROFILE_KEYS
        assert row["gpu_compute_ms"] is None  # CPU path: no hardware timestamps
        assert row["iterations"] == 12 and row["contact_terms"] == m["contact_terms"]
        assert row["minimum_distance_m"] == m["minimum_distance_m"]
        assert isinstance(row["residual_rms_n"], float)
    assert row["contact_terms"] > 0
    on_disk = json.loads((tmp_path / "run.json").read_text())
    assert on_disk == report
    assert list(on_disk)[:len(RUN_KEYS)] == RUN_KEYS and "library_settings" not in on_disk
    assert on_disk["steps"] == 4 and on_disk["vertices"] == sc.n and on_disk["last"] == json.loads(lines[-1])
    s = on_disk["settings"]
    assert list(s) == ["dt", "iterations", "damping", "gravity", "contact"]
    assert list(s["contact"]) == ["radius", "stiffness", "relaxation", "refresh_fraction"]
    assert s["iterations"] == 12 and s["gravity"] == [0.0, -9.81, 0.0] and s["contact"]["radius"] == 0.002
    assert on_disk["seams"] == []  # no stitches on a plain sheet


def test_extensions_are_listed_only_when_on(tmp_path):
    sc = contact_scene()
    st = sc.settings
    st.residual_tolerance, st.residual_check_every, st.acceleration = 1e-3, 2, 0.95
    log = trajectory.RunLog(str(tmp_path), sc, st.to_c(), gpu=True)
    report = log.finish(sc.x0)
    assert report["library_settings"] == {"init_mode": 0, "residual_tolerance": 1e-3, "residual_check_every": 2,
                                          "stall_refresh": 0, "acceleration": 0.95}
    assert report["settings"]["contact"]["radius"] == 0.002 and report["last"] is None


def test_stitch_gaps_and_per_seam_maxima(tmp_path):
    mesh = SimpleNamespace(stitch_offsets=np.array([0, 2, 4, 7]), stitch_vertices=np.array([0, 1, 2, 3, 0, 1, 2]),
                           stitch_weights=np.array([1.0, -1.0, 1.0, -1.0, 0.5, 0.5, -1.0]), triangles=np.zeros((1, 3)))
    x = np.array([[0.0, 0.0, 0.0], [0.0, 0.003, 0.0], [1.0, 0.0, 0.0], [1.0, 0.0, 0.004]])
    gaps = trajectory.stitch_gaps(mesh, x)
    assert np.allclose(gaps, [0.003, 0.004, np.linalg.norm([-1.0, 0.0015, 0.0])])
    sc = SimpleNamespace(mesh=mesh, n=4)
    log = trajectory.RunLog(str(tmp_path), sc, scenes.StepSettings(), gpu=True)
    report = log.finish(x, seams=[("side", [0, 1]), ("shoulder", [2])])
    assert report["seams"] == [{"id": "side", "max_gap_m": 0.004},
                               {"id": "shoulder", "max_gap_m": float(gaps[2])}]


def test_non_finite_values_are_written_as_null():
    m = dict.fromkeys(["time_s", "dt_s", "step_ms", "detection_ms", "refit_ms", "candidates_ms", "narrow_ms",
                       "solve_ms", "gpu_compute_ms", "minimum_distance_m", "max_seam_gap_m",
                       "extension_p95_percent", "extension_max_percent"], 1.0)
    m.update(dict.fromkeys(["candidate_pairs", "aabb_rejections", "iterations", "contacts", "contact_terms",
                            "detection_updates", "broad_phase_rebuilds", "truncated_vertices"], 3))
    m["minimum_distance_m"] = float("inf")
    m["residual_rms_n"] = None
    row = trajectory.metrics_row(m)
    assert row["minimum_distance_m"] is None and row["residual_rms_n"] is None and row["gpu_compute_ms"] == 1.0
    json.dumps(row, allow_nan=False)
