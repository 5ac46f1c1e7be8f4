"""Trajectory records in ClothCraft's run-directory formats.

The reference's drivers (`cloth-fit run_ogc`, src/bin/cloth-fit.rs:127-172;
`motion_probe`, examples/motion_probe.rs:73-95) write one JSON object per
step to `metrics.jsonl` (the serde form of `VbdMetrics`, src/vbd.rs:61-83,
with `DetectionProfile`, src/ogc/world.rs:14-22, nested as
`contact_profile`) and a summary `run.json` (backend, steps, settings,
sizes, wall time, last row, per-seam maximum gap, scope). This module writes
the same records from this library's step metrics, so tools that read a
reference run directory read ours. Keys, nesting and key order follow the
serde derives; `Option` fields are `null` when absent, and so is any
non-finite number (serde_json writes `null` for those). Values are compared as
JSON, not byte for byte: float spelling may differ from serde_json's.

  log = RunLog(out_dir, scene, settings)
  for ...: log.record(solver.step_resident(settings))
  report = log.finish(x)                # writes run.json, returns it

The library's extensions (initial-guess mode, residual target, stall
refresh, acceleration) are not part of `VbdSettings`; `run.json` lists them
under `library_settings` when any is switched on.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

BACKEND = "cuda-b200-vbd-ogc"
SCOPE = ("OGC two-sided VF/EE normal contact, self-contact, isotropic conservative bounds; local seam "
         "exclusions; no friction; FP64 VBD and OGC on one GPU; iterations fixed or until the relative "
         "residual target")


def _num(v):
    if v is None:
        return None
    if isinstance(v, (int, np.integer)):
        return int(v)
    v = float(v)
    return v if math.isfinite(v) else None


def settings_json(settings) -> dict:
    """VbdSettings (src/vbd.rs:18-25) with OgcSettings (src/ogc/world.rs:35-44)
    in serde form, from a StepSettings or a cc_vbd_settings."""
    if hasattr(settings, "contact"):  # cc_vbd_settings
        c = settings.contact
        contact = {"radius": c.radius, "stiffness": c.stiffness, "relaxation": c.relaxation,
                   "refresh_fraction": c.refresh_fraction}
        gravity = [settings.gravity[k] for k in range(3)]
    else:
        contact = {"radius": settings.radius, "stiffness": settings.stiffness, "relaxation": settings.relaxation,
                   "refresh_fraction": settings.refresh_fraction}
        gravity = list(settings.gravity)
    return {"dt": _num(settings.dt), "iterations": int(settings.iterations), "damping": _num(settings.damping),
            "gravity": [_num(g) for g in gravity], "contact": {k: _num(v) for k, v in contact.items()}}


def library_settings(settings) -> dict:
    """The extensions of cc_vbd_settings, or {} when all are off."""
    ext = {"init_mode": int(settings.init_mode), "residual_tolerance": _num(settings.residual_tolerance),
           "residual_check_every": int(settings.residual_check_every),
           "stall_refresh": int(settings.stall_refresh), "acceleration": _num(settings.acceleration)}
    return ext if any(ext.values()) else {}


def metrics_row(m: dict, gpu: bool = True) -> dict:
    """One `metrics.jsonl` row: VbdMetrics in serde field order. `gpu_compute_ms`
    is `Some` for device steps (the reference fills it from hardware
    timestamps) and `null` for the CPU path."""
    return {
        "time_s": _num(m["time_s"]),
        "dt_s": _num(m["dt_s"]),
        "step_ms": _num(m["step_ms"]),
        "detection_ms": _num(m["detection_ms"]),
        "contact_profile": {
            "refit_ms": _num(m["refit_ms"]),
            "candidates_ms": _num(m["candidates_ms"]),
            "narrow_ms": _num(m["narrow_ms"]),
            "candidate_pairs": int(m["candidate_pairs"]),
            "aabb_rejections": int(m["aabb_rejections"]),
        },
        "solve_ms": _num(m["solve_ms"]),
        "gpu_compute_ms": _num(m["gpu_compute_ms"]) if gpu else None,
        "iterations": int(m["iterations"]),
        "contacts": int(m["contacts"]),
        "contact_terms": int(m["contact_terms"]),
        "detection_updates": int(m["detection_updates"]),
        "broad_phase_rebuilds": int(m["broad_phase_rebuilds"]),
        "truncated_vertices": int(m["truncated_vertices"]),
        "minimum_distance_m": _num(m["minimum_distance_m"]),
        "max_seam_gap_m": _num(m["max_seam_gap_m"]),
        "extension_p95_percent": _num(m["extension_p95_percent"]),
        "extension_max_percent": _num(m["extension_max_percent"]),
        "residual_rms_n": _num(m["residual_rms_n"]),
    }


def stitch_gaps(mesh, x) -> np.ndarray:
    """|sum_j w_j x_j| of every stitch (the probe gap of src/garment/seam.rs:420-425)."""
    x = np.asarray(x, np.float64)
    off = np.asarray(mesh.stitch_offsets, np.int64)
    vs = np.asarray(mesh.stitch_vertices, np.int64)
    ws = np.asarray(mesh.stitch_weights, np.float64)
    out = np.zeros(max(len(off) - 1, 0))
    for s in range(len(out)):
        a, b = off[s], off[s + 1]
        out[s] = float(np.linalg.norm((x[vs[a:b]] * ws[a:b, None]).sum(axis=0)))
    return out


class RunLog:
    """`metrics.jsonl` row by row, then `run.json` (src/bin/cloth-fit.rs:127-172)."""

    def __init__(self, out_dir: str, scene, settings, gpu: bool = True, backend: str = BACKEND):
        os.makedirs(out_dir, exist_ok=True)
        self.out_dir = out_dir
        self.scene = scene
        self.settings = settings
        self.gpu = gpu
        self.backend = backend
        self.rows = []
        self._log = open(os.path.join(out_dir, "metrics.jsonl"), "w")
        self._t0 = time.perf_counter()

    def record(self, m: dict) -> dict:
        row = metrics_row(m, self.gpu)
        self._log.write(json.dumps(row, allow_nan=False) + "\n")
        self.rows.append(row)
        return row

    def finish(self, x, seams=None) -> dict:
        """Write run.json. `seams`: list of (id, stitch indices); by default one
        seam "stitches" over all stitches when the mesh has any."""
        wall_ms = (time.perf_counter() - self._t0) * 1000.0
        self._log.close()
        mesh = self.scene.mesh
        gaps = stitch_gaps(mesh, x)
        if seams is None:
            seams = [("stitches", np.arange(len(gaps)))] if len(gaps) else []
        report = {
            "backend": self.backend,
            "steps": len(self.rows),
            "settings": settings_json(self.settings),
            "vertices": int(self.scene.n),
            "triangles": int(len(mesh.triangles)),
            "wall_ms": wall_ms,
            "mean_step_ms": wall_ms / len(self.rows) if self.rows else 0.0,
            "last": self.rows[-1] if self.rows else None,
            "seams": [{"id": sid, "max_gap_m": float(gaps[np.asarray(idx, np.int64)].max()) if len(idx) else 0.0}
                      for sid, idx in seams],
            "scope": SCOPE,
        }
        ext = library_settings(self.settings)
        if ext:
            report["library_settings"] = ext
        with open(os.path.join(self.out_dir, "run.json"), "w") as f:
            f.write(json.dumps(report, indent=2, allow_nan=False))
        return report
