"""Scale run: the 1024x1024 crumple (config 4) on one GPU.

  python -m clothcraft_b200.crumple [--steps 120] [--side 1024] [--sample-every 12] [--learned PATH]

A 1024x1024 sheet (1,048,576 vertices, 2,093,058 triangles) with its four
corners pinned and driven toward the centre at 0.2 m/s (the caller moves the
pinned rows between steps, as the reference's callers do), radius 0.5 mm, 40
iterations per step. Every `sample-every`-th step also evaluates the relative
force residual after its last iteration. Prints one JSON line per step and a
summary (device ms per step, detection ms, vertex-iterations/s).
With --learned, the step starts from the learned guess (init_mode 1).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import scenes
from .vbd import VbdSolver


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--sample-every", type=int, default=12)
    ap.add_argument("--learned", default=None)
    ap.add_argument("--quiet", action="store_true")
    args = ap.parse_args(argv)
    sc = scenes.config4(n_side=args.side)
    t0 = time.time()
    g = VbdSolver(sc)
    create_s = time.time() - t0
    s = sc.settings
    if args.learned:
        from .learned import Mlp

        net = Mlp.load(args.learned)
        g.set_mlp(net, 1)
        s.init_mode = 1
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    free = int((sc.mesh.pinned == 0).sum())
    rows = []
    for k in range(args.steps):
        x = scenes.driven_corners(sc, x, t + s.dt)
        s.residual_check_every = s.iterations if (k + 1) % args.sample_every == 0 else 0
        x, v, t, m = g.step(x, v, t, s.to_c())
        row = {"step": k, "gpu_ms": m["gpu_compute_ms"], "detection_ms": m["detection_ms"],
               "detections": m["detection_updates"], "contact_terms": m["contact_terms"], "colors": m["colors"],
               "relative_residual": m["relative_residual"], "init_used": m["init_used"]}
        rows.append(row)
        if not args.quiet:
            print(json.dumps(row), flush=True)
    steady = rows[1:] if len(rows) > 1 else rows
    gpu_ms = float(np.mean([r["gpu_ms"] for r in steady]))
    res = [r["relative_residual"] for r in rows if r["relative_residual"] is not None]
    print(json.dumps({"summary": True, "vertices": sc.n, "triangles": int(len(sc.mesh.triangles)),
                      "solver_create_s": create_s, "steps": args.steps, "gpu_ms_per_step": gpu_ms,
                      "detection_ms_per_step": float(np.mean([r["detection_ms"] for r in steady])),
                      "vertex_iters_per_s": free * s.iterations / (gpu_ms / 1000.0),
                      "sampled_relative_residuals": res, "learned": bool(args.learned)}), flush=True)


if __name__ == "__main__":
    main()
