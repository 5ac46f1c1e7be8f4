"""Error of the VBD step against the FP64 Newton reference (test infrastructure).

  python -m oracle.newton_error [--steps K] [--threads T]

On the 256x256 fold (config 1) from its committed fold-phase state, samples K
consecutive steps: the VBD step of the oracle restatement (equal to the GPU
step to 1e-5 m per vertex, tests/test_gpu_vbd.py) at 30 and 200 iterations,
and the Newton-PCG step of src/solver.rs:422-646 with the step's OGC contacts
frozen, all from the same state; prints per step the max and RMS per-vertex
distance of each VBD result to the Newton result and each result's relative
force residual ||grad E|| / ||grad E(y)|| (unprojected, Newton objective).
The trajectory advances with the 30-iteration VBD step.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from clothcraft_b200 import scenes  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--newton-iterations", type=int, default=30)
    ap.add_argument("--pcg-iterations", type=int, default=500)
    args = ap.parse_args(argv)
    sc = scenes.config1()
    z = np.load(os.path.join(ROOT, "tests", "golden", "sheet256_fold_state.npz"))
    x, v, t = z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])
    rows = []
    for k in range(args.steps):
        t0 = time.time()
        o = oracle.Solver(sc, threads=args.threads)
        xn, _, conv, its = o.newton_step(x, v, sc.settings.to_c(), newton_iterations=args.newton_iterations,
                                         pcg_iterations=args.pcg_iterations, threads=args.threads)
        res = {"step": k, "newton_converged": conv, "newton_iterations": its,
               "newton_relative_residual": o.relative_residual(x, v, sc.settings.to_c(), xn, args.threads)}
        nxt = None
        for iters in (30, 200):
            s = sc.settings
            s.iterations = iters
            vb = oracle.Solver(sc, threads=args.threads)
            xv, vv, tv, _ = vb.step(x, v, t, s.to_c())
            d = np.linalg.norm(xv - xn, axis=1)
            res["vbd%d_max_m" % iters] = float(d.max())
            res["vbd%d_rms_m" % iters] = float(np.sqrt(np.mean(d * d)))
            res["vbd%d_relative_residual" % iters] = o.relative_residual(x, v, sc.settings.to_c(), xv, args.threads)
            if iters == 30:
                nxt = (xv, vv, tv)
        res["seconds"] = time.time() - t0
        print(json.dumps(res), flush=True)
        rows.append(res)
        x, v, t = nxt
    return rows


if __name__ == "__main__":
    main()
