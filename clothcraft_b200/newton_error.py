"""Error of the VBD step against the FP64 Newton reference, on the GPU.

  python -m clothcraft_b200.newton_error [--steps K] [--pcg 500] [--newton 30]

On the 256x256 self-contact fold (config 1) from its fold-phase state
(tests/golden/sheet256_fold_state.npz), samples K consecutive steps. For each
sampled state: the VBD step at the reference's 30 iterations and at 200, and
the Newton reference step (cc_solver_newton_step: src/solver.rs:422-646 with
the step's OGC contacts frozen), all from the same state; prints one JSON row
per step with the max and RMS per-vertex distance of each VBD result to the
Newton result and each result's relative force residual ||grad E|| /
||grad E(y)|| (unprojected). The trajectory advances with the 30-iteration
VBD step. Needs a CUDA device.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import scenes
from .vbd import VbdSolver

HERE = os.path.dirname(os.path.abspath(__file__))
FOLD = os.path.join(os.path.dirname(HERE), "tests", "golden", "sheet256_fold_state.npz")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--newton", type=int, default=30)
    ap.add_argument("--pcg", type=int, default=500)
    args = ap.parse_args(argv)
    sc = scenes.config1()
    z = np.load(FOLD)
    x, v, t = z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"])
    rows = []
    for k in range(args.steps):
        t0 = time.time()
        xn, rep = VbdSolver(sc).newton_step(x, v, sc.settings.to_c(), newton_iterations=args.newton,
                                            pcg_iterations=args.pcg)
        row = {"step": k, "newton": rep, "newton_s": time.time() - t0}
        nxt = None
        for iters in (30, 200):
            s = sc.settings
            s.iterations = iters
            s.residual_check_every = iters
            xv, vv, tv, m = VbdSolver(sc).step(x, v, t, s.to_c())
            d = np.linalg.norm(xv - xn, axis=1)
            row["vbd%d_max_m" % iters] = float(d.max())
            row["vbd%d_rms_m" % iters] = float(np.sqrt(np.mean(d * d)))
            row["vbd%d_relative_force_residual" % iters] = m["relative_force_residual"]
            if iters == 30:
                nxt = (xv, vv, tv)
        print(json.dumps(row), flush=True)
        rows.append(row)
        x, v, t = nxt
    return rows


if __name__ == "__main__":
    main()
