"""Run a few steps of the benchmark workload for a profiler.

  python -m clothcraft_b200.profile_fold [--steps 2] [--lanes 4] [--learned] [--fixed N] [--acceleration RHO]

The 256x256 self-contact fold from its committed fold-phase state
(tests/golden/sheet256_fold_state.npz), stepped to the benchmark's residual
target (1e-3, checked every 2 iterations, stall refresh 2, cap 200), or a
fixed iteration count with --fixed; --acceleration sets the Chebyshev
estimate of the residual-target form (the benchmark uses 0.95). Nothing is
timed here: wrap it in
`ncu` to see the launches of exactly this workload.
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from . import scenes
from .vbd import VbdSolver

HERE = os.path.dirname(os.path.abspath(__file__))
FOLD_STATE = os.path.join(os.path.dirname(HERE), "tests", "golden", "sheet256_fold_state.npz")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--fixed", type=int, default=0)
    ap.add_argument("--acceleration", type=float, default=0.0)
    ap.add_argument("--precision", type=int, default=0, help="sweep arithmetic: 0 FP64, 1 FP32 assembly")
    ap.add_argument("--lanes32", type=int, default=8 | 4 << 8)
    ap.add_argument("--profile", action="store_true", help="time each iteration's sweeps with CUDA events")
    ap.add_argument("--graphs", action="store_true", help="launch the iteration chunks as CUDA graphs")
    ap.add_argument("--tree-period", type=int, default=None,
                    help="LBVH rebuild period at candidate rebuilds (0: refit the first build's trees)")
    args = ap.parse_args(argv)
    sc = scenes.config1()
    z = np.load(FOLD_STATE)
    g = VbdSolver(sc).set_lanes(args.lanes).set_lanes32(args.lanes32)
    s = sc.settings
    s.sweep_precision = args.precision
    if args.fixed:
        s.iterations = args.fixed
    else:
        s.iterations, s.residual_tolerance, s.residual_check_every, s.stall_refresh = 200, 1e-3, 2, 2
        s.acceleration = args.acceleration
    if args.learned:
        from .learned import Mlp

        g.set_mlp(Mlp.load(os.path.join(HERE, "data", "fold_init_mlp.npz")), 1)
        s.init_mode = 1
    g.set_state(z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"]))
    g.set_profiling(args.profile)
    g.set_graphs(args.graphs)
    if args.tree_period is not None:
        g.world.set_tree_rebuild_period(args.tree_period)
    for k in range(args.steps):
        m = g.step_resident(s.to_c())
        print("step %d: %d iterations, %.2f ms, residual %s, sweeps %.3f ms in %d launches, detection %.3f ms "
              "host (%d; device refit %.3f candidates %.3f narrow %.3f), colouring %.3f ms" % (
                  k, m["iterations"], m["gpu_compute_ms"], m["relative_residual"], m["sweep_ms"],
                  m["sweep_launches"], m["detection_ms"], m["detection_updates"], m["refit_ms"],
                  m["candidates_ms"], m["narrow_ms"], m["color_ms"]), flush=True)


if __name__ == "__main__":
    main()
