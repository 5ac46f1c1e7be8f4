"""Train the learned initial guess on trajectories the solver generates.

  python -m clothcraft_b200.train_init fold    [--out PATH] [--variants N] ...
  python -m clothcraft_b200.train_init garment [--out PATH] [--variants N] ...

`fold`: variants of the 256x256 self-contact fold (config1 with seeds other
than the benchmark's seed 1). Each variant runs `warm` plain steps into its
fold phase, then `steps` sampled steps solved to a tight residual target.
`garment`: seeded variants of the sewn garment proxy (config3), sampled from
the start. `crumple`: seeded 1024x1024 crumple sheets (config4) with their
corners driven inward between steps. Samples stay in HBM (features float32 [rows, 24], targets
float32 [rows, 3]); the network trains with the library's own FP32
forward/backward and Adam kernels (cc_mlp_train) and is saved as .npz.
Needs a CUDA device; there is no CPU path.
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import scenes
from .learned import Mlp
from .vbd import VbdSolver

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")


def sample_settings(sc, tolerance: float, cap: int, check: int, mode: int = 0, stall: int = 2):
    s = sc.settings
    s.iterations = cap
    s.residual_tolerance = tolerance
    s.residual_check_every = check
    s.stall_refresh = stall
    s.init_mode = mode
    return s.to_c()


def _make_garment(seed):
    return scenes.config3(seed=seed)


def _make_fold(seed):
    return scenes.config1(seed=seed)


def _make_crumple(seed):
    return scenes.config4(seed=seed)


def build_scenes(factory, seeds, workers: int = 0):
    """Scene generation is CPU work (Poisson-disk sampling for garments):
    spread it over a spawn-started process pool."""
    if workers <= 1 or len(seeds) <= 1:
        return [factory(s) for s in seeds]
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(factory, seeds)


def _drive(sc, solver):
    """Driven-corner kinematics of the crumple scene: move the pinned rows of
    the resident state to the next step's positions (breaks the adaptive-guess
    history, as the reference's callers do)."""
    x, v, t = solver.get_state()
    solver.set_state(scenes.driven_corners(sc, x, t + sc.settings.dt), v, t)


def evaluate(net, scene_list, warm: int, steps: int, tolerance: float = 1e-3, cap: int = 200, check: int = 2,
             log=print, driven: bool = False, acceleration: float = 0.0):
    """Plain vs learned init at a residual target on each scene: `warm` plain
    steps, then `steps` steps per init from the same state. Returns a list of
    per-scene dicts (mean iterations, device ms per step, learned-used fraction)."""
    out = []
    for sc in scene_list:
        g = VbdSolver(sc)
        g.set_state(sc.x0, sc.v0, 0.0)
        for _ in range(warm):
            if driven:
                _drive(sc, g)
            g.step_resident(sc.settings.to_c())
        start = g.get_state()
        row = {"scene": sc.name + ":" + sc.note}
        for mode, name in ((0, "plain"), (1, "learned")):
            h = VbdSolver(sc)
            if mode:
                h.set_mlp(net, 1)
            h.set_state(*start)
            st = sample_settings(sc, tolerance, cap, check, mode)
            st.acceleration = acceleration
            its, ms, used = [], [], []
            for _ in range(steps):
                if driven:
                    _drive(sc, h)
                m = h.step_resident(st)
                its.append(m["iterations"])
                ms.append(m["gpu_compute_ms"])
                used.append(m["init_used"])
            row[name] = {"mean_iterations": float(np.mean(its)), "ms_per_step": float(np.mean(ms)),
                         "used": float(np.mean(used))}
        row["time_ratio"] = row["plain"]["ms_per_step"] / row["learned"]["ms_per_step"]
        row["iteration_ratio"] = row["plain"]["mean_iterations"] / max(row["learned"]["mean_iterations"], 1e-9)
        log("  %s: plain %.1f it %.2f ms | learned %.1f it %.2f ms (used %.2f) | time x%.2f" % (
            row["scene"], row["plain"]["mean_iterations"], row["plain"]["ms_per_step"],
            row["learned"]["mean_iterations"], row["learned"]["ms_per_step"], row["learned"]["used"],
            row["time_ratio"]), flush=True)
        out.append(row)
    return out


def collect(scene_list, warm: int, steps: int, tolerance: float = 1e-4, cap: int = 200, check: int = 5,
            log=print, driven: bool = False):
    """Run each scene `warm` plain steps, then `steps` sampled steps; returns
    (features, targets) CUDA tensors with one row per free vertex and step."""
    import torch

    feats, targs = [], []
    for sc in scene_list:
        t0 = time.time()
        g = VbdSolver(sc)
        g.set_state(sc.x0, sc.v0, 0.0)
        for _ in range(warm):
            if driven:
                _drive(sc, g)
            g.step_resident(sc.settings.to_c())
        rows = g.free_vertices
        F = torch.empty((steps * rows, 24), dtype=torch.float32, device="cuda")
        T = torch.empty((steps * rows, 3), dtype=torch.float32, device="cuda")
        st = sample_settings(sc, tolerance, cap, check)
        its = []
        for k in range(steps):
            if driven:
                _drive(sc, g)
            m = g.step_sample(st, F[k * rows:(k + 1) * rows], T[k * rows:(k + 1) * rows])
            its.append(m["iterations"])
        feats.append(F)
        targs.append(T)
        log("  %s (%s): %d rows x %d steps, mean iterations %.1f, %.1fs" % (
            sc.name, sc.note, rows, steps, float(np.mean(its)), time.time() - t0), flush=True)
    return torch.cat(feats), torch.cat(targs)


def train(features, targets, steps: int = 6000, batch: int = 16384, lr: float = 1e-3, seed: int = 0, log=print):
    net = Mlp(seed)
    t0 = time.time()
    losses = net.train(features, targets, batch=batch, steps=steps, lr=lr, seed=seed)
    power = float((targets ** 2).sum(dim=1).mean())
    log("  trained %d Adam steps in %.1fs: loss %.4g -> %.4g (target power %.4g)" % (
        steps, time.time() - t0, float(losses[:20].mean()), float(losses[-200:].mean()), power), flush=True)
    return net, losses


def fold_scenes(variants: int, first_seed: int = 2, workers: int = 0):
    return build_scenes(_make_fold, [first_seed + k for k in range(variants)], workers)


def garment_scenes(variants: int, first_seed: int = 100, workers: int = 0):
    return build_scenes(_make_garment, [first_seed + k for k in range(variants)], workers)


def crumple_scenes(variants: int, first_seed: int = 200, workers: int = 0):
    return build_scenes(_make_crumple, [first_seed + k for k in range(variants)], workers)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["fold", "garment", "crumple"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--variants", type=int, default=None)
    ap.add_argument("--warm", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--train-steps", type=int, default=6000)
    ap.add_argument("--tolerance", type=float, default=1e-4)
    ap.add_argument("--workers", type=int, default=min(16, os.cpu_count() or 1))
    ap.add_argument("--evaluate", type=int, default=0, help="held-out seeds to evaluate on after training")
    ap.add_argument("--eval-steps", type=int, default=30)
    ap.add_argument("--weights", default=None, help="skip training: evaluate these weights")
    ap.add_argument("--acceleration", type=float, default=0.0, help="Chebyshev rho of the evaluation steps")
    args = ap.parse_args(argv)
    out = args.out or os.path.join(DATA, "%s_init_mlp.npz" % args.kind)
    if args.weights:
        net = Mlp.load(args.weights)
    else:
        if args.kind == "fold":
            scs = fold_scenes(args.variants or 6, workers=args.workers)
            warm, steps = (args.warm if args.warm is not None else 190), (args.steps or 40)
        elif args.kind == "garment":
            scs = garment_scenes(args.variants or 50, workers=args.workers)
            warm, steps = (args.warm if args.warm is not None else 0), (args.steps or 100)
        else:
            scs = crumple_scenes(args.variants or 2, workers=args.workers)
            warm, steps = (args.warm if args.warm is not None else 20), (args.steps or 20)
        print("collecting %d variants" % len(scs), flush=True)
        F, T = collect(scs, warm, steps, tolerance=args.tolerance, driven=args.kind == "crumple")
        net, losses = train(F, T, steps=args.train_steps)
        del F, T
        os.makedirs(os.path.dirname(out), exist_ok=True)
        np.savez(out, params=net.parameters(), losses=losses, scenes=np.array([s.name + ":" + s.note for s in scs]))
        print("saved", out, flush=True)
    if args.evaluate:
        if args.kind == "fold":
            held = fold_scenes(args.evaluate, first_seed=1000, workers=args.workers)
            warm = 200
        elif args.kind == "garment":
            held = garment_scenes(args.evaluate, first_seed=10000, workers=args.workers)
            warm = 10
        else:
            held = crumple_scenes(args.evaluate, first_seed=20000, workers=args.workers)
            warm = 30
        print("evaluating on %d held-out seeds (tolerance 1e-3)" % len(held), flush=True)
        rows = evaluate(net, held, warm, args.eval_steps, driven=args.kind == "crumple",
                        acceleration=args.acceleration)
        tr = [r["time_ratio"] for r in rows]
        ir = [r["iteration_ratio"] for r in rows]
        print("held-out summary: time ratio plain/learned mean %.3f median %.3f; iteration ratio mean %.3f median %.3f"
              % (float(np.mean(tr)), float(np.median(tr)), float(np.mean(ir)), float(np.median(ir))), flush=True)


if __name__ == "__main__":
    main()
