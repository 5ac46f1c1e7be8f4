"""Train the learned initial guess on trajectories the solver generates.

  python -m clothcraft_b200.train_init fold    [--out PATH] [--variants N] ...
  python -m clothcraft_b200.train_init garment [--out PATH] [--variants N] ...

`fold`: variants of the 256x256 self-contact fold (config1 with seeds other
than the benchmark's seed 1). Each variant runs `warm` plain steps into its
fold phase, then `steps` sampled steps solved to a tight residual target.
`garment`: seeded variants of the sewn garment proxy (config3), sampled from
the start. Samples stay in HBM (features float32 [rows, 24], targets
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


def sample_settings(sc, tolerance: float, cap: int, check: int):
    s = sc.settings
    s.iterations = cap
    s.residual_tolerance = tolerance
    s.residual_check_every = check
    s.init_mode = 0
    return s.to_c()


def collect(scene_list, warm: int, steps: int, tolerance: float = 1e-4, cap: int = 200, check: int = 5,
            log=print):
    """Run each scene `warm` plain steps, then `steps` sampled steps; returns
    (features, targets) CUDA tensors with one row per free vertex and step."""
    import torch

    feats, targs = [], []
    for sc in scene_list:
        t0 = time.time()
        g = VbdSolver(sc)
        g.set_state(sc.x0, sc.v0, 0.0)
        for _ in range(warm):
            g.step_resident(sc.settings.to_c())
        rows = g.free_vertices
        F = torch.empty((steps * rows, 24), dtype=torch.float32, device="cuda")
        T = torch.empty((steps * rows, 3), dtype=torch.float32, device="cuda")
        st = sample_settings(sc, tolerance, cap, check)
        its = []
        for k in range(steps):
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


def fold_scenes(variants: int, first_seed: int = 2):
    return [scenes.config1(seed=first_seed + k) for k in range(variants)]


def garment_scenes(variants: int, first_seed: int = 100):
    return [scenes.config3(seed=first_seed + k) for k in range(variants)]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["fold", "garment"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--variants", type=int, default=None)
    ap.add_argument("--warm", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--train-steps", type=int, default=6000)
    ap.add_argument("--tolerance", type=float, default=1e-4)
    args = ap.parse_args(argv)
    if args.kind == "fold":
        scs = fold_scenes(args.variants or 6)
        warm, steps = (args.warm if args.warm is not None else 190), (args.steps or 40)
    else:
        scs = garment_scenes(args.variants or 50)
        warm, steps = (args.warm if args.warm is not None else 0), (args.steps or 100)
    out = args.out or os.path.join(DATA, "%s_init_mlp.npz" % args.kind)
    print("collecting %d variants" % len(scs), flush=True)
    F, T = collect(scs, warm, steps, tolerance=args.tolerance)
    net, losses = train(F, T, steps=args.train_steps)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez(out, params=net.parameters(), losses=losses, rows=F.shape[0],
             scenes=np.array([s.name + ":" + s.note for s in scs]))
    print("saved", out, flush=True)


if __name__ == "__main__":
    main()
