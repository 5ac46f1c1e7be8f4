"""Kernel timeline of the benchmark's fold steps: GPU busy and idle time.

  python -m clothcraft_b200.timeline_fold [--steps 8] [--warmup 5] [--direct] [--trace out.json]

Steps the 256x256 self-contact fold from its committed fold-phase state with
the benchmark's settings (learned guess, relative residual 1e-3 checked every
2 iterations, stall refresh 2, Chebyshev rho 0.95, lanes 8 | cap 4) and
records the device activity of the timed steps (kernels, memcpys, memsets)
through CUPTI, via torch.profiler. Prints per step: the span from the first
to the last record, the union of busy intervals (concurrent kernels on the
detection's two streams counted once), the idle remainder, the largest idle
gaps by the records on either side, and the kernels by total time. Profiling
slows the host side a little, so the absolute times are above the bench's.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import tempfile

import numpy as np

from . import scenes
from .vbd import VbdSolver

HERE = os.path.dirname(os.path.abspath(__file__))
FOLD_STATE = os.path.join(os.path.dirname(HERE), "tests", "golden", "sheet256_fold_state.npz")
MLP_PATH = os.path.join(HERE, "data", "fold_init_mlp.npz")
DEVICE_CATS = ("kernel", "gpu_memcpy", "gpu_memset")


def device_records(trace_path):
    with open(trace_path) as f:
        tr = json.load(f)
    ev = [e for e in tr["traceEvents"] if e.get("ph") == "X" and e.get("cat") in DEVICE_CATS]
    ev.sort(key=lambda e: e["ts"])
    return ev


def busy_and_gaps(ev):
    """Union of the busy intervals (us) and the idle gaps between them, each
    gap with the names of the records that end before it and start after it."""
    busy, gaps = 0.0, []
    s0, e0, last = ev[0]["ts"], ev[0]["ts"] + ev[0]["dur"], ev[0]["name"]
    for e in ev[1:]:
        s, t = e["ts"], e["ts"] + e["dur"]
        if s > e0:
            busy += e0 - s0
            gaps.append((s - e0, last, e["name"]))
            s0, e0 = s, t
        elif t > e0:
            e0 = t
        if t >= e0:
            last = e["name"]
    busy += e0 - s0
    return busy, gaps


def short(name, k=48):
    name = name.replace("cc::", "").replace("(anonymous namespace)::", "")
    return name.split("(")[0][:k]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--direct", action="store_true", help="launch every kernel directly (no CUDA graphs)")
    ap.add_argument("--trace", default=None, help="also keep the Chrome trace at this path")
    args = ap.parse_args(argv)
    import torch
    from torch.profiler import ProfilerActivity, profile

    from .learned import Mlp

    torch.cuda.set_device(0)
    sc = scenes.config1()
    z = np.load(FOLD_STATE)
    g = VbdSolver(sc).set_lanes(8 | 4 << 8)
    g.set_mlp(Mlp.load(MLP_PATH), 1)
    g.set_graphs(not args.direct)
    s = sc.settings
    s.iterations, s.residual_tolerance, s.residual_check_every, s.stall_refresh = 200, 1e-3, 2, 2
    s.acceleration = 0.95
    s.init_mode = 1
    st = s.to_c()
    g.set_state(z["x"].astype(np.float64), z["v"].astype(np.float64), float(z["time"]))
    for _ in range(args.warmup):
        g.step_resident(st)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
        mets = [g.step_resident(st) for _ in range(args.steps)]
        torch.cuda.synchronize()
    path = args.trace or os.path.join(tempfile.mkdtemp(), "fold_trace.json")
    prof.export_chrome_trace(path)
    ev = device_records(path)
    K = args.steps
    span = ev[-1]["ts"] + ev[-1]["dur"] - ev[0]["ts"]
    busy, gaps = busy_and_gaps(ev)
    print("%d steps (iterations %s), %d device records: span %.3f ms/step, busy %.3f ms/step, idle %.3f ms/step" % (
        K, [m["iterations"] for m in mets], len(ev), span / 1e3 / K, busy / 1e3 / K, (span - busy) / 1e3 / K))
    agg, cnt = collections.Counter(), collections.Counter()
    for gap, a, b in gaps:
        agg[(short(a), short(b))] += gap
        cnt[(short(a), short(b))] += 1
    print("largest idle gaps (us per step, count, record before -> record after):")
    for (a, b), t in agg.most_common(15):
        print("  %8.1f  %5d  %s -> %s" % (t / K, cnt[(a, b)], a, b))
    kt, kc = collections.Counter(), collections.Counter()
    for e in ev:
        kt[short(e["name"], 60)] += e["dur"]
        kc[short(e["name"], 60)] += 1
    print("device time by record (us per step, count, average us):")
    for k, t in kt.most_common(20):
        print("  %8.1f  %5d  %7.2f  %s" % (t / K, kc[k], t / kc[k], k))


if __name__ == "__main__":
    main()
