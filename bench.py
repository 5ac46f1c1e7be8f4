#!/usr/bin/env python
"""Benchmark: VBD+OGC steps/s on the 256x256 self-contact fold.

Workload (one "step" = one implicit-Euler VBD step with on-GPU OGC
detection, colouring and 30 colour sweeps): a 256x256-vertex sheet (65,536
vertices, 130,050 triangles), 1 m side, dropped from y=0.5 m with a seeded
tilt onto a fixed r=0.3 m sphere so that it folds onto itself; OGC radius
1 mm, contact stiffness 1e4 N/m, dt 1/60 s, 30 iterations. Synthetic, seeded.
Timing starts in the fold phase: both arms load the scene's state after
PHASE_START steps (t = 3.33 s, ~95k retained contact terms; committed as
tests/golden/sheet256_fold_state.npz with its generator), then run W warm-up
steps and K timed steps.

  python bench.py [--gpus N --steps K --warmup W]      # B200 library
  python bench.py --impl reference [...]                # CPU path (oracle restatement)

Prints one JSON line (rank 0). A single cloth does not shard, so N GPUs run
N independent replicas ("replicas only"); value = N*K / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "VBD steps/s (256x256 self-contact fold, 30 iterations, 1 GPU replica)"
UNIT = "steps/s"
L2_FLUSH_BYTES = 256 << 20
PHASE_START = 200


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def sweep_traffic():
    """DRAM bytes per k_sweep launch recorded from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_sweep_sheet256_fold.md")) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


def workload():
    from clothcraft_b200 import scenes

    return scenes.config1()


FOLD_STATE = os.path.join(ROOT, "tests", "golden", "sheet256_fold_state.npz")


def fold_state():
    """Fold-phase start state (x, v, time), identical bytes for both arms."""
    d = np.load(FOLD_STATE)
    return (d["x"].astype(np.float64), d["v"].astype(np.float64), float(d["time"]))


def config_dict(sc, n_gpus):
    return {
        "workload": "sheet256_fold: 256x256 sheet (65,536 v / 130,050 t), 1 m, seeded tilt, dropped onto a "
                    "fixed r=0.3 m icosphere (2,562 v), OGC VF+EE self-contact r=1 mm, k=1e4 N/m, "
                    "dt=1/60 s, 30 VBD iterations, StVK-mapped membrane (mu=1e4, lambda=2e4 N/m)",
        "vertices": int(sc.n),
        "triangles": int(len(sc.mesh.triangles)),
        "iterations": int(sc.settings.iterations),
        "l2": "flushed between timed steps (256 MiB device write outside the timed events)",
        "phase": "timed steps start at step %d + warm-up (fold phase, contact-rich)" % PHASE_START,
        "parallelism": "replicas x%d (single cloth does not shard)" % n_gpus,
        "note": sc.note,
    }


def static_bytes_per_sweep(sc):
    """Algorithmic bytes of one colour sweep over every free vertex, from the
    byte model B_v = 64 + 36 T_v + 24 H_v + 12 N_v + 24 S_v (+ 28 per contact
    incidence entry, added per step from the detection)."""
    m = sc.mesh
    n = sc.n
    T = np.bincount(m.triangles.reshape(-1).astype(np.int64), minlength=n)
    H = np.bincount(m.hinges.reshape(-1).astype(np.int64), minlength=n)
    S = np.bincount(m.stitch_vertices.astype(np.int64), minlength=n) if len(m.stitch_vertices) else np.zeros(n, int)
    # unique neighbour vertices referenced by incident triangles and hinges
    pairs = []
    for arr in (m.triangles, m.hinges):
        a = arr.astype(np.int64)
        k = a.shape[1]
        for i in range(k):
            for j in range(k):
                if i != j:
                    pairs.append(a[:, i] * n + a[:, j])
    u = np.unique(np.concatenate(pairs))
    N = np.bincount(u // n, minlength=n)
    free = m.pinned == 0
    B = 64 + 36 * T + 24 * H + 12 * N + 24 * S
    return float(B[free].sum())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_reference_run(sc, state, steps, budget_s, threads):
    """The reference CPU path (FP64 oracle restatement, all host threads) on
    the same workload from `state`; stops after `steps` or `budget_s`."""
    import oracle

    o = oracle.Solver(sc, threads=threads)
    st = sc.settings.to_c()
    x, v, t = state
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        x, v, t, _ = o.step(x, v, t, st)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return done, dt


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from clothcraft_b200 import scenes  # noqa: F401

    sc = workload()
    threads = os.cpu_count() or 1
    st = sc.settings.to_c()
    import oracle

    o = oracle.Solver(sc, threads=threads)
    x, v, t = fold_state()
    budget = float(os.environ.get("CC_REFERENCE_BUDGET_S", "150"))
    t0 = time.perf_counter()
    warm = 0
    for _ in range(args.warmup):
        if time.perf_counter() - t0 > budget / 2:
            break
        x, v, t, _ = o.step(x, v, t, st)
        warm += 1
    done, dt = cpu_reference_run(sc, (x, v, t), args.steps, budget - (time.perf_counter() - t0), threads)
    value = done / dt
    sample = "%d warm-up + %d timed steps from the fold-phase state (bounded to ~%.0f s), %d host threads" % (
        warm, done, budget, threads)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": done, "warmup": warm,
        "ms_per_step": 1000.0 * dt / max(done, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(sc, world),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "C++ FP64 restatement of the reference CPU path (VbdSolver::step + OgcWorld::detect); the Rust "
                "original cannot be compiled in this environment",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lanes", type=int, default=0,
                    help="lanes per vertex solve (1..32); 0 = autotune on the first step")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)

    from clothcraft_b200 import native
    from clothcraft_b200.vbd import VbdSolver

    L = native.load()
    L.cc_set_device(local if world > 1 else 0)
    sc = workload()
    st = sc.settings.to_c()
    solver = VbdSolver(sc)
    if args.lanes:
        if L.cc_solver_set_lanes(solver.h, args.lanes) != 0:
            raise SystemExit("invalid --lanes %d" % args.lanes)
    stream = torch.cuda.ExternalStream(L.cc_solver_stream(solver.h))
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    solver.set_state(*fold_state())
    for _ in range(args.warmup):
        solver.step_resident(st)
    warm_state = solver.get_state()

    def timed(step_fn, k):
        evs = []
        metrics = []
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            metrics.append(step_fn())
            with torch.cuda.stream(stream):
                b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs), metrics

    # ---- device-resident throughput (value); clocks sampled over all GPU legs
    clocks = ClockSampler(local).__enter__()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, mets = timed(lambda: solver.step_resident(st), args.steps)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t_max = ms
    if dist:
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * args.steps / (t_max / 1000.0)

    # ---- end to end through the C ABI with host buffers (e2e)
    x, v, t = warm_state
    n = sc.n
    state = {"x": x.copy(), "v": v.copy(), "t": t}

    def host_step():
        state["x"], state["v"], state["t"], m = solver.step(state["x"], state["v"], state["t"], st)
        return m

    host_step()  # warm the host path once
    if dist:
        dist.barrier()
    ms_e2e, _ = timed(host_step, args.steps)
    e2e_max = ms_e2e
    if dist:
        tt = torch.tensor([ms_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_max = float(tt.item())
    e2e_value = world * args.steps / (e2e_max / 1000.0)

    # ---- per-launch sweep timing (events around every sweep launch), same
    # state and step count as the value leg, for the roofline
    solver.set_state(*warm_state)
    L.cc_solver_set_profiling(solver.h, 1)
    _, mets = timed(lambda: solver.step_resident(st), args.steps)
    L.cc_solver_set_profiling(solver.h, 0)
    clocks.__exit__(None, None, None)

    # ---- roofline of the dominant kernel (colour sweep)
    peak, peak_kind = load_peaks()
    static_b = static_bytes_per_sweep(sc)
    sweep_ms = sum(m["sweep_ms"] for m in mets)
    sweeps = sum(m["sweep_launches"] for m in mets)
    iters = sum(m["iterations"] for m in mets)
    alg_bytes = sum(static_b * m["iterations"] + 28.0 * m["contact_incidence"] * m["iterations"] for m in mets)
    achieved = alg_bytes / (sweep_ms / 1000.0) / 1e9 if sweep_ms > 0 else None
    free = int((sc.mesh.pinned == 0).sum())
    launches = int(sum(m["kernel_launches"] for m in mets))

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        done, dt = cpu_reference_run(sc, warm_state, 2, 25.0, threads)
        cpu = {"value": done / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "%d step(s) of the same workload from the post-warm-up state, FP64 oracle restatement of "
                         "the reference CPU path, %d threads" % (done, threads)}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": config_dict(sc, world),
        "vertex_iters_per_s": world * free * iters / (t_max / 1000.0),
        "roofline": {
            "kernel": "k_sweep (colour sweep)",
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": sweep_traffic(),
            "traffic_note": "dram read+write bytes per k_sweep launch from one ncu capture "
                            "(profiles/k_sweep_sheet256_fold.md, cold cache)",
            "peak_kind": peak_kind,
            "sweep_launches": int(sweeps),
            "avg_launch_us": 1000.0 * sweep_ms / max(sweeps, 1),
            "algorithmic_bytes_per_step": alg_bytes / args.steps,
            "algorithmic_bytes_per_launch": alg_bytes / max(sweeps, 1),
            "sweep_share_of_step": sweep_ms / ms if ms > 0 else None,
        },
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * n * 32, "d2h_bytes_per_step": 2 * n * 32},
        "gpu_launches": launches,
        "lanes_per_vertex": int(L.cc_solver_get_lanes(solver.h)),
        "breakdown_ms_per_step": {
            "detection": sum(m["detection_ms"] for m in mets) / args.steps,
            "coloring": sum(m["color_ms"] for m in mets) / args.steps,
            "sweeps": sweep_ms / args.steps,
        },
        "clocks": clocks.summary(),
        "detections_per_step": sum(m["detection_updates"] for m in mets) / args.steps,
        "contact_terms_last": mets[-1]["contact_terms"] if mets else None,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
