#!/usr/bin/env python
"""Benchmark: VBD+OGC steps/s at equal residual on the 256x256 self-contact fold.

Workload (one "step" = one implicit-Euler VBD step with on-GPU OGC detection,
colouring and colour sweeps): a 256x256-vertex sheet (65,536 vertices,
130,050 triangles), 1 m side, dropped from y=0.5 m with a seeded tilt onto a
fixed r=0.3 m sphere so that it folds onto itself; OGC radius 1 mm, contact
stiffness 1e4 N/m, dt 1/60 s. Synthetic, seeded. Timing starts in the fold
phase: every arm loads the scene's state after PHASE_START steps (t = 3.33 s,
~95k retained contact terms; tests/golden/sheet256_fold_state.npz with its
generator), then runs W warm-up and K timed steps.

Equal residual: every step iterates until the relative force residual
||P grad E(x)|| / ||grad E(y)|| <= 1e-3 (evaluated every 2 iterations, at most
200 iterations, the reference's limit). `value` is the learned-init form
(MLP correction of the adaptive guess, energy-checked) with Chebyshev
acceleration of the sweeps (rho 0.95, restarted when a residual evaluation
rises); the plain adaptive init runs alongside with the same acceleration
(`plain`), both inits run without it (`unaccelerated`, the reference's
iteration), and so does the reference's fixed 30-iteration step
(`fixed_iterations`). The network is clothcraft_b200/data/fold_init_mlp.npz,
trained by `python -m clothcraft_b200.train_init fold` on other seeds.

Further keys time the other configurations on the same box: `batched` (96
uneven instances in one solver, ~3.66M vertices, 20 iterations), `garment`
(the sewn two-panel scene at 20 iterations and at the 1e-3 target) and
`crumple` (the 1024x1024 sheet with driven corners, 40 iterations, host
arrays); --no-batched / --no-garment / --no-crumple skip them.

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

METRIC = ("VBD steps/s at equal residual (relative force residual <= 1e-3), learned init vs plain, "
          "256x256 self-contact fold, 1 GPU")
TOLERANCE = 1e-3
CHECK_EVERY = 2
ITERATION_CAP = 200
FIXED_ITERATIONS = 30
STALL_REFRESH = 2  # refresh the OGC balls after 2 checks without a 5 % residual decrease
ACCELERATION = 0.95  # Chebyshev spectral-radius estimate of the equal-residual legs
SWEEP_PRECISION = 0  # sweep arithmetic of the timed legs: 0 FP64, 1 FP32 element assembly
MLP_PATH = os.path.join(ROOT, "clothcraft_b200", "data", "fold_init_mlp.npz")
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


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one k_sweep
# launch on the fold, from one ncu capture of the profiling driver (the first
# sweep launch of a 30-iteration step from the fold-phase state; cold cache,
# since ncu flushes the caches between its passes):
#   ncu --set full --clock-control none -k regex:k_sweep -s 0 -c 2 \
#       python -m clothcraft_b200.profile_fold --steps 1 --lanes 1032 --fixed 30
# (first launch: 23,093,248 B read + 256 B written)
SWEEP_TRAFFIC_BYTES = 23093504.0


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
                    "dt=1/60 s, StVK-mapped membrane (mu=1e4, lambda=2e4 N/m); iterations until the "
                    "relative force residual <= 1e-3 (checked every 2, cap 200, stall refresh after 2 "
                    "checks without a 5 % decrease)",
        "vertices": int(sc.n),
        "triangles": int(len(sc.mesh.triangles)),
        "residual_tolerance": TOLERANCE,
        "residual_check_every": CHECK_EVERY,
        "iteration_cap": ITERATION_CAP,
        "stall_refresh": STALL_REFRESH,
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


def step_settings(sc, mode, iterations=None, acceleration=ACCELERATION, precision=None):
    """Equal-residual settings (mode 0 adaptive, 1 learned) with the given
    Chebyshev acceleration, or a fixed iteration count with neither a
    residual target nor acceleration when `iterations` is given. `precision`
    is the sweep arithmetic (0 FP64, 1 FP32 assembly; default SWEEP_PRECISION)."""
    s = sc.settings
    s.sweep_precision = SWEEP_PRECISION if precision is None else precision
    if iterations is None:
        s.iterations, s.residual_tolerance, s.residual_check_every = ITERATION_CAP, TOLERANCE, CHECK_EVERY
        s.stall_refresh = STALL_REFRESH
        s.acceleration = acceleration
    else:
        s.iterations, s.residual_tolerance, s.residual_check_every = iterations, 0.0, 0
        s.stall_refresh = 0
        s.acceleration = 0.0
    s.init_mode = mode
    return s.to_c()


def cpu_reference_run(sc, state, steps, budget_s, threads, warmup=0, warmup_budget_s=None):
    """The reference CPU path (FP64 oracle restatement, all host threads) at
    equal residual on the same workload from `state`: up to `warmup` untimed
    steps (within `warmup_budget_s`), then `steps` timed steps, stopping early
    only once the timed steps have taken `budget_s`. Returns (done, seconds,
    iterations and final relative force residuals of the timed steps, warm-up
    steps run)."""
    import oracle

    o = oracle.Solver(sc, threads=threads)
    st = step_settings(sc, 0, acceleration=0.0)  # the reference's iteration and init
    x, v, t = state
    t0 = time.perf_counter()
    warm = 0
    for _ in range(warmup):
        if warmup_budget_s is not None and time.perf_counter() - t0 > warmup_budget_s:
            break
        x, v, t, _ = o.step(x, v, t, st)
        warm += 1
    done, its, force = 0, [], []
    t1 = time.perf_counter()
    while done < steps:
        x, v, t, m = o.step(x, v, t, st)
        its.append(int(m["iterations"]))
        force.append(m["relative_force_residual"])
        done += 1
        if time.perf_counter() - t1 > budget_s:
            break
    return done, time.perf_counter() - t1, (its, force), warm


BATCHED_STEPS = 5
BATCHED_WARMUP = 2


def batched_leg(rank, world, leg, L):
    """Config 2 (96 uneven sheets with their own spheres, ~3.66M vertices,
    20 fixed iterations): this rank's share of the instances as one batched
    solver, BATCHED_WARMUP untimed steps (the first autotunes), then
    BATCHED_STEPS device-timed steps; max over ranks."""
    from clothcraft_b200 import scenes
    from clothcraft_b200.batch import shard
    from clothcraft_b200.vbd import VbdSolver

    instances = scenes.config2_instances()
    mine = shard(instances, rank, world)
    solver = VbdSolver.batch([instances[i] for i in mine])
    st = instances[0].settings.to_c()
    for _ in range(BATCHED_WARMUP):
        solver.step_resident(st)
    ms, mets = leg(solver, lambda: solver.step_resident(st), BATCHED_STEPS)
    vertices = sum(instances[i].n for i in mine)
    total = sum(sc.n for sc in instances)
    its = [int(m["iterations"]) for m in mets]
    return {"workload": "config 2: %d sheets of 32..320 vertices a side (%d vertices in all), each with its own "
                        "sphere, 1-4 pinned corners, moduli x U(0.5, 2); contact r 2 mm, 20 iterations"
                        % (len(instances), total),
            "steps": BATCHED_STEPS, "steps_per_s": BATCHED_STEPS / (ms / 1000.0), "ms_per_step": ms / BATCHED_STEPS,
            "vertex_iters_per_s": world * vertices * sum(its) / (ms / 1000.0),
            "vertices_per_rank": vertices, "instances_per_rank": len(mine),
            "lanes": int(L.cc_solver_get_lanes(solver.h)),
            "timing": "CUDA events on the solver stream, max over ranks; replicas shard the instances"}


GARMENT_WARMUP = 3
GARMENT_STEPS = 5


def garment_leg(rank, world, leg, L):
    """Config 3's scene: two seeded 0.6 x 0.7 m panels (~20k vertices each,
    Poisson-disk sampling and Delaunay triangulation) 5 cm either side of a
    fixed capsule, joined along the sides and shoulders by 1e3 N/m penalty
    stitches, contact radius 1 mm. The adaptive (plain) initial guess: the
    learned form needs a network trained on this scene, which is not shipped.
    Two settings from the same state: the config's fixed 20 iterations, and
    the equal-residual form of the headline legs (1e-3 relative residual,
    checked every 2, cap 200, stall refresh 2, Chebyshev rho 0.95).
    GARMENT_WARMUP untimed steps, then GARMENT_STEPS device-timed steps each."""
    from clothcraft_b200 import scenes
    from clothcraft_b200.vbd import VbdSolver

    sc = scenes.config3()
    out = {"workload": "config 3 scene: two Poisson-disk panels (%d vertices, %d triangles) around a capsule, "
                       "side and shoulder stitches 1e3 N/m, contact r 1 mm, adaptive initial guess"
                       % (sc.n, len(sc.mesh.triangles))}
    free = int((sc.mesh.pinned == 0).sum())
    for name, target in (("fixed_20_iterations", False), ("residual_1e-3", True)):
        s = sc.settings
        s.init_mode = 0
        if target:
            s.iterations, s.residual_tolerance, s.residual_check_every = ITERATION_CAP, TOLERANCE, CHECK_EVERY
            s.stall_refresh, s.acceleration = STALL_REFRESH, ACCELERATION
        else:
            s.iterations, s.residual_tolerance, s.residual_check_every = 20, 0.0, 20
            s.stall_refresh, s.acceleration = 0, 0.0
        st = s.to_c()
        g = VbdSolver(sc)
        g.set_state(sc.x0, sc.v0, 0.0)
        for _ in range(GARMENT_WARMUP):
            g.step_resident(st)
        ms, mets = leg(g, lambda: g.step_resident(st), GARMENT_STEPS)
        its = [int(m["iterations"]) for m in mets]
        out[name] = {"steps_per_s": world * GARMENT_STEPS / (ms / 1000.0), "ms_per_step": ms / GARMENT_STEPS,
                     "vertex_iters_per_s": world * free * sum(its) / (ms / 1000.0),
                     "mean_iterations": float(np.mean(its)),
                     "mean_final_relative_residual": float(np.mean([m["relative_residual"] for m in mets]))}
    out["timing"] = "CUDA events on the solver stream, max over ranks; replicas"
    return out


CRUMPLE_WARMUP = 30   # untimed steps from the flat start (the corners travel 0.1 m), the first autotunes
CRUMPLE_STEPS = 4


def crumple_leg(rank, world, max_over_ranks):
    """Config 4: the 1024x1024 sheet (1,048,576 vertices, 2,093,058 triangles)
    with its corners pinned and driven inward at 0.2 m/s, radius 0.5 mm, 40
    iterations. The caller moves the pinned rows between steps, so each step
    goes through host arrays (VbdSolver.step: x and v copied in and out); after
    CRUMPLE_WARMUP untimed steps, CRUMPLE_STEPS steps are timed by the host
    clock around the blocking step calls (the corner update outside it), each
    with one FP64 relative-residual evaluation after its last iteration. Every
    rank steps its own replica; the time is the maximum over ranks."""
    from clothcraft_b200 import scenes
    from clothcraft_b200.vbd import VbdSolver

    sc = scenes.config4()
    t0 = time.perf_counter()
    g = VbdSolver(sc)
    create_s = time.perf_counter() - t0
    s = sc.settings
    x, v, t = sc.x0.copy(), sc.v0.copy(), 0.0
    s.residual_check_every = 0
    st = s.to_c()
    for _ in range(CRUMPLE_WARMUP):
        x = scenes.driven_corners(sc, x, t + s.dt)
        x, v, t, _ = g.step(x, v, t, st)
    s.residual_check_every = s.iterations
    st = s.to_c()
    wall, mets = 0.0, []
    for _ in range(CRUMPLE_STEPS):
        x = scenes.driven_corners(sc, x, t + s.dt)
        h0 = time.perf_counter()
        x, v, t, m = g.step(x, v, t, st)
        wall += time.perf_counter() - h0
        mets.append(m)
    ms = max_over_ranks(1000.0 * wall)
    free = int((sc.mesh.pinned == 0).sum())
    return {"workload": "config 4: 1024x1024 sheet (%d vertices, %d triangles), 1 m, corners driven inward at "
                        "0.2 m/s, OGC r 0.5 mm, 40 iterations; timed steps %d..%d from the flat start"
                        % (sc.n, len(sc.mesh.triangles), CRUMPLE_WARMUP, CRUMPLE_WARMUP + CRUMPLE_STEPS - 1),
            "steps": CRUMPLE_STEPS, "steps_per_s": world * CRUMPLE_STEPS / (ms / 1000.0),
            "ms_per_step": ms / CRUMPLE_STEPS,
            "vertex_iters_per_s": world * free * sum(int(m["iterations"]) for m in mets) / (ms / 1000.0),
            "detection_ms_per_step": float(np.mean([m["detection_ms"] for m in mets])),
            "detections_per_step": float(np.mean([m["detection_updates"] for m in mets])),
            "coloring_ms_per_step": float(np.mean([m["color_ms"] for m in mets])),
            "coloring_rounds_per_step": float(np.mean([m["color_rounds"] for m in mets])),
            "contact_terms_last": int(mets[-1]["contact_terms"]),
            "relative_residuals": [None if m["relative_residual"] is None else float(m["relative_residual"])
                                   for m in mets],
            "relative_force_residuals": [None if m["relative_force_residual"] is None
                                         else float(m["relative_force_residual"]) for m in mets],
            "residual_note": "relative_residuals: the KKT residual of the step's OGC-ball-constrained problem; "
                             "relative_force_residuals: the unprojected force norm, which keeps the outward "
                             "forces on vertices held at their ball boundaries (next to the driven corners)",
            "solver_create_s": create_s,
            "timing": "host clock around each blocking VbdSolver.step on host arrays (x, v in and out), max over "
                      "ranks; replicas"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sc = workload()
    threads = os.cpu_count() or 1
    # timed part bounded so that warm-up and timed steps end within a few minutes
    # (the oracle takes ~8-11 s a fold step on 16 host threads)
    budget = float(os.environ.get("CC_REFERENCE_BUDGET_S", "200"))
    warm_budget = float(os.environ.get("CC_REFERENCE_WARMUP_BUDGET_S", "45"))
    done, dt, (its, force), warm = cpu_reference_run(sc, fold_state(), args.steps, budget, threads,
                                                     warmup=args.warmup, warmup_budget_s=warm_budget)
    value = done / dt
    sample = ("%d warm-up + %d timed steps from the fold-phase state at equal residual (timed part bounded to "
              "%.0f s, warm-up to %.0f s), %d host threads, iterations %s" % (warm, done, budget, warm_budget,
                                                                              threads, its))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": done, "warmup": warm,
        "ms_per_step": 1000.0 * dt / max(done, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(sc, world),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "mean_iterations": float(np.mean(its)) if its else None,
        "max_final_relative_force_residual": float(np.max(force)) if force else None,
        "note": "C++ FP64 restatement of the reference CPU path (VbdSolver::step + OgcWorld::detect, adaptive "
                "init) run to the same residual target; the Rust original cannot be compiled in this "
                "environment",
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-instances (config 2) leg")
    ap.add_argument("--no-crumple", action="store_true", help="skip the 1024x1024 crumple (config 4) leg")
    ap.add_argument("--no-garment", action="store_true", help="skip the garment-proxy (config 3) leg")
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
    from clothcraft_b200.learned import Mlp
    from clothcraft_b200.vbd import VbdSolver

    if not os.path.exists(MLP_PATH):
        raise SystemExit("missing %s: train it with `python -m clothcraft_b200.train_init fold`" % MLP_PATH)
    L = native.load()
    L.cc_set_device(local if world > 1 else 0)
    sc = workload()
    net = Mlp.load(MLP_PATH)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    start = fold_state()

    # every solver after the first uses the lane variant the first one tuned,
    # so that all legs take the same trajectory bit for bit
    tuned = {"lanes": args.lanes, "lanes32": 0}

    def make(mode, iterations=None, acceleration=ACCELERATION, precision=None):
        s = VbdSolver(sc)
        if tuned["lanes"] and L.cc_solver_set_lanes(s.h, tuned["lanes"]) != 0:
            raise SystemExit("invalid --lanes %d" % tuned["lanes"])
        if tuned["lanes32"]:
            s.set_lanes32(tuned["lanes32"])
        if mode:
            s.set_mlp(net, 1)
        s.set_state(*start)
        for _ in range(args.warmup):
            s.step_resident(step_settings(sc, mode, iterations, acceleration, precision))
        return s

    def timed(solver, step_fn, k, host_clock=False):
        """Device time (CUDA events on the solver's stream) of k steps, or with
        `host_clock` the host wall time of each blocking step call; the L2 flush
        between steps runs outside the timed interval either way."""
        stream = torch.cuda.ExternalStream(L.cc_solver_stream(solver.h))
        evs, metrics, wall = [], [], 0.0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            if host_clock:
                torch.cuda.synchronize()
                h0 = time.perf_counter()
                metrics.append(step_fn())
                wall += time.perf_counter() - h0
            else:
                metrics.append(step_fn())
            with torch.cuda.stream(stream):
                b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        if host_clock:
            return 1000.0 * wall, metrics
        return sum(a.elapsed_time(b) for a, b in evs), metrics

    def max_over_ranks(ms):
        if not dist:
            return ms
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    def leg(solver, step_fn, k, host_clock=False):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms, mets = timed(solver, step_fn, k, host_clock)
        if dist:
            dist.barrier()
        return max_over_ranks(ms), mets

    K = args.steps
    st_l, st_p = step_settings(sc, 1), step_settings(sc, 0)
    learned = make(1)
    tuned["lanes"] = int(L.cc_solver_get_lanes(learned.h))
    tuned["lanes32"] = int(L.cc_solver_get_lanes32(learned.h))
    plain = make(0)
    warm_state = learned.get_state()
    clocks = ClockSampler(local).__enter__()
    # ---- value: learned init at equal residual, device-resident; the colour
    # sweeps of every iteration stamp their span on the device clock (the roofline's
    # launch durations and the breakdown come from this same timed leg)
    L.cc_solver_set_profiling(learned.h, 1)
    t_l, mets_l = leg(learned, lambda: learned.step_resident(st_l), K)
    L.cc_solver_set_profiling(learned.h, 0)
    # ---- plain adaptive init at equal residual
    t_p, mets_p = leg(plain, lambda: plain.step_resident(st_p), K)
    # ---- the value leg's settings with every kernel launched directly (no CUDA
    # graphs) and without the per-iteration sweep stamps
    direct_solver = make(1)
    direct_solver.set_graphs(False)
    t_g, mets_g = leg(direct_solver, lambda: direct_solver.step_resident(st_l), K)
    # ---- the value leg's settings, CUDA graphs, without the sweep stamps or detection phase events
    quiet_solver = make(1)
    t_q, mets_q = leg(quiet_solver, lambda: quiet_solver.step_resident(st_l), K)
    # ---- both inits at the other sweep precision (same target and acceleration)
    other = 1 - SWEEP_PRECISION
    other_legs = {}
    for mode in (0, 1):
        so = step_settings(sc, mode, precision=other)
        solver_o = make(mode, precision=other)
        if mode == 1 and other == 1:
            tuned["lanes32"] = int(L.cc_solver_get_lanes32(solver_o.h))
        other_legs[mode] = leg(solver_o, lambda: solver_o.step_resident(so), K)
    # ---- both inits without acceleration (the reference's iteration)
    unacc = {}
    for mode in (0, 1):
        su = step_settings(sc, mode, acceleration=0.0)
        solver_u = make(mode, acceleration=0.0)
        unacc[mode] = leg(solver_u, lambda: solver_u.step_resident(su), K)
    # ---- end to end through cc_solver_step with host arrays in pinned memory
    # (learned): the caller's x and v go in and come back every step
    e2e_solver = make(1)
    x, v, t = e2e_solver.get_state()
    xh = torch.empty((sc.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    vh = torch.empty((sc.n, 3), dtype=torch.float64, pin_memory=True).numpy()
    xh[:], vh[:] = x, v
    state = {"t": t}

    def host_step():
        state["t"], m = e2e_solver.step_into(xh, vh, state["t"], st_l)
        return m

    t_e2e, mets_e2e = leg(e2e_solver, host_step, K, host_clock=True)
    # ---- the reference's fixed-iteration step (plain init, 30 iterations), for context
    st_f = step_settings(sc, 0, FIXED_ITERATIONS)
    st_f.residual_check_every = FIXED_ITERATIONS  # one residual evaluation, after the last iteration
    fixed = make(0, FIXED_ITERATIONS)
    t_f, mets_f = leg(fixed, lambda: fixed.step_resident(st_f), K)
    # ---- the reference's iteration budget (30) with the same residual target:
    # steps stop early once converged; both inits
    budget = {}
    for mode in (0, 1):
        sb = step_settings(sc, mode, acceleration=0.0)
        sb.iterations = FIXED_ITERATIONS
        solver_b = make(mode, FIXED_ITERATIONS)
        budget[mode] = leg(solver_b, lambda: solver_b.step_resident(sb), K)
    clocks.__exit__(None, None, None)

    value = world * K / (t_l / 1000.0)
    free = int((sc.mesh.pinned == 0).sum())

    def iters(mets):
        return [int(m["iterations"]) for m in mets]

    def summary(t_ms, mets):
        its = iters(mets)
        return {"steps_per_s": world * K / (t_ms / 1000.0), "ms_per_step": t_ms / K,
                "vertex_iters_per_s": world * free * sum(its) / (t_ms / 1000.0),
                "mean_iterations": float(np.mean(its)), "median_iterations": float(np.median(its)),
                "capped_fraction": float(np.mean(np.array(its) >= ITERATION_CAP)),
                "mean_final_relative_residual": float(np.mean([m["relative_residual"] for m in mets])),
                "max_final_relative_residual": float(np.max([m["relative_residual"] for m in mets])),
                "mean_final_relative_force_residual": float(np.mean([m["relative_force_residual"]
                                                                     for m in mets])),
                "max_final_relative_force_residual": float(np.max([m["relative_force_residual"]
                                                                   for m in mets]))}

    # ---- roofline of the dominant kernel (colour sweep), learned leg
    peak, peak_kind = load_peaks()
    static_b = static_bytes_per_sweep(sc)
    sweep_ms = sum(m["sweep_ms"] for m in mets_l)
    sweeps = sum(m["sweep_launches"] for m in mets_l)
    alg_bytes = sum((static_b + 28.0 * m["contact_incidence"]) * m["iterations"] for m in mets_l)
    achieved = alg_bytes / (sweep_ms / 1000.0) / 1e9 if sweep_ms > 0 else None
    det_ms = sum(m["detection_ms"] for m in mets_l) / K
    col_ms = sum(m["color_ms"] for m in mets_l) / K
    init_ms = sum(m["init_ms"] for m in mets_l) / K
    det_dev = {k: sum(m[k + "_ms"] for m in mets_l) / K for k in ("refit", "candidates", "narrow")}
    breakdown = {"detection": det_ms, "detection_device": det_dev, "coloring": col_ms, "learned_guess": init_ms,
                 "sweeps": sweep_ms / K,
                 "other": t_l / K - det_ms - col_ms - init_ms - sweep_ms / K,
                 "note": "from the timed learned leg: detection and colouring by host clock (they end in a "
                         "device sync), learned guess by CUDA events, sweeps by the sweep kernels' device-clock "
                         "stamps; detection_device = the "
                         "detection phases by CUDA events (refit and cache check, candidate rebuilds, narrow "
                         "phase with the canonical sort, incidence and radii); other = ms_per_step minus "
                         "detection, colouring, learned guess and sweeps (predict, warm start, residual "
                         "checks, acceleration, commit, metrics)"}

    # ---- batched uneven instances (config 2): 96 sheets, ~3.66M vertices, one
    # solver per rank over its share (longest-first partition), 20 iterations
    batched = None
    if not args.no_batched:
        batched = batched_leg(rank, world, leg, L)
    garment = None
    if not args.no_garment:
        garment = garment_leg(rank, world, leg, L)
    crumple = None
    if not args.no_crumple:
        crumple = crumple_leg(rank, world, max_over_ranks)

    # ---- CPU baseline (rank 0, N=1 only): the oracle at equal residual from
    # the state the timed legs start from, a sample of about 30 s
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        done, dt, (its_cpu, _), _ = cpu_reference_run(sc, warm_state, 8, 30.0, threads)
        cpu = {"value": done / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": "%d step(s) from the state after the warm-up at equal residual (iterations %s, about "
                         "30 s), FP64 oracle restatement of the reference CPU path, %d threads" % (
                             done, its_cpu, threads)}

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
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": t_l / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": config_dict(sc, world),
        "learned": summary(t_l, mets_l),
        "plain": summary(t_p, mets_p),
        "learned_vs_plain_time_ratio": t_p / t_l,
        "learned_init_used_fraction": float(np.mean([m["init_used"] for m in mets_l])),
        "acceleration": ACCELERATION,
        "launch_forms": {
            "graphs_with_sweep_stamps": {"steps_per_s": world * K / (t_l / 1000.0), "ms_per_step": t_l / K},
            "graphs": {"steps_per_s": world * K / (t_q / 1000.0), "ms_per_step": t_q / K},
            "direct_launches": {"steps_per_s": world * K / (t_g / 1000.0), "ms_per_step": t_g / K},
            "note": "the value leg (iteration chunks launched as CUDA graphs, the sweep kernels stamping "
                    "their per-iteration span on the device clock, detection phases timed by CUDA events) "
                    "against the same steps without any timing, and with every kernel launched directly; "
                    "identical iterates"},
        "sweep_precision": ("fp32 element assembly" if SWEEP_PRECISION else "fp64"),
        "other_precision": {"sweep_precision": ("fp32 element assembly" if other else "fp64"),
                            "learned": summary(*other_legs[1]), "plain": summary(*other_legs[0]),
                            "learned_vs_plain_time_ratio": other_legs[0][0] / other_legs[1][0],
                            "lanes32": tuned["lanes32"]},
        "unaccelerated": {"learned": summary(*unacc[1]), "plain": summary(*unacc[0]),
                          "learned_vs_plain_time_ratio": unacc[0][0] / unacc[1][0],
                          "note": "same residual target, Chebyshev acceleration off (the reference's iteration)"},
        "fixed_iterations": {"iterations": FIXED_ITERATIONS, "steps_per_s": world * K / (t_f / 1000.0),
                             "ms_per_step": t_f / K,
                             "mean_final_relative_residual": float(np.mean([m["relative_residual"]
                                                                            for m in mets_f]))},
        "budget_30_iterations": {"learned": summary(*budget[1]), "plain": summary(*budget[0]),
                                 "note": "same residual target, at most 30 iterations (the reference's count)"},
        "vertex_iters_per_s": world * free * sum(iters(mets_l)) / (t_l / 1000.0),
        "roofline": {
            "kernel": "k_sweep (colour sweep)",
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "traffic": SWEEP_TRAFFIC_BYTES,
            "traffic_note": "dram read+write bytes per k_sweep launch, one ncu capture on the fold (cold cache)",
            "peak_kind": peak_kind,
            "sweep_launches": int(sweeps),
            "avg_launch_us": 1000.0 * sweep_ms / max(sweeps, 1),
            "launch_timing": "each iteration's back-to-back colour sweeps timed in the timed learned leg by "
                             "their own device-clock stamps (first colour's earliest block start to the last "
                             "colour's latest block end), summed and divided by the launches",
            "algorithmic_bytes_per_launch": alg_bytes / max(sweeps, 1),
            "sweep_share_of_step": sweep_ms / t_l,
        },
        "cpu_baseline": cpu,
        "e2e": {"value": world * K / (t_e2e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": 2 * sc.n * 24,
                "d2h_bytes_per_step": 2 * sc.n * 24, "mean_iterations": float(np.mean(iters(mets_e2e))),
                "timing": "host clock around each blocking VbdSolver.step_into call",
                "host_memory": "pinned, [n][3] float64 x and v, stepped in place (VbdSolver.step_into)"},
        "gpu_launches": int(sum(m["kernel_launches"] for m in mets_l)),
        "lanes_per_vertex": int(L.cc_solver_get_lanes(learned.h)) & 0xff,
        "blocks_per_sm_cap": (int(L.cc_solver_get_lanes(learned.h)) >> 8) & 0xff,
        "sweep_variant": {"encoded": int(L.cc_solver_get_lanes(learned.h)),
                          "persistent_grid": bool(int(L.cc_solver_get_lanes(learned.h)) & (1 << 16)),
                          "block_threads": {0: 128, 1: 64, 2: 256}[(int(L.cc_solver_get_lanes(learned.h)) >> 17) & 3]},
        "breakdown_ms_per_step": breakdown,
        "clocks": clocks.summary(),
        "detections_per_step": sum(m["detection_updates"] for m in mets_l) / K,
        "contact_terms_last": mets_l[-1]["contact_terms"] if mets_l else None,
        "batched": batched,
        "garment": garment,
        "crumple": crumple,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
