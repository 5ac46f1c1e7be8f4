"""Batched instances across GPUs: one process per GPU, instances partitioned
by vertex count (greedy longest-first bin packing), each rank stepping its
share as one batched solver (cc_batch_create). Instances are independent, so
the step has no collective; per-step metrics are gathered on the host after
the timed steps (torch.distributed over NCCL or gloo), off the data path.

  python -m torch.distributed.run --nproc-per-node N -m clothcraft_b200.batch [--steps K]
"""
from __future__ import annotations

import argparse
import json
import os
import time

from . import scenes


def shard(instances, rank: int, world: int) -> list:
    """Indices of the instances this rank steps."""
    return scenes.partition_instances([sc.n for sc in instances], world)[rank]


def run(instances, rank: int, world: int, steps: int, settings, solver_factory=None, sync=None, gather=None):
    """Step this rank's share `steps` times; returns the gathered per-rank
    summaries (rank 0) or this rank's summary. `solver_factory(scenes)` builds
    the batched solver (default: VbdSolver.batch), `sync()` waits for the
    device, `gather(obj)` returns the list of every rank's object."""
    if solver_factory is None:
        from .vbd import VbdSolver

        solver_factory = VbdSolver.batch
    mine = shard(instances, rank, world)
    solver = solver_factory([instances[i] for i in mine])
    vertices = sum(instances[i].n for i in mine)
    if sync:
        sync()
    t0 = time.perf_counter()
    iters = 0
    for _ in range(steps):
        m = solver.step_resident(settings)
        iters += int(m["iterations"])
    if sync:
        sync()
    seconds = time.perf_counter() - t0
    mine_summary = {"rank": rank, "instances": mine, "vertices": vertices, "steps": steps, "seconds": seconds,
                    "vertex_iters": vertices * iters}
    return gather(mine_summary) if gather else [mine_summary]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--count", type=int, default=96)
    args = ap.parse_args(argv)
    import datetime

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    from . import native

    native.load().cc_set_device(local)
    instances = scenes.config2_instances(count=args.count)
    st = instances[0].settings.to_c()

    def gather(obj):
        if world == 1:
            return [obj]
        out = [None] * world
        dist.all_gather_object(out, obj)
        return out

    res = run(instances, rank, world, args.steps, st, sync=torch.cuda.synchronize, gather=gather)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        slowest = max(r["seconds"] for r in res)
        print(json.dumps({"instances": len(instances), "vertices": sum(r["vertices"] for r in res),
                          "steps_per_s": args.steps / slowest,
                          "vertex_iters_per_s": sum(r["vertex_iters"] for r in res) / slowest,
                          "per_rank": [{k: r[k] for k in ("rank", "vertices", "seconds")} for r in res]}))


if __name__ == "__main__":
    main()
