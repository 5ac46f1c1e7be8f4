"""Sharding of batched instances across ranks (CPU, gloo, world size 2): the
shards cover every instance exactly once, their vertex loads are balanced to
within the largest instance, and the per-rank summaries gather on every rank.
The solver is a stand-in here: no GPU is used."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from clothcraft_b200 import batch, scenes


class FakeSolver:
    def __init__(self, instances):
        self.n = sum(sc.n for sc in instances)

    def step_resident(self, settings):
        return {"iterations": 3}


def small_instances():
    return scenes.config2_instances(seed=7, count=9, sides=(8, 20), pitch=1.0)


def test_partition_balances_vertex_counts():
    sizes = [sc.n for sc in scenes.config2_instances(seed=2, count=96)]
    for parts in (1, 2, 4, 8):
        bins = scenes.partition_instances(sizes, parts)
        assert sorted(i for b in bins for i in b) == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in b) for b in bins]
        assert max(loads) - min(loads) <= max(sizes)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        inst = small_instances()

        def gather(obj):
            res = [None] * world
            dist.all_gather_object(res, obj)
            return res

        res = batch.run(inst, rank, world, 2, None, solver_factory=FakeSolver, gather=gather)
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_two_ranks_cover_every_instance_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    inst = small_instances()
    for rank in (0, 1):
        res = got[rank]
        assert [r["rank"] for r in res] == [0, 1]
        covered = sorted(i for r in res for i in r["instances"])
        assert covered == list(range(len(inst)))
        assert sum(r["vertices"] for r in res) == sum(sc.n for sc in inst)
        assert all(r["vertex_iters"] == r["vertices"] * 3 * 2 for r in res)
