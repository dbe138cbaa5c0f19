"""Boxes across ranks: the static (ensemble) and trace (serving) splits, and
the sharded serving flow on two gloo ranks on the CPU (each rank schedules
its share against the CPU engine model; one host gather at the end)."""
import os
import socket
import tempfile

import torch.multiprocessing as mp

from hydropad_b200.serve import Scheduler, box_bytes, merge_stats, poisson_trace
from hydropad_b200.shard import assign_lpt, gather_objects, shard_trace


def test_assign_lpt_balances_and_covers():
    work = [s ** 3 for s in (32, 48, 64, 96, 128) * 13][:64]
    for world in (1, 2, 3, 8):
        parts = assign_lpt(work, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in p) for p in parts]
        # LPT bound: no rank exceeds the mean by more than the largest item
        assert max(loads) - sum(loads) / world <= max(work)
    assert assign_lpt(work, 1) == [list(range(len(work)))]


def test_shard_trace_is_a_partition():
    tr = poisson_trace(300, seed=3)
    parts = shard_trace(tr, 4)
    assert sorted(r.rid for p in parts for r in p) == list(range(300))
    loads = [sum(r.cells * r.steps for r in p) for p in parts]
    assert max(loads) - min(loads) <= max(r.cells * r.steps for r in tr)
    assert shard_trace(tr, 4)[2] == parts[2]  # every rank computes the same split


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _serve_rank(rank, world, port, out_path):
    import torch.distributed as dist

    from tests.serve_model import ModelEngine
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tr = poisson_trace(40, rate=500.0, seed=11, side_min=32, side_max=96, step_min=5, step_max=30)
        mine = shard_trace(tr, world)[rank]
        st = Scheduler(ModelEngine(), budget_bytes=4 * box_bytes(96), capacity=8, chunk=4).run(mine)
        merged = merge_stats(gather_objects(st))
        if rank == 0:
            with open(out_path, "w") as f:
                f.write(",".join(str(c.rid) for c in merged.completed) + "\n")
                f.write(f"{merged.summary()['cell_updates']}\n")
    finally:
        dist.destroy_process_group()


def test_sharded_serving_two_gloo_ranks():
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "merged.txt")
        mp.start_processes(_serve_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        rids, work = open(out).read().split("\n")[:2]
    tr = poisson_trace(40, rate=500.0, seed=11, side_min=32, side_max=96, step_min=5, step_max=30)
    assert [int(x) for x in rids.split(",")] == list(range(40))
    assert int(work) == sum(r.cells * r.steps for r in tr)


def test_gather_objects_single_process():
    assert gather_objects({"a": 1}) == [{"a": 1}]
