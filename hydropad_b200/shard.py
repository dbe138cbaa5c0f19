"""Boxes across GPUs: one process per GPU, no data-path collective.

Ensemble members and serving requests are independent boxes, so each rank
advances its own share and the only communication is a host-side gather of
results and metrics at the end (the reference's MPI decomposition splits one
box into blocks instead, hydropad/init_sys.F90:53-60; a box here never
spans GPUs).

* :func:`assign_lpt` -- static split of an ensemble: largest box first, each
  to the rank with the least work so far (longest-processing-time greedy).
* :func:`shard_trace` -- split of a serving trace decided from the trace
  alone (arrival order, work = cells x steps), so every rank computes the
  same assignment without talking to the others.
* :func:`gather_objects` -- host gather of per-rank Python objects on a
  CPU (gloo) group, also under an NCCL job.
"""
from __future__ import annotations

import heapq


def assign_lpt(work, world: int):
    """Indices of ``work`` per rank, balancing the summed work (LPT greedy;
    ties go to the lower rank; within a rank indices stay ascending)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda i: (-work[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(ix) for ix in out]


def shard_trace(trace, world: int):
    """Requests per rank: in arrival order, each request goes to the rank
    whose assigned work (cells x steps) is smallest, ties to the lower rank."""
    load = [0] * world
    out = [[] for _ in range(world)]
    for req in sorted(trace, key=lambda r: (r.arrival, r.rid)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(req)
        load[r] += req.cells * req.steps
    return out


def gather_objects(obj, group=None):
    """All ranks' ``obj`` in rank order, on every rank (one host gather)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out
