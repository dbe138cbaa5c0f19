"""Ensemble runner: many independent cosmological boxes in one batch.

    python -m hydropad_b200.ensemble --boxes 64 --steps 50 --precision mixed

Workload: ``--boxes`` Einstein-de Sitter Gaussian random fields, sides drawn
from {32, 48, 64, 96, 128}, spectral index n uniform in [-2.5, -1.5], one
seed per box (all from ``--seed``), started together at a = 1/51 and
advanced ``--steps`` evolve_sys steps each.  The batch is autotuned, then
timed with CUDA events on its stream; ``--alone`` also times the same boxes
advanced one after another through hp_evolve (the one-box-per-run layout of
the reference's main program, hydropad/main.F90:100-121).  Prints one JSON
line (aggregate cell-updates/s).

Under torchrun (one process per GPU) the boxes are split across the ranks by
:func:`hydropad_b200.shard.assign_lpt` (cells per box); each rank times its
own batch on its device and the job's time is the maximum over the ranks.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import ics
from .params import HydroParams

SIDES = (32, 48, 64, 96, 128)


def ensemble_specs(nboxes: int, seed: int):
    """(side, seed, spectral index) of each box: box i has seed i; sides and
    spectral indices are drawn from ``seed``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sides = rng.choice(SIDES, size=nboxes)
    idx = rng.uniform(-2.5, -1.5, size=nboxes)
    return [(int(s), i, float(n)) for i, (s, n) in enumerate(zip(sides, idx))]


def make_box(side: int, seed: int, spectral_index: float, precision: str, tiles=None, device: int = 0):
    from .api import Hydro
    prm = HydroParams(shape=(side, side, side), cosmo=True, tstop=(1.0 + 10.0) ** (-1.5))
    h = Hydro(prm, precision=precision, device=device)
    h.attach_device(*ics.grf_eds_device(side, seed=seed, spectral_index=spectral_index, device=f"cuda:{device}"))
    if tiles is not None:
        h.set_tiles(*tiles)
    h.start_with_cfl()
    return h


def _event_ms(stream_handle: int, fn):
    import torch
    st = torch.cuda.ExternalStream(stream_handle)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ensemble(boxes: int = 64, steps: int = 50, warmup: int = 3, precision: str = "mixed", seed: int = 4,
                 graph: bool = True, world: int = 1, rank: int = 0, device: int = 0) -> dict:
    """This rank's share of the ensemble (LPT split by cells), autotuned and
    timed with CUDA events on the batch's stream.  Returns the rank's
    figures; the caller takes the maximum time over the ranks."""
    from .batch import Batch
    from .shard import assign_lpt, gather_objects
    specs = ensemble_specs(boxes, seed)
    mine = [specs[i] for i in assign_lpt([s ** 3 for s, _, _ in specs], world)[rank]]
    t0 = time.perf_counter()
    hs = [make_box(s, sd, n, precision, device=device) for s, sd, n in mine]
    t_ic = time.perf_counter() - t0
    with Batch(precision, capacity=max(1, len(mine)), device=device) as b:
        for h in hs:
            b.add(h)
        tiles = b.autotune(reps=1)
        b.step(warmup, graph=graph)
        b.synchronize()
        gather_objects(None)  # barrier
        l0 = b.launch_count()
        ms = _event_ms(b.stream_handle(), lambda: b.step(steps, graph=graph))
        b.synchronize()
        launches = b.launch_count() - l0
        for h in list(b.members):
            b.remove(h)
    for h in hs:
        h.close()
    return {"ms": ms, "cells": sum(s ** 3 for s, _, _ in mine), "boxes": len(mine), "tiles": list(tiles),
            "launches": launches, "ic_seconds": t_ic, "total_cells": sum(s ** 3 for s, _, _ in specs),
            "sides": sorted(set(s for s, _, _ in specs))}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--alone", action="store_true", help="also time the boxes one after another")
    args = ap.parse_args(argv)

    import os

    import torch

    from .shard import gather_objects
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(dev)
    mine = run_ensemble(args.boxes, args.steps, args.warmup, args.precision, args.seed, not args.no_graph,
                        world, rank, dev)
    per_rank = gather_objects(mine)
    ms = max(r["ms"] for r in per_rank)
    cells = mine["total_cells"]
    tiles = mine["tiles"]
    out = {"workload": "ensemble", "boxes": args.boxes, "sides": mine["sides"], "cells": cells,
           "steps": args.steps, "warmup": args.warmup, "precision": args.precision, "graph": not args.no_graph,
           "n_gpus": world, "tiles": tiles, "batch_ms": round(ms, 3), "batch_ms_per_step": round(ms / args.steps, 4),
           "batch_cell_updates_per_s": cells * args.steps / (ms * 1e-3),
           "launches_per_step": per_rank[0]["launches"] / args.steps}
    if world > 1:
        out["per_rank"] = per_rank
    if args.alone and world == 1:
        specs = ensemble_specs(args.boxes, args.seed)
        boxes = [make_box(s, sd, n, args.precision, tiles=tiles) for s, sd, n in specs]
        for h in boxes:
            h.evolve(args.warmup, graph=not args.no_graph)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for h in boxes:
            h.evolve_async(args.steps, graph=not args.no_graph)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        out["alone_ms"] = round(ms, 3)
        out["alone_cell_updates_per_s"] = cells * args.steps / (ms * 1e-3)
        out["batch_speedup"] = out["batch_cell_updates_per_s"] / out["alone_cell_updates_per_s"]
        for h in boxes:
            h.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
