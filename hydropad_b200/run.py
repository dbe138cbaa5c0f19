"""Command-line runner: advance one box of a benchmark configuration.

    python -m hydropad_b200.run --case eds --n 256 --steps 10 --precision mixed
    python -m hydropad_b200.run --case sod --n 64 --steps 100 --precision fp64 --tiles 4,4,4
    python -m hydropad_b200.run --case eds --n 256 --precision fp64 --sweep-times 4,6,10,11,12,13

Mirrors the reference's main program for the hydro part (main.F90:100-121:
the time loop over evolve_sys) on synthetic initial conditions, and prints
one JSON line with the step count, simulated time, wall time and
cell-updates/s.  Used for profiling single configurations.

``--sweep-times``: instead of the time loop, the duration of single sweeps
along x, y and z for each listed tile (CUDA events on the library's stream
around three sweeps through the drop-in entry point, after one warm-up
sweep per axis; the state advances with every sweep).
"""
from __future__ import annotations

import argparse
import json
import time

from . import ics
from .api import Hydro
from .params import HydroParams


def sweep_times(h, tiles, reps=3):
    """{tile: [x, y, z] ms per sweep} on the attached box."""
    import torch
    st = torch.cuda.ExternalStream(h.stream_handle())
    out = {}
    for tile in tiles:
        h.set_tiles(tile, tile, tile)
        row = []
        for nd in (1, 2, 3):
            h.ppmsolver(nd)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            for _ in range(reps):
                h.ppmsolver(nd)
            e1.record(st)
            torch.cuda.synchronize()
            row.append(e0.elapsed_time(e1) / reps)
        out[tile] = row
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["sod", "eds"], default="eds")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--tiles", default="", help="tile per axis 'x,y,z' (default: autotune)")
    ap.add_argument("--sweep-times", default="", help="tiles 'a,b,...' to time single sweeps of (no time loop)")
    ap.add_argument("--no-graph", action="store_true")
    args = ap.parse_args(argv)

    n = args.n
    if args.case == "sod":
        state = ics.sod(n, axis=0)
        prm = HydroParams(shape=(n, n, n), cour=0.8)
    else:
        state = ics.grf_eds(n, seed=args.seed)
        prm = HydroParams(shape=(n, n, n), cosmo=True, tstop=(1.0 + 10.0) ** (-1.5))
    with Hydro(prm, precision=args.precision) as h:
        h.attach_state(*state)
        if args.sweep_times:
            h.start_with_cfl()
            tiles = [int(t) for t in args.sweep_times.split(",")]
            res = sweep_times(h, tiles)
            print(json.dumps({"case": args.case, "n": n, "precision": args.precision,
                              "sweep_ms_xyz": {str(t): v for t, v in res.items()}}))
            return
        if args.tiles:
            h.set_tiles(*[int(t) for t in args.tiles.split(",")])
        else:
            h.autotune(reps=1)
        h.start_with_cfl()
        t0 = time.perf_counter()
        h.evolve(args.steps, graph=not args.no_graph)
        el = time.perf_counter() - t0
        s = h.get_scalars()
        print(json.dumps({"case": args.case, "n": n, "precision": args.precision, "steps": args.steps,
                          "tiles": h.get_tiles(), "t": s.t, "dt": s.dt, "wall_s": el,
                          "cell_updates_per_s": args.steps * n ** 3 / el}))


if __name__ == "__main__":
    main()
