"""Large boxes and the precision comparison.

    python -m hydropad_b200.precision --n 512 --steps 100
    python -m hydropad_b200.precision --n 1024 --steps 100 --mixed-only

Workload: the 256^3 EdS recipe (seeded Gaussian random field, k_c = N/8,
rms 0.5, T = 100 K, a = 1/51) at side ``--n``, initial conditions generated
on the GPU.  With both precisions, three boxes run from the same initial
state:

* FP64 (free running) -- the reference of the comparison (the FP64 path
  equals the CPU oracle to <= 1e-10 relative L1 on the parity cases);
* mixed with the FP64 run's time scalars replayed every step (the FP64 dt
  sequence), so that the difference is the precision alone;
* mixed, free running (its own dt from its own CFL).

Reports L1 (relative) and L_inf (relative to max |reference|) of rho, the
momentum components rho*v and the total energy density
E = p/(gamma-1) + rho|v|^2/2 after ``--steps`` steps, the final time and dt
of each run, and the throughput of each precision (CUDA events over
``--time-steps`` graph-replayed steps).  ``--mixed-only`` (1024^3: the FP64
state is 43 GB) runs the free-running mixed box alone.  One JSON line.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import ics
from .params import HydroParams

GAMMA = 5.0 / 3.0


def _derived(f):
    p, rho, vx, vy, vz = f
    e = p / (GAMMA - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return {"rho": rho, "rho_vx": rho * vx, "rho_vy": rho * vy, "rho_vz": rho * vz, "E": e}


def _norms(test, ref):
    out = {}
    a, b = _derived(test), _derived(ref)
    for k in a:
        d = np.abs(a[k] - b[k])
        out[k] = {"l1": float(d.sum() / np.abs(b[k]).sum()), "linf": float(d.max() / np.abs(b[k]).max())}
    return out


def _time_steps(h, steps):
    import torch
    st = torch.cuda.ExternalStream(h.stream_handle())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    h.evolve_async(steps, graph=True)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--time-steps", type=int, default=10)
    ap.add_argument("--mixed-only", action="store_true")
    args = ap.parse_args(argv)

    import torch

    from .api import Hydro
    n = args.n
    prm = HydroParams(shape=(n, n, n), cosmo=True, tstop=1.0e4)
    ic = ics.grf_eds_device(n, seed=args.seed)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the generator's temporaries go back to the driver
    out = {"workload": f"{n}^3 EdS GRF (seed {args.seed})", "n": n, "steps": args.steps, "cells": n ** 3}

    def make(precisions):
        # attach every box, free the initial conditions, then tune (the
        # autotuner's scratch copy needs the room at 1024^3)
        nonlocal ic
        hs = []
        for precision in precisions:
            h = Hydro(prm, precision=precision)
            h.attach_device(*ic)
            hs.append(h)
        ic = None
        torch.cuda.empty_cache()
        for h in hs:
            h.autotune(reps=1)
            h.start_with_cfl()
        return hs

    if args.mixed_only:
        (h,) = make(["mixed"])
        h.evolve(args.steps, graph=True)
        s = h.get_scalars()
        ms = _time_steps(h, args.time_steps)
        out["mixed"] = {"t": s.t, "dt": s.dt, "nstep": s.nstep, "tiles": h.get_tiles(),
                        "ms_per_step": ms / args.time_steps,
                        "cell_updates_per_s": n ** 3 * args.time_steps / (ms * 1e-3)}
        h.close()
        print(json.dumps(out))
        return

    ref, rep, free = make(["fp64", "mixed", "mixed"])
    for _ in range(args.steps):
        rep.set_scalars(ref.get_scalars())
        ref.evolve(1, graph=True)
        rep.evolve(1, graph=True)
    free.evolve(args.steps, graph=True)
    sr, sf = ref.get_scalars(), free.get_scalars()
    fr = ref.download(nbound=0)
    out["mixed_replayed_dt_vs_fp64"] = _norms(rep.download(nbound=0), fr)
    out["mixed_free_vs_fp64"] = _norms(free.download(nbound=0), fr)
    del fr
    out["fp64_final"] = {"t": sr.t, "dt": sr.dt, "a": sr.t ** (2.0 / 3.0)}
    out["mixed_free_final"] = {"t": sf.t, "dt": sf.dt, "a": sf.t ** (2.0 / 3.0)}
    for name, h in (("fp64", ref), ("mixed", free)):
        ms = _time_steps(h, args.time_steps)
        out[name] = {"tiles": h.get_tiles(), "ms_per_step": ms / args.time_steps,
                     "cell_updates_per_s": n ** 3 * args.time_steps / (ms * 1e-3)}
    out["mixed_over_fp64"] = out["mixed"]["cell_updates_per_s"] / out["fp64"]["cell_updates_per_s"]
    for h in (ref, rep, free):
        h.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
