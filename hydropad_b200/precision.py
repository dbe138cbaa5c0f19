"""The precision comparison: mixed against FP64, per configuration.

    python -m hydropad_b200.precision --n 512 --steps 100            # config 3, 512^3
    python -m hydropad_b200.precision --n 1024 --steps 100 --mixed-only
    python -m hydropad_b200.precision --case sod --n 64 --steps 100  # config 1
    python -m hydropad_b200.precision --n 256 --to-z10               # config 2
    python -m hydropad_b200.precision --case ensemble                # config 4

Workloads: ``--case eds`` (default) is the EdS recipe (seeded Gaussian random
field, k_c = N/8, rms 0.5, T = 100 K, a = 1/51) at side ``--n``, initial
conditions generated on the GPU; ``--case sod`` the plane-parallel Sod
shock along x of the 64^3 configuration; ``--case ensemble`` the 64 boxes of
the ensemble configuration (sides 32..128, spectral index in [-2.5, -1.5],
50 steps each), every box compared on its own and the norms pooled over the
boxes.  With both precisions, three runs start from the same initial state:

* FP64 (free running) -- the reference of the comparison (the FP64 path
  equals the CPU oracle to <= 1e-10 relative L1 on the parity cases);
* mixed with the FP64 run's time scalars replayed every step (the FP64 dt
  sequence), so that the difference is the precision alone;
* mixed, free running (its own dt from its own CFL).

Reports L1 (relative) and L_inf (relative to max |reference|) of rho, the
momentum components rho*v and the total energy density
E = p/(gamma-1) + rho|v|^2/2 after ``--steps`` steps (``--to-z10``: until the
FP64 run reaches z = 10), the final time and dt of each run, and the
throughput of each precision (CUDA events over ``--time-steps``
graph-replayed steps).  ``--mixed-only`` (1024^3: the FP64 state is 43 GB)
runs the free-running mixed box alone.  One JSON line.
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


def _sums(test, ref):
    """Per derived field: sum |test - ref|, sum |ref|, max |test - ref|, max |ref|."""
    out = {}
    a, b = _derived(test), _derived(ref)
    for k in a:
        d = np.abs(a[k] - b[k])
        out[k] = (float(d.sum()), float(np.abs(b[k]).sum()), float(d.max()), float(np.abs(b[k]).max()))
    return out


def _norms_from_sums(s):
    """Relative norms; a field that is zero everywhere in the reference (the
    transverse momenta of a plane Sod shock) gets the absolute ones."""
    out = {}
    for k, v in s.items():
        if v[1] > 0.0:
            out[k] = {"l1": v[0] / v[1], "linf": v[2] / v[3]}
        else:
            out[k] = {"l1_abs": v[0], "linf_abs": v[2], "reference": "zero everywhere"}
    return out


def _norms(test, ref):
    return _norms_from_sums(_sums(test, ref))


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


def _compare(make, steps, to_tstop):
    """Run FP64, mixed with the FP64 dt replayed, and free mixed from one
    initial state; returns (fp64 box, replayed, free, steps run)."""
    ref, rep, free = make(["fp64", "mixed", "mixed"])
    tstop = ref.params.tstop
    done = 0
    while True:
        if to_tstop:
            if not ref.get_scalars().told < tstop or done >= 10000:
                break
        elif done >= steps:
            break
        rep.set_scalars(ref.get_scalars())
        ref.evolve(1, graph=True)
        rep.evolve(1, graph=True)
        done += 1
    free.evolve(done, graph=True)
    return ref, rep, free, done


def _ensemble(args):
    """Configuration 4: every box of the ensemble compared on its own (a box
    in a batch is bitwise the box alone), norms pooled over the boxes."""
    import torch

    from .ensemble import ensemble_specs
    from .api import Hydro
    specs = ensemble_specs(args.boxes, args.ensemble_seed)
    pooled = {"replayed": {}, "free": {}}
    for side, seed, sidx in specs:
        prm = HydroParams(shape=(side, side, side), cosmo=True, tstop=(1.0 + 10.0) ** (-1.5))
        ic = ics.grf_eds_device(side, seed=seed, spectral_index=sidx)

        def make(precisions):
            hs = []
            for p in precisions:
                h = Hydro(prm, precision=p)
                h.attach_device(*ic)
                h.start_with_cfl()
                hs.append(h)
            return hs

        ref, rep, free, _ = _compare(make, args.ensemble_steps, False)
        fr = ref.download(nbound=0)
        for name, h in (("replayed", rep), ("free", free)):
            for k, v in _sums(h.download(nbound=0), fr).items():
                acc = pooled[name].setdefault(k, [0.0, 0.0, 0.0, 0.0])
                acc[0] += v[0]
                acc[1] += v[1]
                acc[2] = max(acc[2], v[2])
                acc[3] = max(acc[3], v[3])
        for h in (ref, rep, free):
            h.close()
        del ic
        torch.cuda.empty_cache()
    return {"workload": f"ensemble of {args.boxes} EdS boxes (sides {sorted({s for s, _, _ in specs})}, "
                        f"spectral index in [-2.5, -1.5], seed {args.ensemble_seed}), {args.ensemble_steps} steps each",
            "boxes": args.boxes, "steps": args.ensemble_steps,
            "cells": int(sum(s ** 3 for s, _, _ in specs)),
            "mixed_replayed_dt_vs_fp64": _norms_from_sums(pooled["replayed"]),
            "mixed_free_vs_fp64": _norms_from_sums(pooled["free"])}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="eds", choices=["eds", "sod", "ensemble"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--to-z10", action="store_true", help="run until the FP64 box reaches z = 10")
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--time-steps", type=int, default=10)
    ap.add_argument("--mixed-only", action="store_true")
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--ensemble-steps", type=int, default=50)
    ap.add_argument("--ensemble-seed", type=int, default=4)
    args = ap.parse_args(argv)

    import torch

    from .api import Hydro

    if args.case == "ensemble":
        print(json.dumps(_ensemble(args)))
        return

    n = args.n
    if args.case == "sod":
        prm = HydroParams(shape=(n, n, n), cosmo=False)
        ic_host = ics.sod(n, axis=0)
        ic = None
        out = {"workload": f"{n}^3 Sod shock along x (static, cour 0.8)", "n": n, "cells": n ** 3}
    else:
        # config 2 stops at z = 10; the 100-step runs of config 3 go past it
        tstop = (1.0 + 10.0) ** (-1.5) if args.to_z10 else 1.0e4
        prm = HydroParams(shape=(n, n, n), cosmo=True, tstop=tstop)
        ic = ics.grf_eds_device(n, seed=args.seed)
        ic_host = None
        torch.cuda.synchronize()
        torch.cuda.empty_cache()  # the generator's temporaries go back to the driver
        out = {"workload": f"{n}^3 EdS GRF (seed {args.seed})", "n": n, "cells": n ** 3}

    def make(precisions):
        # attach every box, free the initial conditions, then tune (the
        # autotuner's scratch copy needs the room at 1024^3)
        nonlocal ic
        hs = []
        for precision in precisions:
            h = Hydro(prm, precision=precision)
            if ic_host is not None:
                h.attach_state(*ic_host)
            else:
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
        out["steps"] = args.steps
        out["mixed"] = {"t": s.t, "dt": s.dt, "nstep": s.nstep, "a": s.t ** (2.0 / 3.0), "tiles": h.get_tiles(),
                        "ms_per_step": ms / args.time_steps,
                        "cell_updates_per_s": n ** 3 * args.time_steps / (ms * 1e-3)}
        h.close()
        print(json.dumps(out))
        return

    ref, rep, free, done = _compare(make, args.steps, args.to_z10)
    out["steps"] = done
    sr, sf = ref.get_scalars(), free.get_scalars()
    fr = ref.download(nbound=0)
    out["mixed_replayed_dt_vs_fp64"] = _norms(rep.download(nbound=0), fr)
    out["mixed_free_vs_fp64"] = _norms(free.download(nbound=0), fr)
    del fr
    out["fp64_final"] = {"t": sr.t, "dt": sr.dt, "a": sr.t ** (2.0 / 3.0)}
    out["mixed_free_final"] = {"t": sf.t, "dt": sf.dt, "a": sf.t ** (2.0 / 3.0)}
    if not args.to_z10:  # a box at tstop no longer advances: time only open-ended runs
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
