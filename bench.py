#!/usr/bin/env python
"""Benchmark of the PPM hydro step (cell-updates/s) -- one JSON line.

Workload: the single large box of the precision configuration, 512^3 cells,
Einstein-de Sitter background from z=50 (a = 1/51), seeded Gaussian random
baryon field (rms delta 0.5, P(k) ~ k^-2 exp(-(k/k_c)^2), k_c = N/8), linear
velocities, T = 100 K, gamma = 5/3.  One step = one evolve_sys hydro step:
three fused directional sweeps, expand, CFL reduction and timedet, all on
the device.  Both precisions run the same initial state for 100 steps (the
steps before the timed window are untimed); the headline value is the
mixed-precision path over the timed window, the FP64 path is measured
beside it, and the L1 / L_inf errors of density, momentum and total energy
of the mixed state against the FP64 state after the 100 steps are reported
(the metric's density rel-L1 <= 1e-5 gate).  100 steps run past z = 10
(about 77 steps with the 2 % expansion limit), so the end time is open.
Beside the headline: the batched ensemble (64 boxes of 32^3..128^3, mixed,
50 steps, one persistent launch per sweep axis, CUDA graphs) and a bounded
serving trace (the first 256 Poisson arrivals at 200/s, sides 32..256,
50..500 steps; p50/p99 latency from arrival to result on the host,
aggregate cell-updates/s), mixed and FP64.

    python bench.py [--steps K] [--warmup W] [--n 512]
    python bench.py --gpus N          # N ranks (re-launched under torchrun)
    python bench.py --impl reference  # CPU oracle on the host cores
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PPM cell-updates/s, mixed vs FP64 GPU at density rel-L1≤1e-5; p50/p99 latency"
UNIT = "cell-updates/s"
BASE_SEED = 12345
BYTES_PER_CELL_SWEEP = 80  # 5 FP64 fields read + written once per sweep
COMPARE_STEPS = 100        # steps after which mixed is compared with FP64
TSTOP = 1.0e4              # open end time: 100 steps run past z = 10
REF_SLAB = 32              # planes of the reference arm's per-step sample


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-threads", type=int, default=0)
    ap.add_argument("--serve-requests", type=int, default=256,
                    help="requests of the serving trace (0: skip the serving and ensemble runs)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def relaunch_under_torchrun(n):
    """--gpus N without a torchrun environment: start N ranks of this same
    command under torch.distributed.run (one process per GPU)."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    os.execv(sys.executable, cmd)


def workload_config(n, world, precision):
    return {
        "workload": f"{n}^3 EdS cosmological box (z=50 start, GRF rms 0.5, k_c=N/8, T=100K, gamma 5/3), "
                    f"{COMPARE_STEPS} steps compared, one box per GPU",
        "grid": n,
        "global_cells": n ** 3 * world,
        "precision": precision,
        "ic_seed": f"{BASE_SEED}+rank",
        "l2_policy": f"state {5 * 8 * n ** 3 / 1e6:.0f} MB per box > 126 MB L2: no flush needed",
        "parallelism": f"{world} independent boxes (no data-path collective)",
    }


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if smax and v > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
class _DeviceArray:
    """A device pointer viewed by torch without a copy (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


def _fields(h, torch):
    n = 1
    for v in h.params.shape:
        n *= int(v)
    return [torch.as_tensor(_DeviceArray(p, n), device="cuda") for p in h.device_field_ptrs()]


def precision_errors(test, ref, gamma=5.0 / 3.0):
    """L1 (relative) and L_inf (relative to max |ref|) of rho, rho*v and E of
    two device states (p, rho, vx, vy, vz), on the device."""
    def derived(f):
        p, rho, vx, vy, vz = f
        e = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
        return {"rho": rho, "rho_vx": rho * vx, "rho_vy": rho * vy, "rho_vz": rho * vz, "E": e}
    a, b = derived(test), derived(ref)
    out = {}
    for k in a:
        d = (a[k] - b[k]).abs()
        out[k] = {"l1": float(d.sum() / b[k].abs().sum()), "linf": float(d.max() / b[k].abs().max())}
    return out


def run_ours(args):
    import torch

    from hydropad_b200 import _lib as L
    from hydropad_b200 import ics
    from hydropad_b200.api import Hydro
    from hydropad_b200.params import HydroParams

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n, K, W = args.n, args.steps, args.warmup
    pre = max(W, COMPARE_STEPS - K)  # untimed steps before the timed window
    ic = ics.grf_eds_device(n, seed=BASE_SEED + rank, noise="host", device=f"cuda:{local}")
    torch.cuda.synchronize()
    prm = HydroParams(shape=(n, n, n), cosmo=True, tstop=TSTOP)
    cells = float(n) ** 3

    results = {}
    boxes = {}
    for prec in ("fp64", "mixed"):
        h = Hydro(prm, precision=prec, device=local)
        h.attach_device(*ic)
        h.autotune(reps=1)  # tiles of the untimed steps
        h.start_with_cfl()
        h.evolve(pre, graph=True)
        # tile shape per axis, timed on a scratch copy of the state the timed
        # steps start from (tiles change the speed only: every tile gives the
        # same bits)
        tiles = h.autotune(reps=3)
        stream = torch.cuda.ExternalStream(h.stream_handle())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = h.launch_count()
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            e0.record(stream)
            h.evolve_async(K, graph=True)
            e1.record(stream)
            h.synchronize()
            torch.cuda.synchronize()
        barrier()
        s = h.get_scalars()
        # every timed step advanced the box: the step loop had not reached
        # tstop (a finished box makes each sweep return at once)
        if not (s.told < prm.tstop) or s.nstep != 1 + pre + K:
            raise RuntimeError(f"timed steps did no work: told={s.told} tstop={prm.tstop} nstep={s.nstep}")
        ms = max_over_ranks(e0.elapsed_time(e1)) / K
        results[prec] = {"ms_per_step": ms, "value": world * cells / (ms * 1e-3),
                         "launches": h.launch_count() - l0, "clocks": clk.summary(), "tiles": tiles,
                         "steps_run": pre + K, "t_end": s.t, "a_end": s.t ** (2.0 / 3.0)}
        boxes[prec] = h
    errs = precision_errors(_fields(boxes["mixed"], torch), _fields(boxes["fp64"], torch))

    # per-sweep duration of the dominant kernel (the fused sweep), CUDA
    # events on the launching stream; 3 sweeps per ppm_lxlylz call
    for prec, h in boxes.items():
        stream = torch.cuda.ExternalStream(h.stream_handle())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 3
        torch.cuda.synchronize()
        e0.record(stream)
        for r in range(reps):
            L.check(L.lib().hp_ppm_lxlylz(h._ctx, 1 + r % 6), "hp_ppm_lxlylz")
        e1.record(stream)
        h.synchronize()
        torch.cuda.synchronize()
        results[prec]["sweep_ms"] = e0.elapsed_time(e1) / (3 * reps)
    state_host = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        state_host = boxes["fp64"].download()  # the FP64 state after the run, ghosted, for the CPU sample
    for h in boxes.values():
        h.close()
    del boxes

    # end to end through the C ABI with host buffers: upload the ghosted
    # Fortran arrays from pinned host memory, one step, download + ghost fill
    e2e = None
    if not args.no_e2e:
        nbg = n + 6
        pinned = [torch.empty(nbg ** 3, dtype=torch.float64, pin_memory=True) for _ in range(5)]
        host = [p.numpy().reshape((nbg, nbg, nbg), order="F") for p in pinned]
        h = Hydro(prm, precision="mixed", device=local)
        h.attach_device(*ic)
        h.download(out=host)
        h.set_tiles(*results["mixed"]["tiles"])
        h.attach_state(*host)
        h.start_with_cfl()
        h.evolve(1, graph=True)
        h.sync_to_host()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            h.attach_state(*host)          # H2D of the step's input state
            h.evolve(1, graph=True)        # the step (status read included)
            h.sync_to_host()               # D2H of the result + ghost refill
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        barrier()
        el = max_over_ranks(t1 - t0)
        # the interior planes of the ghosted arrays go up, the whole ghosted
        # arrays come back (ghosts refilled)
        h2d = 5 * 8 * n * nbg ** 2
        d2h = 5 * 8 * nbg ** 3
        e2e = {"value": world * cells * K / el, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * el / K,
               "path": "hp_attach_state + hp_evolve(1) + hp_sync_to_host, pinned ghosted Fortran arrays"}
        h.close()
        del pinned, host
    del ic
    torch.cuda.empty_cache()

    # the batched paths: the 64-box ensemble (mixed, 50 steps) and a bounded
    # serving trace (Poisson arrivals at 200/s), both split across the ranks
    ensemble = serving = None
    if args.serve_requests > 0:
        from hydropad_b200.ensemble import run_ensemble
        from hydropad_b200.serve import run_serving
        from hydropad_b200.shard import gather_objects
        per_rank = gather_objects(run_ensemble(64, 50, 3, "mixed", 4, True, world, rank, local))
        ems = max(r["ms"] for r in per_rank)
        ensemble = {"boxes": 64, "sides": per_rank[0]["sides"], "cells": per_rank[0]["total_cells"], "steps": 50,
                    "precision": "mixed", "tiles": per_rank[0]["tiles"], "ms_per_step": ems / 50,
                    "value": per_rank[0]["total_cells"] * 50 / (ems * 1e-3), "unit": UNIT,
                    "launches_per_step": per_rank[0]["launches"] / 50}
        serving = {"requests": args.serve_requests, "rate_per_s": 200.0, "trace_seed": 2024}
        for prec in ("mixed", "fp64"):
            st, stiles = run_serving(args.serve_requests, 200.0, 2024, prec, world=world, rank=rank, device=local)
            sm = st.summary()
            serving[prec] = {"p50_s": sm["latency_p50_s"], "p99_s": sm["latency_p99_s"],
                             "value": sm["cell_updates_per_s"], "unit": UNIT, "makespan_s": sm["makespan_s"],
                             "admission_stalls": sm["admission_stalls"], "budget_stalls": sm["budget_stalls"],
                             "peak_resident_gb": sm["peak_resident_gb"], "tiles": list(stiles),
                             # where the host's time went (seconds over the trace)
                             "host_admission_s": sm["host_admission_s"], "host_sync_wait_s": sm["host_sync_wait_s"],
                             "host_retire_s": sm["host_retire_s"], "batch_steps": sm["batch_steps"],
                             "max_queue": sm["max_queue"]}
        serving["offered_cell_updates_per_s"] = st.offered
        serving["budget_gb_per_gpu"] = st.budget_bytes / 1e9

    cpu = None
    if state_host is not None:
        cpu = cpu_baseline(state_host, prm, args)

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return

    mx, fp = results["mixed"], results["fp64"]
    peaks = load_peaks()
    sweep_s = mx["sweep_ms"] * 1e-3
    achieved = BYTES_PER_CELL_SWEEP * cells / sweep_s / 1e9
    traffic = load_traffic(n)
    line = {
        "metric": METRIC,
        "value": mx["value"],
        "unit": UNIT,
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": mx["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 reconstruction + f64 Riemann/update (mixed)",
        "data": "synthetic (seeded GRF initial conditions)",
        "config": workload_config(n, world, "mixed"),
        "fp64": {"value": fp["value"], "ms_per_step": fp["ms_per_step"], "sweep_ms": fp["sweep_ms"],
                 "tiles": fp["tiles"], "launches": fp["launches"], "clocks": fp["clocks"],
                 "roofline_frac": BYTES_PER_CELL_SWEEP * cells / (fp["sweep_ms"] * 1e-3) / 1e9 / peaks[0],
                 # the FP64 sweep's own ceiling: its FP64 pipe's active fraction
                 # (ncu, profiles/ppm_sweep_fp64_160_ncu_full.md)
                 "fp64_pipe_frac": load_profile_figure("fp64_pipe_frac")},
        "mixed_over_fp64": mx["value"] / fp["value"],
        "density_rel_l1_mixed_vs_fp64": errs["rho"]["l1"],
        "errors_mixed_vs_fp64": errs,
        "steps_compared": mx["steps_run"],
        "timed_window": f"steps {pre + 1}..{pre + K} of {pre + K} (untimed before)",
        "a_end": mx["a_end"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks[0], "unit": "GB/s",
                     "frac": achieved / peaks[0], "traffic": traffic, "peak_source": peaks[1],
                     "kernel": "ppm_sweep_kernel (mixed)",
                     "algorithmic_bytes_per_launch": BYTES_PER_CELL_SWEEP * cells},
        "gpu_launches": mx["launches"],
        "tiles": mx["tiles"],
        "clocks": mx["clocks"],
        "e2e": e2e,
        "cpu_baseline": cpu,
        "ensemble": ensemble,
        "serving": serving,
    }
    print(json.dumps(line), flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def load_profile_figure(key):
    """A figure of the committed ncu summary (profiles/ppm_sweep_traffic.txt),
    or None."""
    path = os.path.join(ROOT, "profiles", "ppm_sweep_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


def load_traffic(n):
    """DRAM bytes per sweep launch from the committed ncu summary (bytes
    per cell per sweep, times the cells of the box), or None."""
    per_cell = load_profile_figure("dram_bytes_per_cell_sweep")
    return None if per_cell is None else per_cell * n ** 3


# --------------------------------------------------------------------------
# CPU arms (oracle: the reference algorithm restated in C, all host cores)
# --------------------------------------------------------------------------
def _slab(state, planes, nb=3):
    """The first `planes` z planes of a ghosted state as a periodic box of
    its own (ghosts refilled)."""
    import numpy as np
    out = []
    for a in state:
        inner = a[nb:-nb, nb:-nb, nb:nb + planes]
        out.append(np.asfortranarray(np.pad(inner, nb, mode="wrap")))
    return out


def cpu_baseline(state, prm, args):
    """The oracle on the host cores, one step of a 512x512x32 sample of the
    box (the first 32 z planes as a periodic box): about the work of one
    sweep of the whole box in time, the same per-cell work."""
    from hydropad_b200.params import HydroParams
    from oracle import hp_oracle
    from tests.helpers import oracle_first_dt

    n = prm.shape[0]
    planes = min(REF_SLAB, n)
    threads = args.cpu_threads or os.cpu_count() or 1
    sub = HydroParams(shape=(n, n, planes), cosmo=True, tstop=prm.tstop)  # dx = 1/n, as the box's
    st = hp_oracle.OracleState(*_slab(state, planes))
    s = hp_oracle.make_scalars(sub)
    oracle_first_dt(hp_oracle, st, s)
    t0 = time.perf_counter()
    st.evolve(s, 1, threads)
    el = time.perf_counter() - t0
    return {"value": float(n) * n * planes / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"1 full step of a {n}x{n}x{planes} sample of the {n}^3 box (its first {planes} z planes "
                      f"after the GPU run, as a periodic box); C restatement of the reference STENCIL path "
                      f"(-O3, OpenMP over pencils, {threads} threads); per cell-update"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from hydropad_b200 import ics
    from hydropad_b200.params import HydroParams
    from oracle import hp_oracle
    from tests.helpers import oracle_first_dt

    n = args.n
    threads = args.cpu_threads or os.cpu_count() or 1
    # bounded sample of the workload: the n^3 initial state is generated in
    # full, and every step advances its first REF_SLAB z planes (a periodic
    # box of its own) by one full step -- the per-cell work of the box, in a
    # time that keeps the whole --steps/--warmup run within minutes
    planes = min(REF_SLAB, n)
    state = _slab(ics.grf_eds(n, seed=BASE_SEED), planes)
    prm = HydroParams(shape=(n, n, planes), cosmo=True, tstop=TSTOP)
    st = hp_oracle.OracleState(*state)
    s = hp_oracle.make_scalars(prm)
    oracle_first_dt(hp_oracle, st, s)
    st.evolve(s, args.warmup, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        st.evolve(s, 1, threads)
        times.append(time.perf_counter() - t0)
    el = sum(times)
    cells = float(n) * n * planes
    val = args.steps * cells / el
    sample = (f"each step: one full evolve_sys step of the first {planes} z planes of the {n}^3 initial state "
              f"({n}x{n}x{planes} cells, periodic), {args.steps} timed after {args.warmup} warm-up steps; "
              f"C restatement of the reference STENCIL path (FP64, -O3, OpenMP over pencils, {threads} threads); "
              f"per cell-update")
    line = {
        "impl": "reference",
        "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded GRF initial conditions)",
        "config": workload_config(n, 1, "fp64"),
        "ms_per_step_is": f"one step of the {n}x{n}x{planes} sample",
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(args.gpus)
    rank, world, _ = dist_env()
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
    run_ours(args)


if __name__ == "__main__":
    main()
