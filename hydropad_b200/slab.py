"""One box split into z slabs: one slab per GPU for boxes that a single GPU
cannot hold or advance fast enough.

The reference decomposes its box into MPI blocks (hydropad/init_sys.F90:
53-60) and refreshes their ghost layers after every sweep
(exchange_mesh.F90 / exchange_var.F90); the CFL velmax is reduced over the
ranks (speed.F90).  Here each slab is an ordinary context made a slab by
``hp_slab_init``: its x and y sweeps are local, its z sweep reads 4 planes
below and 3 above from halo buffers refilled right before every z sweep,
and the step's velmax is the maximum over the slabs.  Every slab follows the
same nrot schedule and dt, so the split box gives the same bits as the box
advanced whole.

* :class:`LocalSlabs` -- all slabs of a box on one device in one process; the
  halo exchange is a device-to-device copy.  This is the single-GPU form of
  the split (and what the tests compare against the whole box).
* :class:`DistSlab` -- one slab per rank of a ``torch.distributed`` job
  (NCCL between GPUs): the edge planes go to the neighbours with
  point-to-point send/recv into local buffers, velmax with an all-reduce.
  The exchange and reduction logic is shared with :class:`LocalSlabs` and
  tested on CPU ranks (gloo) with host buffers.
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L


def slab_bounds(nz: int, world: int):
    """(z0, planes) of each of ``world`` slabs of an ``nz``-plane box: an
    even split, the remainder on the first slabs; every slab >= 4 planes."""
    if world < 1 or nz < 4 * world:
        raise ValueError(f"{nz} planes cannot be split into {world} slabs of >= 4 planes")
    base, extra = divmod(nz, world)
    out, z0 = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((z0, k))
        z0 += k
    return out


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def halo_buffers(nx: int, ny: int, device):
    """(top4, bottom3, lower4, upper3) buffers in the halo layout
    [p, rho, vx, vy, vz][planes][nx*ny]."""
    import torch
    plane = nx * ny
    mk = lambda k: torch.empty(5 * k * plane, dtype=torch.float64, device=device)
    return mk(4), mk(3), mk(4), mk(3)


def exchange_p2p(top4, bottom3, lower4, upper3, rank: int, world: int, group=None):
    """Send this slab's top 4 planes up and bottom 3 planes down; receive the
    lower halo from below and the upper halo from above (periodic in z).
    Posted in a fixed order so that two slabs that are each other's both
    neighbours (world = 2) match the right buffers."""
    import torch.distributed as dist
    if world == 1:
        lower4.copy_(top4)
        upper3.copy_(bottom3)
        return
    up, down = (rank + 1) % world, (rank - 1) % world
    ops = [dist.P2POp(dist.isend, top4, up, group), dist.P2POp(dist.isend, bottom3, down, group),
           dist.P2POp(dist.irecv, lower4, down, group), dist.P2POp(dist.irecv, upper3, up, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


class _Slabs:
    """Step logic shared by the local and the distributed forms."""

    ctxs: list  # Hydro objects of the slabs held by this process

    def _exchange(self):
        raise NotImplementedError

    def _max_all(self, v: float) -> float:
        return v

    def _step_once(self):
        lib = L.lib()
        for s in range(3):
            axis = lib.hp_step_axis(self.ctxs[0]._ctx, s)
            if axis < 0:
                L.check(axis, "hp_step_axis")
            if axis == 2:
                self._exchange()
            for h in self.ctxs:
                L.check(lib.hp_step_sweep(h._ctx, s), "hp_step_sweep")
        v = 0.0
        for h in self.ctxs:
            x = C.c_double()
            L.check(lib.hp_step_velmax(h._ctx, C.byref(x)), "hp_step_velmax")
            v = max(v, x.value)
        v = self._max_all(v)
        for h in self.ctxs:
            L.check(lib.hp_step_finish(h._ctx, v), "hp_step_finish")

    def step(self, nsteps: int = 1):
        for _ in range(int(nsteps)):
            self._step_once()

    def start_with_cfl(self):
        """dt of the first step from the CFL condition of the whole box (the
        configurations' choice; Hydro.start_with_cfl for one box)."""
        v = 0.0
        for h in self.ctxs:
            s = h.get_scalars()
            s.t = s.told
            h.set_scalars(s)
            v = max(v, h.speed())
        v = self._max_all(v)
        for h in self.ctxs:
            h.timedet(v)

    def autotune(self, reps: int = 1):
        """Tile shapes from the first slab of this process (hp_autotune on a
        scratch copy of its state), applied to every slab it holds.  The z
        sweep's halos do not change the per-cell work, so a slab tunes like
        a box of its own size."""
        tiles = self.ctxs[0].autotune(reps=reps)
        for h in self.ctxs[1:]:
            h.set_tiles(*tiles)
        return tiles

    def close(self):
        for h in self.ctxs:
            h.close()
        self.ctxs = []


class LocalSlabs(_Slabs):
    """A box of ``params.shape`` split into ``nslab`` z slabs on one device."""

    def __init__(self, params, nslab: int, precision: str = "fp64", device: int = 0):
        from dataclasses import replace

        from .api import Hydro
        nx, ny, nz = (int(v) for v in params.shape)
        self.bounds = slab_bounds(nz, nslab)
        self.ctxs = []
        for z0, k in self.bounds:
            h = Hydro(replace(params, shape=(nx, ny, k)), precision=precision, device=device)
            L.check(L.lib().hp_slab_init(h._ctx, nz, z0), "hp_slab_init")
            self.ctxs.append(h)
        dev = f"cuda:{device}"
        self.bufs = [halo_buffers(nx, ny, dev) for _ in self.bounds]

    def attach_device(self, p, rho, vx, vy, vz):
        """Whole-box device tensors (nz, ny, nx), split along z."""
        for h, (z0, k) in zip(self.ctxs, self.bounds):
            h.attach_device(*[t[z0:z0 + k].contiguous() for t in (p, rho, vx, vy, vz)])

    def _exchange(self):
        lib = L.lib()
        n = len(self.ctxs)
        for h, (top4, bottom3, _, _) in zip(self.ctxs, self.bufs):
            L.check(lib.hp_slab_get_edges(h._ctx, _ptr(top4), _ptr(bottom3)), "hp_slab_get_edges")
        for i, h in enumerate(self.ctxs):
            lower4 = self.bufs[(i - 1) % n][0]
            upper3 = self.bufs[(i + 1) % n][1]
            L.check(lib.hp_slab_set_halos(h._ctx, _ptr(lower4), _ptr(upper3)), "hp_slab_set_halos")

    def download(self):
        """The whole box (p, rho, vx, vy, vz), dense Fortran-order host arrays."""
        import numpy as np
        parts = [h.download(nbound=0) for h in self.ctxs]
        return [np.asfortranarray(np.concatenate([p[q] for p in parts], axis=2)) for q in range(5)]


class DistSlab(_Slabs):
    """This rank's slab of a box split over the ranks of the default
    ``torch.distributed`` group (one GPU per rank)."""

    def __init__(self, params, precision: str = "fp64", device: int = 0):
        from dataclasses import replace

        import torch.distributed as dist

        from .api import Hydro
        ready = dist.is_available() and dist.is_initialized()
        self.rank, self.world = (dist.get_rank(), dist.get_world_size()) if ready else (0, 1)
        nx, ny, nz = (int(v) for v in params.shape)
        self.bounds = slab_bounds(nz, self.world)
        self.z0, self.k = self.bounds[self.rank]
        h = Hydro(replace(params, shape=(nx, ny, self.k)), precision=precision, device=device)
        L.check(L.lib().hp_slab_init(h._ctx, nz, self.z0), "hp_slab_init")
        self.ctxs = [h]
        self.bufs = halo_buffers(nx, ny, f"cuda:{device}")

    def _exchange(self):
        import torch
        top4, bottom3, lower4, upper3 = self.bufs
        h = self.ctxs[0]
        L.check(L.lib().hp_slab_get_edges(h._ctx, _ptr(top4), _ptr(bottom3)), "hp_slab_get_edges")
        exchange_p2p(top4, bottom3, lower4, upper3, self.rank, self.world)
        torch.cuda.current_stream().synchronize()
        L.check(L.lib().hp_slab_set_halos(h._ctx, _ptr(lower4), _ptr(upper3)), "hp_slab_set_halos")

    def _max_all(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.bufs[0].device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def attach_device(self, p, rho, vx, vy, vz):
        """Whole-box device tensors (nz, ny, nx): this rank takes its planes."""
        z0, k = self.z0, self.k
        self.ctxs[0].attach_device(*[t[z0:z0 + k].contiguous() for t in (p, rho, vx, vy, vz)])


def main(argv=None):
    """One box split into z slabs over the ranks of a torchrun job (one GPU
    each, NCCL); strong scaling: the box is fixed, each rank advances its
    slab.  Prints one JSON line on rank 0 (cell-updates/s of the whole box,
    device time as the maximum over the ranks)."""
    import argparse
    import datetime
    import json
    import os

    import torch
    import torch.distributed as dist

    from . import ics
    from .params import HydroParams
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--seed", type=int, default=12345)
    args = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n = args.n
    prm = HydroParams(shape=(n, n, n), cosmo=True, tstop=1.0e4)
    sl = DistSlab(prm, precision=args.precision, device=dev)
    ic = ics.grf_eds_device(n, seed=args.seed, device=f"cuda:{dev}", noise="device")
    sl.attach_device(*ic)
    del ic
    torch.cuda.empty_cache()
    tiles = sl.autotune(reps=1)
    sl.start_with_cfl()
    sl.step(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    sl.step(args.steps)
    t1.record()
    t1.synchronize()
    ms = t0.elapsed_time(t1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if sl.rank == 0:
        print(json.dumps({"workload": f"{n}^3 EdS box in {world} z slab(s)", "precision": args.precision,
                          "n_gpus": world, "steps": args.steps, "ms_per_step": ms / args.steps,
                          "cell_updates_per_s": n ** 3 * args.steps / (ms * 1e-3), "scaling": "strong",
                          "tiles": list(tiles)}))
    sl.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
