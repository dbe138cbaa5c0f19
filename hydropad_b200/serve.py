"""Serving engine: simulation requests arriving over time, continuously batched.

    python -m hydropad_b200.serve --requests 100 --precision mixed

A request is one cosmological box (side, steps, seed); its response is the
box's final state, downloaded to the host.  The server keeps one
:class:`~hydropad_b200.batch.Batch` on the GPU and, at every step boundary,

* moves the requests that have arrived into a FIFO queue,
* admits queued requests while their device footprint fits the HBM budget
  (and the batch has a free slot); a head-of-queue request that does not fit
  is an admission stall -- later requests do not overtake it,
* generates each admitted box's initial conditions on the GPU and adds it to
  the batch,
* advances the batch by a chunk of steps (never past the step count of the
  member that finishes first),
* retires the members that are done: download, remove, record the latency
  from arrival to result.

Every member follows its own evolve_sys step, so a response is bitwise the
result of the same request run alone.  The reference has no serving layer:
it advances one box per run (hydropad/main.F90:100-121).

The scheduling logic (:class:`Scheduler`) is independent of the GPU: it
drives an engine object, which :class:`GpuEngine` implements on the library
and the tests replace by a CPU model.
"""
from __future__ import annotations

import argparse
import json
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

# device bytes per cell of one box: 5 FP64 state fields, 1 FP64
# density-peak buffer and the 4 fields of expand's step-start snapshot
# (FP64 in the FP64 path, FP32 in the mixed path)
BYTES_PER_CELL = {"fp64": 10 * 8, "mixed": 6 * 8 + 4 * 4}
CTL_BYTES = 4096


def box_bytes(side: int, precision: str = "fp64") -> int:
    return BYTES_PER_CELL[precision] * side ** 3 + CTL_BYTES


@dataclass
class Request:
    rid: int
    arrival: float      # seconds after the start of the trace
    side: int
    steps: int
    seed: int
    spectral_index: float = -2.0

    @property
    def cells(self) -> int:
        return self.side ** 3


@dataclass
class Completed:
    rid: int
    side: int
    steps: int
    arrival: float
    admitted: float
    done: float
    result: object = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def poisson_trace(n: int, rate: float = 200.0, seed: int = 2024, side_min: int = 32, side_max: int = 256,
                  step_min: int = 50, step_max: int = 500, seed_base: int = 12345):
    """The serving workload: Poisson arrivals at ``rate`` per second, sides
    log-uniform in [side_min, side_max] rounded to a multiple of 16, steps
    uniform in [step_min, step_max], one seed per request."""
    rng = np.random.Generator(np.random.PCG64(seed))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    raw = np.exp(rng.uniform(math.log(side_min), math.log(side_max), size=n))
    sides = np.clip(16 * np.rint(raw / 16.0), side_min, side_max).astype(int)
    steps = rng.integers(step_min, step_max + 1, size=n)
    return [Request(i, float(arrivals[i]), int(sides[i]), int(steps[i]), seed_base + i) for i in range(n)]


@dataclass
class Member:
    req: Request
    box: object
    remaining: int
    admitted: float


@dataclass
class ServeStats:
    completed: list = field(default_factory=list)
    admission_stalls: int = 0          # step boundaries at which the queue head did not fit
    budget_stalls: int = 0             # ... of them because of the HBM budget (a free slot, no room)
    stall_seconds: float = 0.0         # summed time the queue head waited for room
    max_queue: int = 0
    peak_resident_bytes: int = 0
    steps_launched: int = 0
    wall: float = 0.0
    budget_bytes: int = 0              # HBM budget of one rank
    offered: float = 0.0               # offered load of the whole trace, cell-updates/s
    create_s: float = 0.0              # host time in admission (allocation, initial conditions)
    sync_s: float = 0.0                # host time waiting for the batch at completions
    finish_s: float = 0.0              # host time in retirement (download of the results)

    def summary(self) -> dict:
        lat = np.array([c.latency for c in self.completed]) if self.completed else np.zeros(1)
        work = sum(c.side ** 3 * c.steps for c in self.completed)
        t0 = min((c.arrival for c in self.completed), default=0.0)
        t1 = max((c.done for c in self.completed), default=0.0)
        return {
            "requests": len(self.completed),
            "cell_updates": work,
            "cell_updates_per_s": work / (t1 - t0) if t1 > t0 else 0.0,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_mean_s": float(lat.mean()),
            "admission_stalls": self.admission_stalls,
            "budget_stalls": self.budget_stalls,
            "admission_stall_s": self.stall_seconds,
            "max_queue": self.max_queue,
            "peak_resident_gb": self.peak_resident_bytes / 1e9,
            "batch_steps": self.steps_launched,
            "makespan_s": t1 - t0,
            "host_admission_s": self.create_s,
            "host_sync_wait_s": self.sync_s,
            "host_retire_s": self.finish_s,
        }


def merge_stats(parts) -> ServeStats:
    """One job's statistics from the per-rank ones (each rank serves its own
    share of the trace on its own GPU)."""
    out = ServeStats()
    for st in parts:
        out.completed.extend(st.completed)
        out.admission_stalls += st.admission_stalls
        out.budget_stalls += st.budget_stalls
        out.stall_seconds += st.stall_seconds
        out.max_queue = max(out.max_queue, st.max_queue)
        out.peak_resident_bytes = max(out.peak_resident_bytes, st.peak_resident_bytes)
        out.steps_launched += st.steps_launched
        out.wall = max(out.wall, st.wall)
        out.create_s += st.create_s
        out.sync_s += st.sync_s
        out.finish_s += st.finish_s
    out.completed.sort(key=lambda c: c.rid)
    return out


class Scheduler:
    """Continuous batching at step boundaries under an HBM budget.

    engine interface: ``now()`` (seconds since the trace start),
    ``wait_until(t)``, ``create(req) -> box`` (allocate + initial
    conditions), ``add(box)``, ``step(k)`` (asynchronous), ``sync()``,
    ``detach(box)`` (leave the batch), ``finish(box) -> result``
    (download), ``release(box)``.

    When members finish, the scheduler waits for the batch, detaches them,
    enqueues the next chunk of the remaining members and only then reads
    the finished boxes back, so that the downloads overlap the GPU's work
    on the others."""

    def __init__(self, engine, budget_bytes: int, capacity: int = 64, chunk: int = 8, keep_results: bool = False):
        self.engine = engine
        self.precision = getattr(engine, "precision", "fp64")
        self.budget = int(budget_bytes)
        self.capacity = int(capacity)
        self.chunk = max(1, int(chunk))
        self.keep_results = keep_results

    def run(self, trace) -> ServeStats:
        eng = self.engine
        st = ServeStats()
        pending = deque(sorted(trace, key=lambda r: r.arrival))
        queue: deque = deque()
        active: list = []
        resident = 0
        stall_since = None
        inflight = False  # a chunk of the current members is enqueued and not yet accounted
        for r in pending:
            if box_bytes(r.side, self.precision) > self.budget:
                raise ValueError(f"request {r.rid} (side {r.side}) can never fit the HBM budget")
        while pending or queue or active:
            now = eng.now()
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            st.max_queue = max(st.max_queue, len(queue))
            # admission, FIFO: the head blocks the rest
            while queue and len(active) < self.capacity:
                need = box_bytes(queue[0].side, self.precision)
                if resident + need > self.budget:
                    break
                req = queue.popleft()
                tc = time.perf_counter()
                box = eng.create(req)
                eng.add(box)
                st.create_s += time.perf_counter() - tc
                resident += need
                active.append(Member(req, box, req.steps, eng.now()))
            st.peak_resident_bytes = max(st.peak_resident_bytes, resident)
            blocked = bool(queue) and (len(active) >= self.capacity or
                                       resident + box_bytes(queue[0].side, self.precision) > self.budget)
            if blocked:
                st.admission_stalls += 1
                if len(active) < self.capacity:
                    st.budget_stalls += 1
                if stall_since is None:
                    stall_since = eng.now()
            elif stall_since is not None:
                st.stall_seconds += eng.now() - stall_since
                stall_since = None
            if not active:
                if pending:
                    eng.wait_until(pending[0].arrival)
                continue
            if not inflight:
                self._launch(eng, st, active)
            inflight = False
            done = [m for m in active if m.remaining == 0]
            if done:
                tc = time.perf_counter()
                eng.sync()
                st.sync_s += time.perf_counter() - tc
                for m in done:
                    eng.detach(m.box)
                    active.remove(m)
                if active:
                    # the others run on while the finished boxes are read back
                    self._launch(eng, st, active)
                    inflight = True
                for m in done:
                    tc = time.perf_counter()
                    res = eng.finish(m.box)
                    st.finish_s += time.perf_counter() - tc
                    t = eng.now()
                    st.completed.append(Completed(m.req.rid, m.req.side, m.req.steps, m.req.arrival, m.admitted, t,
                                                  res if self.keep_results else None))
                    eng.release(m.box)
                    resident -= box_bytes(m.req.side, self.precision)
        if stall_since is not None:
            st.stall_seconds += eng.now() - stall_since
        st.wall = eng.now()
        return st

    def _launch(self, eng, st: ServeStats, active: list):
        """Enqueue a chunk of steps of every member, never past the step
        count of the member that finishes first."""
        k = min(self.chunk, min(m.remaining for m in active))
        eng.step(k)
        st.steps_launched += k
        for m in active:
            m.remaining -= k


class GpuEngine:
    """The scheduler's engine on the library: one batch, boxes created with
    GPU-generated initial conditions.  Finished contexts of a side are kept
    for the next request of that side while they fit ``pool_bytes``."""

    def __init__(self, precision: str = "mixed", capacity: int = 64, tiles=None, device: int = 0,
                 graph: bool = True, pool_bytes: int = 0, download: bool = True):
        from .batch import Batch
        self.precision = precision
        self.device = device
        self.graph = graph
        self.download = download
        self.batch = Batch(precision, capacity=capacity, device=device)
        if tiles is not None:
            self.batch.set_tiles(*tiles)
        self.pool: dict = {}
        self.pool_bytes = int(pool_bytes)
        self.pooled = 0
        self.reused = 0      # requests served by a kept context
        self.initial = {}
        self.t0 = time.perf_counter()

    def start_clock(self):
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def wait_until(self, t: float):
        d = t - self.now()
        if d > 0:
            time.sleep(d)

    @staticmethod
    def params(side: int):
        from .params import HydroParams
        # the box runs exactly its step count: the time limit is out of reach
        return HydroParams(shape=(side, side, side), cosmo=True, tstop=1.0e4)

    def create(self, req: Request):
        from . import ics
        from .api import Hydro
        free = self.pool.get(req.side)
        if free:
            h = free.pop()
            self.pooled -= box_bytes(req.side, self.precision)
            self.reused += 1
            h.set_scalars(self.initial[req.side])
        else:
            h = Hydro(self.params(req.side), precision=self.precision, device=self.device)
            if req.side not in self.initial:
                self.initial[req.side] = h.get_scalars()
        state = ics.grf_eds_device(req.side, seed=req.seed, spectral_index=req.spectral_index,
                                   device=f"cuda:{self.device}", noise="device")
        h.attach_device(*state)
        del state
        h.start_with_cfl()
        return h

    def add(self, h):
        self.batch.add(h)

    def step(self, k: int):
        self.batch.step(k, graph=self.graph)

    def sync(self):
        self.batch.synchronize()

    def detach(self, h):
        self.batch.remove(h)

    def finish(self, h):
        if not self.download:
            return None
        return h.download(nbound=0, out=pinned_fields(tuple(int(n) for n in h.params.shape)))

    def release(self, h):
        side = int(h.params.shape[0])
        if self.pooled + box_bytes(side, self.precision) <= self.pool_bytes:
            self.pool.setdefault(side, []).append(h)
            self.pooled += box_bytes(side, self.precision)
        else:
            h.close()

    def close(self):
        for hs in self.pool.values():
            for h in hs:
                h.close()
        self.pool = {}
        self.batch.close()


def tune_tiles(precision: str, sides=(64, 128, 192, 256), device: int = 0):
    """Batched-sweep tiles tuned on a warm-up batch of boxes with sides
    spanning the serving range (the batch autotuner, on scratch copies)."""
    eng = GpuEngine(precision, capacity=len(sides), device=device)
    try:
        boxes = [eng.create(Request(-1 - i, 0.0, s, 1, 777 + i)) for i, s in enumerate(sides)]
        for h in boxes:
            eng.add(h)
        tiles = eng.batch.autotune(reps=1)
        for h in boxes:
            eng.batch.remove(h)
            h.close()
    finally:
        eng.close()
    return tuple(tiles)


def pinned_fields(shape):
    """Five float64 Fortran-ordered arrays of ``shape`` in pinned host memory
    (torch's caching host allocator: a block freed with its arrays is handed
    out again), so that a finished box's download runs at DMA speed instead
    of faulting in fresh pageable pages."""
    import torch
    n = int(np.prod(shape))
    return [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape, order="F")
            for _ in range(5)]


def warm_up(sides=range(32, 257, 16), device: int = 0):
    """Server start-up: one initial-condition draw per admissible side, so
    that the FFT plans and kernels of the generator exist before the first
    request (the first draw of a side in a process costs tens of ms), and
    the pinned result buffers of each side, so that no request pays for
    pinning host memory."""
    import torch

    from . import ics
    for side in sides:
        ics.grf_eds_device(int(side), seed=0, device=f"cuda:{device}", noise="device")
    torch.cuda.synchronize(device)
    for side in sorted({int(s) for s in sides}, reverse=True):
        pinned_fields((side, side, side))  # allocated and freed: left in the cache


def run_alone(req: Request, precision: str, tiles=None, device: int = 0):
    """One request advanced by itself through hp_evolve (the parity
    reference of the serving path); returns the final state."""
    from . import ics
    from .api import Hydro
    h = Hydro(GpuEngine.params(req.side), precision=precision, device=device)
    with h:
        h.attach_device(*ics.grf_eds_device(req.side, seed=req.seed, spectral_index=req.spectral_index,
                                            device=f"cuda:{device}", noise="device"))
        if tiles is not None:
            h.set_tiles(*tiles)
        h.start_with_cfl()
        h.evolve(req.steps, graph=False)
        return h.download(nbound=0)


def run_serving(requests: int = 100, rate: float = 200.0, trace_seed: int = 2024, precision: str = "mixed",
                budget_bytes: int = 0, capacity: int = 64, chunk: int = 8, tiles=None, pool_bytes: int = -1,
                world: int = 1, rank: int = 0, device: int = 0):
    """This rank's share of the serving trace (:func:`shard_trace`), then one
    host gather: returns (merged statistics of every rank, tiles).
    ``pool_bytes`` < 0 keeps finished contexts for reuse up to a tenth of the
    budget (a context that is kept is not freed, and freeing device memory
    waits for the whole device)."""
    import torch

    from .shard import gather_objects, shard_trace
    trace = poisson_trace(requests, rate=rate, seed=trace_seed)
    mine = shard_trace(trace, world)[rank]
    if budget_bytes <= 0:
        free, _total = torch.cuda.mem_get_info(device)
        budget_bytes = int(0.8 * free)
    if pool_bytes < 0:
        pool_bytes = budget_bytes // 10
    if tiles is None:
        tiles = tune_tiles(precision, device=device)
    warm_up(device=device)
    eng = GpuEngine(precision, capacity=capacity, tiles=tiles, device=device, pool_bytes=pool_bytes)
    try:
        sched = Scheduler(eng, budget_bytes - eng.pool_bytes, capacity=capacity, chunk=chunk)
        gather_objects(None)  # barrier: the ranks start the trace clock together
        eng.start_clock()
        st = sched.run(mine)
    finally:
        eng.close()
    st = merge_stats(gather_objects(st))
    st.budget_bytes = budget_bytes
    st.offered = rate * float(np.mean([r.cells * r.steps for r in trace]))
    return st, tuple(tiles)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=100)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--trace-seed", type=int, default=2024)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--budget-gb", type=float, default=0.0, help="HBM budget (default: 80%% of free memory)")
    ap.add_argument("--capacity", type=int, default=64)
    ap.add_argument("--chunk", type=int, default=8)
    ap.add_argument("--tiles", default="auto",
                    help="batched-sweep tile per axis 'x,y,z', or 'auto' (tuned on a warm-up batch)")
    ap.add_argument("--pool-gb", type=float, default=-1.0,
                    help="keep finished contexts for reuse up to this size (default: a tenth of the budget)")
    args = ap.parse_args(argv)

    import os

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=3600))
    torch.cuda.set_device(dev)
    tiles = None if args.tiles == "auto" else tuple(int(t) for t in args.tiles.split(","))
    pool = int(args.pool_gb * 1e9) if args.pool_gb >= 0 else -1
    st, tiles = run_serving(args.requests, args.rate, args.trace_seed, args.precision, int(args.budget_gb * 1e9),
                            args.capacity, args.chunk, tiles, pool, world, rank, dev)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {"workload": "serving", "precision": args.precision, "rate_per_s": args.rate, "n_gpus": world,
           "trace_seed": args.trace_seed, "budget_gb": st.budget_bytes / 1e9, "capacity": args.capacity,
           "chunk": args.chunk, "tiles": list(tiles), "pool_gb": args.pool_gb,
           "offered_cell_updates_per_s": st.offered}
    out.update(st.summary())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
