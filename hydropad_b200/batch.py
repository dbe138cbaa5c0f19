"""Many boxes advanced together (the ensemble and the serving engine).

A :class:`Batch` holds :class:`~hydropad_b200.api.Hydro` boxes of one
device and precision.  Each step sweeps every member with one persistent
launch per sweep axis (boxes of any size share the SMs through one work
queue) and runs timedet once per member; every member follows its own
evolve_sys step exactly (its own nrot, dt, nstep), so a box advanced in a
batch is bitwise identical to the same box advanced alone with the same
tiles.  The reference has no counterpart: it advances one box per run
(hydropad/main.F90:100-121).
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .api import Hydro

_PREC = {"fp64": L.HP_PREC_FP64, "mixed": L.HP_PREC_MIXED}


class BatchStatusError(L.HydroError):
    """A member's device status reported an error; ``statuses`` lists every
    member's code (0 = ok) in member order."""

    def __init__(self, code: int, statuses: list, what: str = ""):
        super().__init__(code, what)
        self.statuses = statuses


class Batch:
    """Members are driven only by the batch while they belong to it; read
    their state (``get_scalars``, ``download``, ``sync_to_host``) after
    :meth:`synchronize`."""

    def __init__(self, precision: str = "mixed", capacity: int = 64, device: int = 0):
        self.precision = precision
        self.capacity = int(capacity)
        self._b = C.c_void_p()
        L.check(L.lib().hp_batch_create(C.byref(self._b), int(device), _PREC[precision], self.capacity),
                "hp_batch_create")
        self.members: list[Hydro] = []

    def close(self):
        if self._b:
            L.lib().hp_batch_destroy(self._b)
            self._b = C.c_void_p()
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.members)

    # -- membership ----------------------------------------------------------
    def add(self, h: Hydro):
        L.check(L.lib().hp_batch_add(self._b, h._ctx), "hp_batch_add")
        self.members.append(h)

    def remove(self, h: Hydro):
        L.check(L.lib().hp_batch_remove(self._b, h._ctx), "hp_batch_remove")
        self.members.remove(h)

    # -- stepping ------------------------------------------------------------
    def step(self, nsteps: int = 1, graph: bool = True):
        """Enqueue nsteps steps of every member (returns without waiting)."""
        L.check(L.lib().hp_batch_step(self._b, int(nsteps), 1 if graph else 0), "hp_batch_step")

    def synchronize(self, raise_on_error: bool = True) -> list:
        """Wait for the batch; return each member's status code (0 = ok)."""
        n = len(self.members)
        st = (C.c_int * max(n, 1))()
        rc = L.lib().hp_batch_synchronize(self._b, st)
        codes = [int(st[i]) for i in range(n)]
        if rc != L.HP_OK and raise_on_error:
            if any(codes):
                raise BatchStatusError(rc, codes, "hp_batch_synchronize")
            L.check(rc, "hp_batch_synchronize")
        return codes

    # -- launch shape --------------------------------------------------------
    def set_tiles(self, tx: int, ty: int, tz: int):
        L.check(L.lib().hp_batch_set_tiles(self._b, int(tx), int(ty), int(tz)), "hp_batch_set_tiles")

    def get_tiles(self):
        t = (C.c_int * 3)()
        L.check(L.lib().hp_batch_get_tiles(self._b, t), "hp_batch_get_tiles")
        return tuple(t)

    def autotune(self, reps: int = 2):
        """Pick the fastest batched-sweep tile per axis over the current
        members (on scratch copies; the states are unchanged)."""
        L.check(L.lib().hp_batch_autotune(self._b, int(reps)), "hp_batch_autotune")
        return self.get_tiles()

    def stream_handle(self) -> int:
        return int(L.lib().hp_batch_stream(self._b) or 0)

    def launch_count(self) -> int:
        return int(L.lib().hp_batch_launch_count(self._b))
