"""Host-side mirror of the reference's hydro-step interface.

One :class:`Hydro` object is one box whose state lives in HBM.  Method names
follow the reference routines they replace:

=====================  =====================================================
``ppmsolver(nd)``      hydro/ppmsolver.F90:1-467 (one directional sweep)
``ppm_lxlylz(nrot)``   hydro/ppm_lxlylz.F90:1-223 (+ exchange_mesh)
``speed()``            hydropad/speed.F90:2-59
``timedet(velmax)``    hydropad/functions.F90:2-151
``evolve(nsteps)``     hydro part of evolve_sys.F90:30-130, looped as in
                       main.F90:100-121
``attach_state``       the `!$acc update device` of ppmsolver.F90:95
``sync_to_host``       the `!$acc update host` of ppm_lxlylz.F90:20
=====================  =====================================================

Host arrays are REAL(8) Fortran-order ``(nx, ny, nz)`` with ``nbound`` ghost
layers, the reference's module arrays (hydropad/matrix.F90:10).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .params import HydroParams


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous, "state arrays must be Fortran-ordered float64"
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Hydro:
    """One box advanced by the fused B200 sweeps."""

    def __init__(self, params: HydroParams, precision: str = "fp64", device: int = 0):
        self.params = params
        self.precision = precision
        p = L.HpParams()
        p.ngridx, p.ngridy, p.ngridz = (int(v) for v in params.shape)
        p.nbound = params.nbound
        p.gamma = params.gamma
        p.cour = params.cour
        p.ca = params.ca
        p.eta1 = params.eta1
        p.eta2 = params.eta2
        p.dmax = params.dmax
        p.flatvalue = params.flatvalue
        p.mingradflat = params.mingradflat
        p.dtinit = params.dtinit
        p.tstop = params.tstop
        p.cosmo = 1 if params.cosmo else 0
        p.expand_zero_old = 1 if params.expand_zero_old else 0
        p.a_start = params.a_start
        p.dt_cap = params.dt_cap
        p.precision = {"fp64": L.HP_PREC_FP64, "mixed": L.HP_PREC_MIXED}[precision]
        p.device = device
        self._ctx = C.c_void_p()
        L.check(L.lib().hp_init(C.byref(p), C.byref(self._ctx)), "hp_init")
        self._host = None
        self._gforce = None

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._ctx:
            L.lib().hp_finalize(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state --------------------------------------------------------------
    def attach_state(self, p3d, rho3d, vx3d, vy3d, vz3d, gforce=None):
        """Upload ghosted Fortran-order host arrays; the device copy becomes
        the working state (the arrays are kept for :meth:`sync_to_host`).
        ``gforce``: the static gravity force ``(3, nx, ny, nz)`` (ghosted,
        e.g. :func:`hydropad_b200.ics.static_gravity`), or None."""
        arrs = [np.asfortranarray(a, dtype=np.float64) for a in (p3d, rho3d, vx3d, vy3d, vz3d)]
        nx, ny, nz = arrs[0].shape
        nb = (nx - self.params.shape[0]) // 2
        g = None
        if gforce is not None:
            g = np.asfortranarray(gforce, dtype=np.float64)
            if g.shape != (3, nx, ny, nz):
                raise ValueError(f"gforce must have shape (3, {nx}, {ny}, {nz})")
        L.check(L.lib().hp_attach_state(self._ctx, *[_dptr(a) for a in arrs], None if g is None else _dptr(g),
                                        nx, ny, nz, nb), "hp_attach_state")
        self._host = arrs
        self._gforce = g
        return arrs

    def attach_device(self, p, rho, vx, vy, vz):
        """Take the state from device tensors (contiguous float64, shape
        ``(nz, ny, nx)``, x fastest, no ghosts; e.g. from
        :func:`hydropad_b200.ics.grf_eds_device`).  The tensors are copied;
        no host arrays are attached (use :meth:`download`)."""
        import torch
        shp = tuple(int(v) for v in self.params.shape)[::-1]
        ts = (p, rho, vx, vy, vz)
        for t in ts:
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or tuple(t.shape) != shp:
                raise ValueError(f"device state must be contiguous float64 CUDA tensors of shape {shp}")
        torch.cuda.current_stream(ts[0].device).synchronize()
        L.check(L.lib().hp_attach_device_state(self._ctx, *[C.c_void_p(t.data_ptr()) for t in ts]),
                "hp_attach_device_state")
        self._host = None
        self._gforce = None

    def attach_device_gforce(self, gx, gy, gz):
        """Static gravity force from device tensors (the three components,
        same layout as :meth:`attach_device`); ``None`` x3 switches it off."""
        import torch
        if gx is None:
            L.check(L.lib().hp_attach_device_gforce(self._ctx, None, None, None), "hp_attach_device_gforce")
            return
        shp = tuple(int(v) for v in self.params.shape)[::-1]
        for t in (gx, gy, gz):
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous() or tuple(t.shape) != shp:
                raise ValueError(f"gforce components must be contiguous float64 CUDA tensors of shape {shp}")
        torch.cuda.current_stream(gx.device).synchronize()
        L.check(L.lib().hp_attach_device_gforce(self._ctx, *[C.c_void_p(t.data_ptr()) for t in (gx, gy, gz)]),
                "hp_attach_device_gforce")

    def write_var(self, directory: str, fp64: bool = False):
        """The reference's end-of-run dump (write_var_mpi): rho.bin,
        pressure.bin, vx.bin, vy.bin, vz.bin, raw REAL(4) interiors in
        Fortran order (``fp64=True``: REAL(8) to ``*.f64.bin``)."""
        L.check(L.lib().hp_write_var(self._ctx, str(directory).encode(), 1 if fp64 else 0), "hp_write_var")

    def sync_to_host(self):
        L.check(L.lib().hp_sync_to_host(self._ctx), "hp_sync_to_host")
        return self._host

    def download(self, nbound: int | None = None, out=None):
        """Return (p, rho, vx, vy, vz) as ghosted Fortran arrays: new ones, or
        the five arrays of ``out`` (float64, Fortran order, the ghosted shape),
        e.g. views of pinned host memory, which the copies reach at full
        speed."""
        nb = self.params.nbound if nbound is None else nbound
        shp = tuple(int(n) + 2 * nb for n in self.params.shape)
        if out is None:
            out = [np.zeros(shp, dtype=np.float64, order="F") for _ in range(5)]
        else:
            out = list(out)
            if len(out) != 5 or any(a.shape != shp or a.dtype != np.float64 or not a.flags.f_contiguous
                                    for a in out):
                raise ValueError(f"download: out must be five float64 Fortran-ordered arrays of shape {shp}")
        L.check(L.lib().hp_download_state(self._ctx, *[_dptr(a) for a in out], *shp, nb), "hp_download_state")
        return out

    # -- the hydro step ----------------------------------------------------------
    def ppmsolver(self, ndirection: int):
        """One sweep through the drop-in entry point (Fortran by-reference
        argument list; the host arrays identify the attached state)."""
        a = self._host
        nx, ny, nz = (C.c_int(v) for v in a[0].shape)
        nb = C.c_int(self.params.nbound)
        nd = C.c_int(int(ndirection))
        g = getattr(self, "_gforce", None)
        rc = L.lib().hp_ppmsolver(self._ctx, *[_dptr(x) for x in a], None, None, None if g is None else _dptr(g),
                                  C.byref(nx), C.byref(ny), C.byref(nz), C.byref(nb), C.byref(nd))
        L.check(rc, "hp_ppmsolver")

    def set_variant(self, variant: str):
        """``"stencil"`` (default) or ``"pencil"``: the sweep of
        :meth:`ppm_lxlylz`, :meth:`evolve` and the step pieces -- the STENCIL
        build's sweeps or the non-STENCIL build's full-pencil ppm()
        (hydro/ppm.F90; FP64 only)."""
        code = {"stencil": L.HP_VARIANT_STENCIL, "pencil": L.HP_VARIANT_PENCIL}[variant]
        L.check(L.lib().hp_set_variant(self._ctx, code), "hp_set_variant")

    def get_variant(self) -> str:
        return "pencil" if L.lib().hp_get_variant(self._ctx) == L.HP_VARIANT_PENCIL else "stencil"

    def attach_cho(self, cho3d):
        """The cho3d array the full-pencil solver reads at density peaks
        (ghosted Fortran order, the shape of the attached arrays), or None."""
        if cho3d is None:
            L.check(L.lib().hp_attach_cho(self._ctx, None, 0, 0, 0, 0), "hp_attach_cho")
            self._cho = None
            return
        c = np.asfortranarray(cho3d, dtype=np.float64)
        nx, ny, nz = c.shape
        nb = (nx - self.params.shape[0]) // 2
        L.check(L.lib().hp_attach_cho(self._ctx, _dptr(c), nx, ny, nz, nb), "hp_attach_cho")
        self._cho = c

    def ppmsolver_pencil(self, ndirection: int):
        """One full-pencil sweep through the drop-in of the non-STENCIL
        ppmsolver (its argument list; the *3dnew arrays are not written)."""
        a = self._host
        nx, ny, nz = (C.c_int(v) for v in a[0].shape)
        nb = C.c_int(self.params.nbound)
        nd = C.c_int(int(ndirection))
        g = getattr(self, "_gforce", None)
        cho = getattr(self, "_cho", None)
        rc = L.lib().hp_ppmsolver_pencil(self._ctx, *[_dptr(x) for x in a], None if cho is None else _dptr(cho),
                                         None, None if g is None else _dptr(g), *[None] * 6,
                                         C.byref(nx), C.byref(ny), C.byref(nz), C.byref(nb), C.byref(nd))
        L.check(rc, "hp_ppmsolver_pencil")

    def bad_cell(self):
        """(i, j, k) interior indices of the first cell that the last error
        status reported (NaN, or non-positive density or pressure), or None."""
        c = int(L.lib().hp_bad_cell(self._ctx))
        if c < 0:
            return None
        nx, ny, _ = (int(v) for v in self.params.shape)
        return (c % nx, (c // nx) % ny, c // (nx * ny))

    def _check_status(self, rc: int, what: str):
        if rc in (-5, -6):  # HP_ERR_NAN, HP_ERR_NEGATIVE_STATE: name the first cell
            what = f"{what} (first bad cell {self.bad_cell()})"
        L.check(rc, what)

    def ppm_lxlylz(self, nrot: int):
        L.check(L.lib().hp_ppm_lxlylz(self._ctx, int(nrot)), "hp_ppm_lxlylz")
        self._check_status(L.lib().hp_synchronize(self._ctx), "hp_ppm_lxlylz")

    def speed(self) -> float:
        v = C.c_double()
        L.check(L.lib().hp_speed(self._ctx, C.byref(v)), "hp_speed")
        return v.value

    def timedet(self, velmax: float):
        L.check(L.lib().hp_timedet(self._ctx, float(velmax)), "hp_timedet")

    def start_with_cfl(self):
        """Take the first step's dt from the CFL condition of the attached
        state instead of dtinit: the clock is put back to the initial time
        (told) and speed + timedet run once (the configurations' choice)."""
        s = self.get_scalars()
        s.t = s.told
        self.set_scalars(s)
        self.timedet(self.speed())

    def evolve(self, nsteps: int, graph: bool = True):
        self._check_status(L.lib().hp_evolve(self._ctx, int(nsteps), 1 if graph else 0), "hp_evolve")

    def evolve_async(self, nsteps: int, graph: bool = True):
        """Enqueue nsteps without waiting or reading the status (for timing
        loops); call :meth:`synchronize` afterwards."""
        L.check(L.lib().hp_evolve_async(self._ctx, int(nsteps), 1 if graph else 0), "hp_evolve_async")

    def synchronize(self):
        self._check_status(L.lib().hp_synchronize(self._ctx), "hp_synchronize")

    # -- scalars ------------------------------------------------------------------
    def get_scalars(self) -> L.HpScalars:
        s = L.HpScalars()
        L.check(L.lib().hp_get_scalars(self._ctx, C.byref(s)), "hp_get_scalars")
        return s

    def set_scalars(self, s: L.HpScalars):
        L.check(L.lib().hp_set_scalars(self._ctx, C.byref(s)), "hp_set_scalars")

    # -- launch shape --------------------------------------------------------------
    def set_tiles(self, tx: int, ty: int, tz: int):
        L.check(L.lib().hp_set_tiles(self._ctx, int(tx), int(ty), int(tz)), "hp_set_tiles")

    def get_tiles(self):
        t = (C.c_int * 3)()
        L.check(L.lib().hp_get_tiles(self._ctx, t), "hp_get_tiles")
        return tuple(t)

    def autotune(self, reps: int = 2):
        """Pick the fastest sweep tile per axis on a scratch copy of the state."""
        L.check(L.lib().hp_autotune(self._ctx, int(reps)), "hp_autotune")
        return self.get_tiles()

    def stream_handle(self) -> int:
        return int(L.lib().hp_stream(self._ctx) or 0)

    def launch_count(self) -> int:
        return int(L.lib().hp_launch_count(self._ctx))

    def device_field_ptrs(self):
        ptrs = [C.POINTER(C.c_double)() for _ in range(5)]
        L.check(L.lib().hp_device_fields(self._ctx, *[C.byref(p) for p in ptrs]), "hp_device_fields")
        return [C.cast(p, C.c_void_p).value for p in ptrs]
