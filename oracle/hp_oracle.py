"""ctypes binding of the CPU oracle (oracle/libhp_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline legs of bench.py, always as the checker or the timed
CPU reference, never on the product path.  Parity of the oracle with the
Fortran reference is UNPINNED (no Fortran compiler, no reference test
vectors); see the header of hp_oracle.c.

Arrays are numpy float64 in Fortran order, shape (nx, ny, nz) with ``nbound``
ghost layers, exactly the reference's module arrays (hydropad/matrix.F90:10).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libhp_oracle.so")


class HpoScalars(C.Structure):
    """Mirror of ``hpo_scalars`` (hp_oracle.h)."""

    _fields_ = [(n, C.c_double) for n in (
        "gamma", "rgamma", "gamma1", "rgamma1", "m", "rm", "gf",
        "mingradflat", "flatvalue",
        "dmax", "eta1", "eta2", "cour", "ca",
        "dx", "rdx",
        "dt", "rdtath", "at", "dat", "rat", "ath", "dath",
        "t", "told", "thalf", "dtold", "tstop", "atnew", "datnew",
        "dt_cap", "velmax")] + [
        ("nstep", C.c_int), ("cosmo", C.c_int), ("expand_zero_old", C.c_int), ("pencil", C.c_int)]


def build() -> str:
    """Compile the oracle with its Makefile if the library is missing/stale."""
    src = os.path.join(_HERE, "hp_oracle.c")
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "hp_oracle.h"))):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        sp = C.POINTER(HpoScalars)
        L.hpo_derive_constants.argtypes = [sp, C.c_double, C.c_int]
        L.hpo_ppmsolver.argtypes = [dp] * 5 + [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, sp, C.c_int]
        L.hpo_ppmsolver.restype = C.c_int
        L.hpo_ppmsolver_pencil.argtypes = [dp] * 5 + [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, sp, C.c_int]
        L.hpo_ppmsolver_pencil.restype = C.c_int
        L.hpo_exchange_mesh.argtypes = [dp] * 5 + [C.c_int] * 4
        L.hpo_ppm_lxlylz.argtypes = [dp] * 5 + [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, sp, C.c_int]
        L.hpo_ppm_lxlylz.restype = C.c_int
        L.hpo_speed.argtypes = [dp] * 5 + [C.c_int] * 4 + [sp]
        L.hpo_speed.restype = C.c_double
        L.hpo_timedet.argtypes = [sp]
        L.hpo_timedet_cosmo.argtypes = [sp]
        L.hpo_init_time.argtypes = [sp, C.c_double, C.c_double]
        L.hpo_expand.argtypes = [dp] * 4 + [dp] * 4 + [C.c_int] * 3 + [sp]
        L.hpo_evolve.argtypes = [dp] * 5 + [dp, C.c_int, C.c_int, C.c_int, C.c_int, sp, C.c_int, C.c_int]
        L.hpo_evolve.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.f_contiguous, "oracle arrays must be Fortran-ordered float64"
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_scalars(params) -> HpoScalars:
    """Build oracle scalars from a ``hydropad_b200.params.HydroParams``-like
    object (any object with the namelist attributes)."""
    s = HpoScalars()
    lib().hpo_derive_constants(C.byref(s), float(params.gamma), int(params.ngrid_max))
    s.mingradflat = params.mingradflat
    s.flatvalue = params.flatvalue
    s.dmax = params.dmax
    s.eta1 = params.eta1
    s.eta2 = params.eta2
    s.cour = params.cour
    s.ca = params.ca
    s.tstop = params.tstop
    s.dt_cap = params.dt_cap
    s.cosmo = 1 if params.cosmo else 0
    s.expand_zero_old = 1 if params.expand_zero_old else 0
    lib().hpo_init_time(C.byref(s), float(params.dtinit), float(params.a_start))
    return s


class OracleState:
    """Ghosted Fortran-order state (p, rho, vx, vy, vz) driven by the oracle."""

    def __init__(self, p, rho, vx, vy, vz, nbound=3, gforce=None, cho=None):
        self.f = [np.array(a, dtype=np.float64, order="F", copy=True) for a in (p, rho, vx, vy, vz)]
        self.nbound = nbound
        self.gforce = None if gforce is None else np.asfortranarray(gforce, dtype=np.float64)
        # cho3d of the non-STENCIL build's pencil solver (ghosted), or None (zeros)
        self.cho = None if cho is None else np.asfortranarray(cho, dtype=np.float64)
        self.nx, self.ny, self.nz = self.f[0].shape

    @property
    def p(self):
        return self.f[0]

    @property
    def rho(self):
        return self.f[1]

    def exchange(self):
        lib().hpo_exchange_mesh(*[_ptr(a) for a in self.f], self.nx, self.ny, self.nz, self.nbound)

    def ppmsolver(self, s: HpoScalars, ndirection: int, nthreads: int = 0) -> int:
        return lib().hpo_ppmsolver(*[_ptr(a) for a in self.f], _ptr(self.gforce), self.nx, self.ny,
                                   self.nz, self.nbound, ndirection, C.byref(s), nthreads)

    def ppmsolver_pencil(self, s: HpoScalars, ndirection: int, nthreads: int = 0) -> int:
        """One sweep of the non-STENCIL build (ppm() per pencil + savetn);
        the ghost fill that ppm_lxlylz does after it is left to the caller."""
        return lib().hpo_ppmsolver_pencil(*[_ptr(a) for a in self.f], _ptr(self.cho), self.nx, self.ny,
                                          self.nz, self.nbound, ndirection, C.byref(s), nthreads)

    def ppm_lxlylz(self, s: HpoScalars, nrot: int, nthreads: int = 0) -> int:
        return lib().hpo_ppm_lxlylz(*[_ptr(a) for a in self.f], _ptr(self.gforce), self.nx, self.ny,
                                    self.nz, self.nbound, nrot, C.byref(s), nthreads)

    def speed(self, s: HpoScalars) -> float:
        return lib().hpo_speed(*[_ptr(a) for a in self.f], self.nx, self.ny, self.nz, self.nbound,
                               C.byref(s))

    def evolve(self, s: HpoScalars, nsteps: int, nthreads: int = 0) -> int:
        return lib().hpo_evolve(*[_ptr(a) for a in self.f], _ptr(self.gforce), self.nx, self.ny, self.nz,
                                self.nbound, C.byref(s), nsteps, nthreads)

    def interior(self, idx):
        nb = self.nbound
        return self.f[idx][nb:self.nx - nb, nb:self.ny - nb, nb:self.nz - nb]
