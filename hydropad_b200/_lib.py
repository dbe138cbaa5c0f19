"""ctypes binding of libhydropad_b200.so (the C ABI in include/hydropad_b200.h).

The library is the only compute path: if it is missing this module raises
at import time instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

from .build import LIB_PATH

HP_OK = 0
HP_ERR = {
    -1: "HP_ERR_ARG", -2: "HP_ERR_CUDA", -3: "HP_ERR_OOM", -4: "HP_ERR_NEWTON", -5: "HP_ERR_NAN",
    -6: "HP_ERR_NEGATIVE_STATE", -7: "HP_ERR_NOT_ATTACHED", -8: "HP_ERR_STATE_MISMATCH", -9: "HP_ERR_NO_DEVICE",
    -10: "HP_ERR_UNSUPPORTED", -11: "HP_ERR_TIMEOUT",
}
HP_PREC_FP64 = 0
HP_PREC_MIXED = 1
HP_VARIANT_STENCIL = 0   # the STENCIL build's sweeps (default)
HP_VARIANT_PENCIL = 1    # the non-STENCIL build's full-pencil ppm() (hydro/ppm.F90)


class HpParams(C.Structure):
    _fields_ = [
        ("ngridx", C.c_int), ("ngridy", C.c_int), ("ngridz", C.c_int), ("nbound", C.c_int),
        ("gamma", C.c_double), ("cour", C.c_double), ("ca", C.c_double), ("eta1", C.c_double),
        ("eta2", C.c_double), ("dmax", C.c_double), ("flatvalue", C.c_double), ("mingradflat", C.c_double),
        ("dtinit", C.c_double), ("tstop", C.c_double),
        ("cosmo", C.c_int), ("expand_zero_old", C.c_int),
        ("a_start", C.c_double), ("dt_cap", C.c_double),
        ("precision", C.c_int), ("device", C.c_int),
    ]


class HpScalars(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dt", "rdtath", "at", "dat", "rat", "ath", "dath",
        "t", "told", "thalf", "dtold", "atnew", "datnew", "velmax")] + [
        ("nstep", C.c_int), ("pad", C.c_int)]


class HydroError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = HP_ERR.get(code, str(code))
        msg = lib().hp_strerror(code).decode()
        super().__init__(f"{what}: {name} ({msg})" if what else f"{name} ({msg})")


EXPORTS = (
    "hp_init", "hp_finalize", "hp_set_scalars", "hp_get_scalars", "hp_attach_state", "hp_sync_to_host",
    "hp_download_state", "hp_ppmsolver", "hp_ppm_lxlylz", "hp_speed", "hp_timedet", "hp_evolve",
    "hp_synchronize", "hp_stream", "hp_device_fields", "hp_strerror", "hp_launch_count", "hp_set_tiles",
    "hp_get_tiles", "hp_autotune", "hp_ppmsolver_noalloc", "hp_attach_device_state",
    "hp_write_var", "hp_evolve_async", "hp_attach_device_gforce", "hp_num_tiles",
    "hp_slab_init", "hp_slab_get_edges", "hp_slab_set_halos", "hp_step_axis", "hp_step_sweep",
    "hp_step_velmax", "hp_step_finish",
    "hp_batch_create", "hp_batch_destroy", "hp_batch_add", "hp_batch_remove", "hp_batch_size",
    "hp_batch_step", "hp_batch_synchronize", "hp_batch_member", "hp_batch_set_tiles", "hp_batch_get_tiles",
    "hp_batch_autotune", "hp_batch_stream", "hp_batch_launch_count",
    "hp_set_variant", "hp_get_variant", "hp_attach_cho", "hp_ppmsolver_pencil", "hp_bad_cell",
)
_NOT_INT = ("hp_stream", "hp_strerror", "hp_launch_count", "hp_batch_member", "hp_batch_stream",
            "hp_batch_launch_count", "hp_bad_cell")

_lib = None


def lib():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m hydropad_b200.build` (needs nvcc)")
    L = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    cp = C.c_void_p
    L.hp_init.argtypes = [C.POINTER(HpParams), C.POINTER(cp)]
    L.hp_finalize.argtypes = [cp]
    L.hp_set_scalars.argtypes = [cp, C.POINTER(HpScalars)]
    L.hp_get_scalars.argtypes = [cp, C.POINTER(HpScalars)]
    L.hp_attach_state.argtypes = [cp, dp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.hp_attach_device_state.argtypes = [cp, cp, cp, cp, cp, cp]
    L.hp_write_var.argtypes = [cp, C.c_char_p, C.c_int]
    L.hp_num_tiles.argtypes = []
    L.hp_slab_init.argtypes = [cp, C.c_int, C.c_int]
    L.hp_slab_get_edges.argtypes = [cp, cp, cp]
    L.hp_slab_set_halos.argtypes = [cp, cp, cp]
    L.hp_step_axis.argtypes = [cp, C.c_int]
    L.hp_step_sweep.argtypes = [cp, C.c_int]
    L.hp_step_velmax.argtypes = [cp, dp]
    L.hp_step_finish.argtypes = [cp, C.c_double]
    L.hp_attach_device_gforce.argtypes = [cp, cp, cp, cp]
    L.hp_sync_to_host.argtypes = [cp]
    L.hp_download_state.argtypes = [cp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.hp_ppmsolver.argtypes = [cp, dp, dp, dp, dp, dp, dp, dp, dp, ip, ip, ip, ip, ip]
    L.hp_ppm_lxlylz.argtypes = [cp, C.c_int]
    L.hp_set_variant.argtypes = [cp, C.c_int]
    L.hp_get_variant.argtypes = [cp]
    L.hp_attach_cho.argtypes = [cp, dp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.hp_ppmsolver_pencil.argtypes = [cp] + [dp] * 14 + [ip] * 5
    L.hp_speed.argtypes = [cp, dp]
    L.hp_timedet.argtypes = [cp, C.c_double]
    L.hp_evolve.argtypes = [cp, C.c_int, C.c_int]
    L.hp_evolve_async.argtypes = [cp, C.c_int, C.c_int]
    L.hp_synchronize.argtypes = [cp]
    L.hp_stream.argtypes = [cp]
    L.hp_stream.restype = cp
    L.hp_device_fields.argtypes = [cp] + [C.POINTER(dp)] * 5
    L.hp_strerror.argtypes = [C.c_int]
    L.hp_strerror.restype = C.c_char_p
    L.hp_launch_count.argtypes = [cp]
    L.hp_launch_count.restype = C.c_longlong
    L.hp_bad_cell.argtypes = [cp]
    L.hp_bad_cell.restype = C.c_longlong
    L.hp_set_tiles.argtypes = [cp, C.c_int, C.c_int, C.c_int]
    L.hp_get_tiles.argtypes = [cp, ip]
    L.hp_autotune.argtypes = [cp, C.c_int]
    L.hp_ppmsolver_noalloc.argtypes = [cp, cp, cp, cp, cp, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(HpParams), C.POINTER(HpScalars), cp]
    L.hp_batch_create.argtypes = [C.POINTER(cp), C.c_int, C.c_int, C.c_int]
    L.hp_batch_destroy.argtypes = [cp]
    L.hp_batch_add.argtypes = [cp, cp]
    L.hp_batch_remove.argtypes = [cp, cp]
    L.hp_batch_size.argtypes = [cp]
    L.hp_batch_step.argtypes = [cp, C.c_int, C.c_int]
    L.hp_batch_synchronize.argtypes = [cp, ip]
    L.hp_batch_member.argtypes = [cp, C.c_int]
    L.hp_batch_member.restype = cp
    L.hp_batch_set_tiles.argtypes = [cp, C.c_int, C.c_int, C.c_int]
    L.hp_batch_get_tiles.argtypes = [cp, ip]
    L.hp_batch_autotune.argtypes = [cp, C.c_int]
    L.hp_batch_stream.argtypes = [cp]
    L.hp_batch_stream.restype = cp
    L.hp_batch_launch_count.argtypes = [cp]
    L.hp_batch_launch_count.restype = C.c_longlong
    for name in EXPORTS:
        if name not in _NOT_INT:
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def num_tiles() -> int:
    """Tile shapes per axis of the sweep kernels."""
    return int(lib().hp_num_tiles())


def check(rc: int, what: str = "") -> None:
    if rc != HP_OK:
        raise HydroError(rc, what)
