"""hp_ppmsolver_noalloc: the sweep for callers that cannot allocate device
memory -- a host that owns every device array and budgets device memory
itself, a process whose device memory is capped, or a framework whose
caching allocator owns the device.  The caller passes the state arrays; the
scratch lives in a static device array inside the library.

Checked against the allocating entry point (hp_ppmsolver on an attached
context) on three calls in a row (x, y, z sweeps), with the single-sweep
tolerance the parity tests use: on a cosmological box, and on a non-cubic
box with density spikes and a low dmax, where the y/z sweeps run the
density-peak pre-pass (its values occupy the second part of the static
array).  Collected last on purpose (file name), so a failure here comes
after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import grf_state, interior, params_for, rel_l1

pytestmark = pytest.mark.gpu

SWEEP_TOL = 1e-13  # test_gpu_parity.test_single_sweep_fp64


def _dense(a):
    """Ghosted Fortran-order host array -> dense interior, x fastest."""
    return np.ascontiguousarray(interior(a).ravel(order="F"))


def _params_struct(h):
    from hydropad_b200 import _lib as L
    prm = h.params
    p = L.HpParams()
    p.ngridx, p.ngridy, p.ngridz = prm.shape
    p.nbound = prm.nbound
    p.gamma, p.cour, p.ca, p.eta1, p.eta2, p.dmax = prm.gamma, prm.cour, prm.ca, prm.eta1, prm.eta2, prm.dmax
    p.flatvalue, p.mingradflat, p.dtinit, p.tstop = prm.flatvalue, prm.mingradflat, prm.dtinit, prm.tstop
    p.cosmo, p.expand_zero_old = int(prm.cosmo), int(prm.expand_zero_old)
    p.a_start, p.dt_cap = prm.a_start, prm.dt_cap
    p.precision = {"fp64": L.HP_PREC_FP64, "mixed": L.HP_PREC_MIXED}[h.precision]
    p.device = 0
    return p


@pytest.mark.parametrize("case", ["grf", "peak"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_noalloc_matches_allocating_entry_point(prec, case):
    import torch

    from hydropad_b200 import _lib as L
    from hydropad_b200.api import Hydro

    if case == "grf":
        shape = (32, 32, 32)
        state = grf_state(32, seed=29)
        prm = params_for(shape, cosmo=True)
    else:
        from tests.test_gpu_peak import spiky_state
        shape = (32, 24, 40)
        state = spiky_state(shape, seed=31)
        prm = params_for(shape, dmax=1.5)
    nx, ny, nz = shape
    with Hydro(prm, precision=prec) as h:
        h.attach_state(*state)
        h.start_with_cfl()
        scal = h.get_scalars()
        pstruct = _params_struct(h)
        dev = [torch.from_numpy(_dense(a)).cuda() for a in state]  # p, rho, vx, vy, vz
        torch.cuda.synchronize()
        for call, nd in enumerate((1, 2, 3)):  # three calls in a row
            h.ppmsolver(nd)
            ref = h.download()
            rc = L.lib().hp_ppmsolver_noalloc(*[C.c_void_p(t.data_ptr()) for t in dev], nx, ny, nz, nd,
                                              C.byref(pstruct), C.byref(scal), None)
            assert rc == 0, L.lib().hp_strerror(rc)
            for q in range(5):
                got = dev[q].cpu().numpy()
                want = _dense(ref[q])
                if np.abs(want).sum() == 0:
                    assert np.abs(got).max() == 0.0
                    continue
                e = rel_l1(got, want)
                assert e <= SWEEP_TOL, (prec, case, call, q, e)


def test_noalloc_rejects_boxes_beyond_its_scratch():
    import torch

    from hydropad_b200 import _lib as L
    from hydropad_b200.params import HydroParams

    p = L.HpParams()
    p.ngridx = p.ngridy = p.ngridz = 128  # 2,097,152 cells > 1,048,576
    p.nbound = 3
    p.gamma = 5.0 / 3.0
    p.precision = L.HP_PREC_FP64
    s = L.HpScalars()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    ptr = C.c_void_p(t.data_ptr())
    rc = L.lib().hp_ppmsolver_noalloc(ptr, ptr, ptr, ptr, ptr, 128, 128, 128, 1, C.byref(p), C.byref(s), None)
    assert rc == -1  # HP_ERR_ARG, nothing launched
    del HydroParams
