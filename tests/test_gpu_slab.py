"""GPU: a box split into z slabs (halo planes refilled before every z sweep,
velmax reduced over the slabs) against the same box advanced whole: the
same bits, for every nrot order and both precisions."""
import numpy as np
import pytest

from tests.helpers import grf_state, params_for, sod_state

pytestmark = pytest.mark.gpu


def _device(state):
    import torch
    nb = 3
    return [torch.from_numpy(np.ascontiguousarray(a[nb:-nb, nb:-nb, nb:-nb].transpose(2, 1, 0))).cuda()
            for a in state]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nslab", [2, 3])
@pytest.mark.parametrize("case", ["grf", "sodz"])
def test_slabs_match_whole_box(precision, nslab, case):
    from hydropad_b200.api import Hydro
    from hydropad_b200.slab import LocalSlabs
    if case == "grf":
        # a non-cubic box: a (24, 20, 28) block of a 28^3 field, periodic again
        shape = (24, 20, 28)
        prm = params_for(shape, cosmo=True)
        state = [np.asfortranarray(np.pad(a[3:27, 3:23, 3:31], 3, mode="wrap")) for a in grf_state(28, seed=9)]
    else:
        shape = (16, 16, 32)
        state = sod_state(shape, axis=2)
        prm = params_for(shape)
    steps = 7
    with Hydro(prm, precision=precision) as h:
        h.attach_state(*state)
        h.start_with_cfl()
        h.evolve(steps, graph=False)
        whole = h.download(nbound=0)
        ref_t = h.get_scalars().t
    sl = LocalSlabs(prm, nslab, precision=precision)
    try:
        sl.attach_device(*_device(state))
        sl.start_with_cfl()
        sl.step(steps)
        split = sl.download()
        t = sl.ctxs[0].get_scalars().t
    finally:
        sl.close()
    assert t == ref_t
    for q, (a, b) in enumerate(zip(split, whole)):
        assert np.array_equal(a, b), f"field {q}: max |d| {np.abs(a - b).max():.3e}"


def test_slab_reports_peak_fix_across_slabs():
    from hydropad_b200._lib import HydroError
    from hydropad_b200.slab import LocalSlabs
    n = 16
    prm = params_for((n, n, n), cosmo=True, dmax=1.5)
    sl = LocalSlabs(prm, 2, precision="fp64")
    try:
        sl.attach_device(*_device(grf_state(n, seed=3)))
        sl.start_with_cfl()
        with pytest.raises(HydroError, match="UNSUPPORTED"):
            sl.step(3)
    finally:
        sl.close()


def test_slab_context_refuses_whole_box_stepping():
    from hydropad_b200._lib import HydroError
    from hydropad_b200.slab import LocalSlabs
    sl = LocalSlabs(params_for((16, 16, 16)), 2)
    try:
        sl.attach_device(*_device(sod_state(16)))
        with pytest.raises(HydroError, match="ARG"):
            sl.ctxs[0].evolve(1)
    finally:
        sl.close()


def test_dist_slab_single_rank_matches_whole_box():
    """The per-rank form with one rank (no process group): its exchange is
    the periodic self-copy."""
    from hydropad_b200.api import Hydro
    from hydropad_b200.slab import DistSlab
    n = 20
    prm = params_for((n, n, n), cosmo=True)
    state = grf_state(n, seed=4)
    with Hydro(prm, precision="mixed") as h:
        h.attach_state(*state)
        h.start_with_cfl()
        h.evolve(6, graph=False)
        whole = h.download(nbound=0)
    sl = DistSlab(prm, precision="mixed")
    try:
        sl.attach_device(*_device(state))
        sl.start_with_cfl()
        sl.step(6)
        split = sl.ctxs[0].download(nbound=0)
    finally:
        sl.close()
    for a, b in zip(split, whole):
        assert np.array_equal(a, b)
