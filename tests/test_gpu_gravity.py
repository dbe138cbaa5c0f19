"""GPU parity with the static gravity source (the reference's -DGRAVITY
build: gforce from initialize_gravity.F90, the g parabola in the tracing of
order2interp.F90:170-172 and the source terms of integrate.F90:41-57),
against the oracle, through the C ABI."""
import numpy as np
import pytest

from hydropad_b200 import ics
from tests.helpers import NB, grf_state, interior, oracle_first_dt, params_for, rel_l1, sod_state
from tests.test_gpu_parity import FP64_TOL, _assert_fields, _copy_scalars, _hydro

from hydropad_b200._lib import num_tiles  # noqa: E402

pytestmark = pytest.mark.gpu

# the reference's potential (alpha = 1) gives gforce ~ 1e-2 at 16^3; scale
# it up so that the source terms move the flow visibly in a few steps
ALPHA = 40.0


def _gforce(n, alpha=ALPHA):
    return ics.static_gravity(n, nb=NB, alpha=alpha)


@pytest.mark.parametrize("ndirection", [1, 2, 3])
@pytest.mark.parametrize("case", ["sod", "grf"])
def test_single_sweep_gravity_fp64(oracle, ndirection, case):
    n = 16
    if case == "sod":
        state = sod_state(n, axis=ndirection - 1)
        prm = params_for((n, n, n))
    else:
        state = grf_state(n, seed=12)
        prm = params_for((n, n, n), cosmo=True)
    g = _gforce(n)
    st = oracle.OracleState(*state, gforce=g)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state, gforce=g)
        _copy_scalars(h, s)
        h.ppmsolver(ndirection)
        out = h.download()
    st.ppmsolver(s, ndirection)
    _assert_fields(out, st.f, 1e-13, f"{case} gravity sweep {ndirection}")


@pytest.mark.parametrize("case,n,steps", [("sod", 24, 10), ("grf", 20, 10)])
def test_evolve_gravity_fp64(oracle, case, n, steps):
    if case == "sod":
        state = sod_state(n, axis=1)
        prm = params_for((n, n, n))
    else:
        state = grf_state(n, seed=4)
        prm = params_for((n, n, n), cosmo=True)
    g = _gforce(n)
    st = oracle.OracleState(*state, gforce=g)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state, gforce=g)
        _copy_scalars(h, s)
        h.evolve(steps, graph=True)
        out = h.download()
    assert st.evolve(s, steps) == 0
    _assert_fields(out, st.f, FP64_TOL, f"{case} gravity {steps} steps")
    # the source acted: the run differs from the gravity-free one
    st0 = oracle.OracleState(*state)
    s0 = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st0, s0)
    st0.evolve(s0, steps)
    assert rel_l1(interior(st.f[1]), interior(st0.f[1])) > 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gravity_tiles_bitwise_identical(prec):
    n = 20
    state = grf_state(n, seed=14)
    prm = params_for((n, n, n), cosmo=True)
    g = _gforce(n)
    outs = []
    for t in range(num_tiles()):
        with _hydro(prm, prec) as h:
            h.attach_state(*state, gforce=g)
            h.set_tiles(t, t, t)
            h.start_with_cfl()
            h.evolve(3, graph=True)
            outs.append(h.download())
    for t in range(1, num_tiles()):
        for a, b in zip(outs[0], outs[t]):
            assert np.array_equal(a, b), t


def test_gravity_mixed_close_to_fp64():
    # the reference's amplitude: at 40x this cold box runs into NaN within
    # 7 steps in the oracle too
    n = 32
    state = grf_state(n, seed=22)
    prm = params_for((n, n, n), cosmo=True)
    g = _gforce(n, alpha=1.0)
    outs = []
    for prec in ("fp64", "mixed"):
        with _hydro(prm, prec) as h:
            h.attach_state(*state, gforce=g)
            h.start_with_cfl()
            h.evolve(10, graph=True)
            outs.append(h.download())
    assert rel_l1(interior(outs[1][1]), interior(outs[0][1])) <= 1e-5


def test_gravity_drop_in_and_batch_checks():
    from hydropad_b200._lib import HydroError
    from hydropad_b200.batch import Batch
    n = 16
    state = sod_state(n)
    prm = params_for((n, n, n))
    g = _gforce(n)
    with _hydro(prm) as h:
        h.attach_state(*state, gforce=g)
        h.ppmsolver(1)                       # the attached gforce: accepted
        h._gforce = np.asfortranarray(g.copy())
        with pytest.raises(HydroError, match="STATE_MISMATCH"):
            h.ppmsolver(2)                   # another array: rejected
        with Batch("fp64", capacity=1) as b:
            with pytest.raises(HydroError, match="ARG"):
                b.add(h)                     # batches carry no gravity source
        h.attach_state(*state)               # gravity off again
        h.ppmsolver(2)


def test_device_gforce_matches_host_gforce():
    import torch
    n = 16
    state = grf_state(n, seed=2)
    prm = params_for((n, n, n), cosmo=True)
    g = _gforce(n)
    outs = []
    with _hydro(prm) as h:
        h.attach_state(*state, gforce=g)
        h.start_with_cfl()
        h.evolve(3)
        outs.append(h.download())
    with _hydro(prm) as h:
        h.attach_state(*state)
        comps = [torch.from_numpy(np.ascontiguousarray(interior(g[d]).transpose(2, 1, 0))).cuda() for d in range(3)]
        h.attach_device_gforce(*comps)
        h.start_with_cfl()
        h.evolve(3)
        outs.append(h.download())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
