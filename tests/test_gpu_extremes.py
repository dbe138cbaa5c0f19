"""GPU parity on strong waves, through the C ABI: strong shocks, vacuum and
near-vacuum faces (all four wave patterns of riemannsolver.F90, and the
Newton iteration of riemann.F90 far from its start value).

The states (tests.helpers.extreme_state, and the golden extreme_* cases of
tests/golden/gen_golden.py) cycle blocks of 3 cells through cold gas
(p ~ 1e-2), dense gas (rho ~ 100) and hot gas (p ~ 1e3), with velocities
flipping between +0.5 and -0.5, about 4 cold sound speeds: streams collide
(strong two-shock faces), recede (vacuum faces) and meet pressure jumps of
1e5.

FP64: the gates of the other parity tests, single sweeps <= 1e-13 and 10
steps <= 1e-10 relative L1 per field against the oracle; the golden cases
also against the second restatement's vectors.  Mixed precision, whose
strong shocks and vacuum faces take the FP64 solvers and the rest the FP32
ones: relative L1 of every field against the FP64 path after 10 steps
<= MIXED_TOL, with a clean status word (evolve raises otherwise).
"""
import numpy as np
import pytest

from tests.helpers import extreme_state, interior, oracle_first_dt, params_for, rel_l1
from tests.test_gpu_parity import FP64_TOL, _assert_fields, _copy_scalars, _hydro
from tests.test_oracle_golden import load_case, oracle_scalars

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
FIELDS = ("p", "rho", "vx", "vy", "vz")


@pytest.mark.parametrize("name", ["extreme_x", "extreme_y", "extreme_z"])
def test_extreme_golden_sweep(oracle, name):
    """One sweep of the golden extreme case (the generator's own time
    scalars) against the second restatement's output."""
    z, inp, out = load_case(name)
    shape = tuple(int(v) for v in z["shape"])
    prm = params_for(shape)
    with _hydro(prm) as h:
        h.attach_state(*[a.copy(order="F") for a in inp])
        _copy_scalars(h, oracle_scalars(oracle, z))
        h.ppmsolver(int(z["nd"]))
        got = h.download()
    _assert_fields(got, out, 1e-13, f"{name} golden")


@pytest.mark.parametrize("shape", [(16, 16, 16), (18, 12, 24)])
@pytest.mark.parametrize("ndirection", [1, 2, 3])
def test_extreme_single_sweep_fp64(oracle, shape, ndirection):
    state = extreme_state(shape, seed=60 + ndirection)
    prm = params_for(shape)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.ppmsolver(ndirection)
        out = h.download()
    assert st.ppmsolver(s, ndirection) == 0
    _assert_fields(out, st.f, 1e-13, f"extreme {shape} sweep {ndirection}")


@pytest.mark.parametrize("cosmo", [False, True])
def test_extreme_evolve_fp64(oracle, cosmo):
    shape = (16, 16, 16)
    state = extreme_state(shape, seed=5)
    prm = params_for(shape, cosmo=cosmo)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.evolve(10, graph=True)
        out = h.download()
    assert st.evolve(s, 10) == 0
    _assert_fields(out, st.f, FP64_TOL, f"extreme cosmo={cosmo} 10 steps")


@pytest.mark.parametrize("cosmo", [False, True])
def test_extreme_mixed_close_to_fp64(cosmo):
    shape = (16, 16, 16)
    state = extreme_state(shape, seed=5)
    prm = params_for(shape, cosmo=cosmo)
    outs = []
    for prec in ("fp64", "mixed"):
        with _hydro(prm, prec) as h:
            h.attach_state(*[a.copy(order="F") for a in state])
            h.start_with_cfl()
            h.evolve(10, graph=True)
            outs.append(h.download())
    for name, a, b in zip(FIELDS, outs[1], outs[0]):
        assert np.isfinite(interior(a)).all(), name
        e = rel_l1(interior(a), interior(b))
        assert e <= MIXED_TOL, f"mixed {name}: rel L1 {e:.3e} against FP64"
