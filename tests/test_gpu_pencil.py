"""GPU parity of the non-STENCIL build's full-pencil solver (hydro/ppm.F90,
called per pencil by the #else branches of ppmsolver.F90) against the
oracle's restatement of it, through the C ABI.

The solver differs from the STENCIL sweep in four places (sound speed of
the next cell in the characteristic speeds, the density-peak window along
the sweep, cho3d at density peaks, the 3-cell dual-energy switch); the
cases below make each of them act: a non-isothermal state for the sound
speed, a low dmax with a cho3d field for the peaks, Sod shocks for the
dual-energy switch.  Tolerances as for the STENCIL sweeps: 1e-13 relative
L1 per field for one sweep, 1e-10 after 10 steps.
"""
import numpy as np
import pytest

from tests.helpers import grf_state, interior, oracle_first_dt, params_for, rel_l1, sod_state
from tests.test_gpu_parity import FP64_TOL, _assert_fields, _copy_scalars, _hydro

from hydropad_b200._lib import num_tiles  # noqa: E402

pytestmark = pytest.mark.gpu


def _warm_grf(oracle, n, seed):
    """The GRF state with a pressure that varies by up to 50 % from cell to
    cell (a sound speed that varies), ghosts refilled periodically."""
    st = oracle.OracleState(*grf_state(n, seed=seed))
    rng = np.random.default_rng(seed)
    st.f[0][...] *= 1.0 + 0.5 * rng.random(st.f[0].shape)
    st.exchange()
    return [a.copy(order="F") for a in st.f]


def _case(oracle, case, n, axis=0, **kw):
    if case == "sod":
        return sod_state(n, axis=axis), params_for((n, n, n), **kw)
    if case == "grf_static":  # the GRF in a static box: dt from the CFL condition
        return grf_state(n, seed=4), params_for((n, n, n), **kw)
    return _warm_grf(oracle, n, 21 + axis), params_for((n, n, n), cosmo=True, **kw)


@pytest.mark.parametrize("ndirection", [1, 2, 3])
@pytest.mark.parametrize("case", ["sod", "grf"])
def test_single_pencil_sweep(oracle, ndirection, case):
    n = 16
    state, prm = _case(oracle, case, n, axis=ndirection - 1)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.ppmsolver_pencil(ndirection)
        out = h.download()
    st.ppmsolver_pencil(s, ndirection)
    _assert_fields(out, st.f, 1e-13, f"{case} pencil sweep {ndirection}")


def test_pencil_differs_from_stencil(oracle):
    """With a varying sound speed the two builds' sweeps differ (the check
    that the variant is the one that ran)."""
    n = 16
    state, prm = _case(oracle, "grf", n)
    outs = []
    for variant in ("stencil", "pencil"):
        with _hydro(prm) as h:
            h.attach_state(*state)
            h.set_variant(variant)
            assert h.get_variant() == variant
            h.start_with_cfl()
            h.evolve(2)
            outs.append(h.download())
    assert rel_l1(interior(outs[0][0]), interior(outs[1][0])) > 1e-8


@pytest.mark.parametrize("case,n,steps,cour,zero_old", [("sod", 32, 10, 0.8, False), ("grf", 24, 10, 0.8, False),
                                                        ("grf", 24, 10, 0.8, True), ("grf_static", 12, 4, 0.8, False)])
def test_evolve_pencil(oracle, case, n, steps, cour, zero_old):
    """The static GRF box at Courant number 0.8 also runs the density
    fallback of the solver's update (ppm.F90:651) in a few cells, which the
    solver's characteristic speeds (the next cell's sound speed) reach
    there.  zero_old: expand with the non-STENCIL build's vxold / pold3d,
    allocated as zeros and never assigned (alloc_arrays.F90:132-133)."""
    state, prm = _case(oracle, case, n, cour=cour, expand_zero_old=zero_old)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    s.pencil = 1
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        h.set_variant("pencil")
        _copy_scalars(h, s)
        h.evolve(steps, graph=True)
        out = h.download()
        g = h.get_scalars()
    assert st.evolve(s, steps) == 0
    _assert_fields(out, st.f, FP64_TOL, f"{case} pencil {steps} steps")
    assert abs(g.t - s.t) <= 1e-12 * abs(s.t)


@pytest.mark.parametrize("ndirection", [1, 2, 3])
def test_pencil_density_peaks_with_cho(oracle, ndirection):
    """dmax low enough that the peak fix and the cho3d cases of pmean act;
    cho3d = 0, 1, 2 at random."""
    n = 16
    state, prm = _case(oracle, "grf", n, axis=ndirection - 1, dmax=1.3)
    # density noise of up to 60 %: isolated peaks above dmax x both neighbours
    st0 = oracle.OracleState(*state)
    st0.f[1][...] *= 1.0 + 0.6 * np.random.default_rng(9).random(st0.f[1].shape)
    st0.exchange()
    state = [a.copy(order="F") for a in st0.f]
    rng = np.random.default_rng(5)
    cho = oracle.OracleState(*[rng.integers(0, 3, state[0].shape).astype(np.float64)] * 5)
    cho.exchange()
    cho = cho.f[0].copy(order="F")
    outs = []
    for with_cho in (True, False):
        st = oracle.OracleState(*state, cho=cho if with_cho else None)
        s = oracle.make_scalars(prm)
        oracle_first_dt(oracle, st, s)
        with _hydro(prm) as h:
            h.attach_state(*state)
            if with_cho:
                h.attach_cho(cho)
            _copy_scalars(h, s)
            h.ppmsolver_pencil(ndirection)
            out = h.download()
        st.ppmsolver_pencil(s, ndirection)
        _assert_fields(out, st.f, 1e-13, f"peaks cho={with_cho} sweep {ndirection}")
        outs.append(out)
    assert any(not np.array_equal(a, b) for a, b in zip(*outs)), "cho3d never acted"


def test_pencil_tiles_bitwise_identical(oracle):
    n = 20
    state, prm = _case(oracle, "grf", n)
    outs = []
    for t in range(num_tiles()):
        with _hydro(prm) as h:
            h.attach_state(*state)
            h.set_variant("pencil")
            h.set_tiles(t, t, t)
            h.start_with_cfl()
            h.evolve(3, graph=True)
            outs.append(h.download())
    for t in range(1, num_tiles()):
        for a, b in zip(outs[0], outs[t]):
            assert np.array_equal(a, b), t


def test_pencil_rejections():
    from hydropad_b200._lib import HydroError
    from hydropad_b200.batch import Batch
    n = 16
    prm = params_for((n, n, n))
    with _hydro(prm, "mixed") as h:
        with pytest.raises(HydroError, match="UNSUPPORTED"):
            h.set_variant("pencil")
    with _hydro(prm) as h:
        h.attach_state(*sod_state(n))
        h.set_variant("pencil")
        with Batch("fp64", capacity=1) as b:
            with pytest.raises(HydroError, match="ARG"):
                b.add(h)
        h.set_variant("stencil")
        h.ppmsolver(1)
