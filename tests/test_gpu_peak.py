"""GPU parity of the STENCIL density-peak fix (riemannsolver.F90:279-285)
against the oracle, through the C ABI.

The fix raises a face's star pressure when the four densities around it
form a peak above dmax times both outer ones.  The x sweep reads them from
its own pencil; the y and z sweeps gather them with the x-index slot of the
reference's ghosted arrays (ppmsolver.F90:244-256, 372-384: rho3d(iaux,j,k)
with j, k the other two indices), which a pre-pass evaluates on the
pre-sweep state.  On a non-cubic box that gather runs past the end of a row
(or plane) of the ghosted array into the next one, so the non-cubic cases
pin the linear-index form of the gather.

The states carry two-cell density spikes (x40) every fifth cell along x,
where the transposed gathers of all three sweeps read, with dmax = 1.5; each
single-sweep case first checks that the fix acts (the oracle's result
differs from the same sweep at the namelist dmax of 2e10).  Tolerances: the
single-sweep and 10-step gates of the other parity tests.
"""
import numpy as np
import pytest

from tests.helpers import NB, oracle_first_dt, params_for
from tests.test_gpu_parity import FP64_TOL, _assert_fields, _copy_scalars, _hydro

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16, 16), (16, 24, 20), (24, 16, 20)]


def spiky_state(shape, seed, spike=40.0, vrms=0.6):
    """Smooth density and pressure with noise, two-cell density spikes along
    x (cells 3, 4 of every 5), random velocities; periodic ghosts."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = np.linspace(0, 2 * np.pi, shape[0], endpoint=False)[:, None, None]
    rho = 1.0 + 0.4 * np.sin(x) * np.ones(shape) + 0.3 * rng.random(shape)
    p = 0.8 + 0.5 * np.cos(x) * np.ones(shape) + 0.3 * rng.random(shape)
    rho[3::5, :, :] *= spike
    rho[4::5, :, :] *= spike
    vel = [vrms * rng.standard_normal(shape) for _ in range(3)]
    return [np.asfortranarray(np.pad(a, NB, mode="wrap")) for a in (p, rho, *vel)]


def _oracle_sweep(oracle, state, prm, nd):
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    assert st.ppmsolver(s, nd) == 0
    return st, s


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("ndirection", [1, 2, 3])
def test_peak_fix_single_sweep(oracle, shape, ndirection):
    state = spiky_state(shape, seed=40 + ndirection)
    prm = params_for(shape, dmax=1.5)
    ref, _ = _oracle_sweep(oracle, state, prm, ndirection)
    plain, _ = _oracle_sweep(oracle, state, params_for(shape), ndirection)
    assert any(not np.array_equal(a, b) for a, b in zip(ref.f, plain.f)), "the peak fix never acted"
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.ppmsolver(ndirection)
        out = h.download()
    _assert_fields(out, ref.f, 1e-13, f"peak sweep {ndirection} {shape}")


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("cosmo", [False, True])
def test_peak_fix_ten_steps(oracle, shape, cosmo):
    # milder spikes: ten steps of the x40 state end in vacuum cells
    state = spiky_state(shape, seed=50, spike=5.0, vrms=0.3)
    prm = params_for(shape, cosmo=cosmo, dmax=1.5)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.evolve(10, graph=True)
        out = h.download()
        g = h.get_scalars()
    assert st.evolve(s, 10) == 0
    _assert_fields(out, st.f, FP64_TOL, f"peak 10 steps {shape} cosmo={cosmo}")
    assert abs(g.t - s.t) <= 1e-12 * abs(s.t)
