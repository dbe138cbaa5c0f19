"""Physics pins of the CPU oracle (the reference ships no test vectors):
exact Sod solution, conservation on periodic grids, axis symmetry and
invariance of a uniform state."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import NB, grf_state, interior, oracle_first_dt, params_for, sod_state
from tests.sod_exact import sample

GAMMA = 5.0 / 3.0


def _run(oracle, state, prm, steps):
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    fails = st.evolve(s, steps)
    assert fails == 0
    return st, s


def test_sod_exact_solution(oracle):
    """Until the two Sod interfaces of the periodic box interact (t < 0.14),
    each is an isolated Riemann problem with a known exact solution."""
    n = 256
    st, s = _run(oracle, sod_state((n, 2, 2), axis=0), params_for((n, 2, 2)), 60)
    t = s.told
    assert 0.04 < t < 0.13, t
    x = (np.arange(n) + 0.5) / n
    # interface at x=0.5 (left state on the left) and its mirror at x=0/1
    ex = np.empty((n, 3))
    mid = (x >= 0.25) & (x < 0.75)
    ex[mid] = sample((x[mid] - 0.5) / t, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, GAMMA)
    # mirrored interface at x=0 (=1): low-density state on its left
    d = np.where(x < 0.25, x, x - 1.0)
    ex[~mid] = sample(d[~mid] / t, 0.125, 0.0, 0.1, 1.0, 0.0, 1.0, GAMMA)
    rho = interior(st.rho)[:, 0, 0]
    l1 = np.abs(rho - ex[:, 0]).mean()
    assert l1 < 0.01, l1
    assert np.abs(rho - ex[:, 0]).max() < 0.35  # only at discontinuities


def test_conservation_periodic(oracle):
    n = 12
    state = grf_state(n, seed=4)
    st, s = _run(oracle, state, params_for((n, n, n)), 4)
    r0, r1 = interior(state[1]), interior(st.rho)
    assert abs(r1.sum() - r0.sum()) <= 1e-12 * r0.sum()
    for q in (2, 3, 4):
        m0 = (r0 * interior(state[q])).sum()
        m1 = (r1 * interior(st.f[q])).sum()
        assert abs(m1 - m0) <= 1e-11 * np.abs(r0 * interior(state[q])).sum()


ORDERS = {1: (1, 2, 3), 2: (3, 2, 1), 3: (2, 3, 1), 4: (1, 3, 2), 5: (3, 1, 2), 6: (2, 1, 3)}


def _run_relabelled(oracle, state, prm, steps, relabel):
    """evolve_sys with the nrot sweep order relabelled by `relabel`
    (direction -> direction), so a tube along another axis sees the same
    sequence of normal/transverse sweeps."""
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    for _ in range(steps):
        s.nstep += 1
        nrot = 1 if s.nstep == 1 else s.nstep % 6 + 1
        for d in ORDERS[nrot]:
            assert st.ppmsolver(s, relabel[d]) == 0
            st.exchange()
        s.velmax = st.speed(s)
        oracle.lib().hpo_timedet(C.byref(s))
    return st


@pytest.mark.parametrize("axis", [1, 2])
def test_axis_symmetry(oracle, axis):
    """A Sod tube along y or z, swept in the relabelled order, evolves
    bit-identically to the tube along x (transverse sweeps round p at the
    ulp level, so the order of sweeps matters bit-wise)."""
    n = 16
    prm = params_for((n, n, n))
    ident = {1: 1, 2: 2, 3: 3}
    relabel = {1: {1: 2, 2: 1, 3: 3}, 2: {1: 3, 2: 2, 3: 1}}[axis]
    sx = _run_relabelled(oracle, sod_state(n, axis=0), prm, 6, ident)
    sa = _run_relabelled(oracle, sod_state(n, axis=axis), prm, 6, relabel)
    perm = {1: (1, 0, 2), 2: (2, 1, 0)}[axis]
    vel = {1: (3, 2, 4), 2: (4, 3, 2)}[axis]  # normal velocity moves with the axis
    for q_x, q_a in ((0, 0), (1, 1), (2, vel[0]), (3, vel[1]), (4, vel[2])):
        a = np.transpose(interior(sa.f[q_a]), perm)
        assert np.array_equal(interior(sx.f[q_x]), a), (q_x, q_a)


def test_uniform_state_is_steady(oracle):
    n = 10
    shape = (n + 2 * NB,) * 3
    one = np.ones(shape, order="F")
    z = np.zeros(shape, order="F")
    state = (0.6 * one, 1.3 * one, 0.2 * one, -0.1 * one, 0.05 * one)
    st, s = _run(oracle, state, params_for((n, n, n)), 3)
    for q in range(5):
        assert np.array_equal(interior(st.f[q]), interior(state[q])), q
    del z


def test_newton_cap_reported(oracle):
    """The reference stops after 100 Newton iterations; the oracle reports
    the failure count instead (never silently)."""
    n = 8
    state = sod_state(n)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(params_for((n, n, n)))
    oracle_first_dt(oracle, st, s)
    assert st.ppmsolver(s, 1) == 0


# ---- the non-STENCIL build's full-pencil solver (hydro/ppm.F90) ----------

def _pencil_run(oracle, state, prm, steps):
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    s.pencil = 1
    oracle_first_dt(oracle, st, s)
    assert st.evolve(s, steps) == 0
    return st, s


def test_pencil_uniform_state_is_steady(oracle):
    n = 10
    shape = (n + 2 * NB,) * 3
    one = np.ones(shape, order="F")
    state = (0.6 * one, 1.3 * one, 0.2 * one, -0.1 * one, 0.05 * one)
    st, _ = _pencil_run(oracle, state, params_for((n, n, n)), 3)
    for q in range(5):
        assert np.array_equal(interior(st.f[q]), interior(state[q])), q


def test_pencil_conservation_periodic(oracle):
    """Mass and momentum to round-off, at Courant number 0.3: on this rough
    field the full-pencil solver's characteristic speeds (the next cell's
    sound speed) drive a few densities negative from 0.5 up, and the
    reference's fallback (keep the old density, ppm.F90:651) then does not
    conserve mass; the STENCIL sweep stays positive at 0.8."""
    n = 12
    state = grf_state(n, seed=4)
    st, _ = _pencil_run(oracle, state, params_for((n, n, n), cour=0.3), 4)
    r0, r1 = interior(state[1]), interior(st.rho)
    assert abs(r1.sum() - r0.sum()) <= 1e-12 * r0.sum()
    for q in (2, 3, 4):
        m0 = (r0 * interior(state[q])).sum()
        m1 = (r1 * interior(st.f[q])).sum()
        assert abs(m1 - m0) <= 1e-11 * np.abs(r0 * interior(state[q])).sum()


def test_pencil_sound_speed_of_next_cell(oracle):
    """The only tracing difference from the STENCIL sweep is the sound speed
    of the characteristic speeds (cell k takes cell k+1's, ppm.F90:106-107):
    with a uniform sound speed (the isothermal GRF) and no density peak the
    two sweeps give the same bits; with a varying one they differ."""
    n = 12
    state = grf_state(n, seed=8)
    prm = params_for((n, n, n), cosmo=True)
    outs = []
    for pencil in (False, True):
        st = oracle.OracleState(*state)
        s = oracle.make_scalars(prm)
        oracle_first_dt(oracle, st, s)
        (st.ppmsolver_pencil if pencil else st.ppmsolver)(s, 1)
        outs.append([interior(a).copy() for a in st.f])
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
    warm = oracle.OracleState(*state)
    warm.f[0][...] *= 1.0 + 0.5 * np.random.default_rng(3).random(warm.f[0].shape)
    warm.exchange()
    outs = []
    for pencil in (False, True):
        st = oracle.OracleState(*warm.f)
        s = oracle.make_scalars(prm)
        oracle_first_dt(oracle, st, s)
        (st.ppmsolver_pencil if pencil else st.ppmsolver)(s, 1)
        outs.append(interior(st.f[1]).copy())
    assert not np.array_equal(outs[0], outs[1])
