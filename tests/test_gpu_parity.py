"""GPU parity: the fused CUDA sweeps against the CPU oracle, through the C ABI.

FP64 gate: relative L1 <= 1e-10 per field after 10 steps; in
practice the FP64 path is compiled without FMA contraction and agrees with
the oracle to a few ulp.  Mixed precision: density relative L1 <= 1e-5.
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import NB, grf_state, interior, oracle_first_dt, params_for, rel_l1, sod_state

from hydropad_b200._lib import num_tiles  # noqa: E402

pytestmark = pytest.mark.gpu

FIELDS = ("p", "rho", "vx", "vy", "vz")
FP64_TOL = 1e-10


def _hydro(params, precision="fp64"):
    from hydropad_b200.api import Hydro
    return Hydro(params, precision=precision)


def _copy_scalars(h, s):
    """Give the GPU context the oracle's time scalars."""
    g = h.get_scalars()
    for name in ("dt", "rdtath", "at", "dat", "rat", "ath", "dath", "t", "told", "thalf", "dtold", "atnew",
                 "datnew", "velmax"):
        setattr(g, name, getattr(s, name))
    g.nstep = max(1, s.nstep)
    h.set_scalars(g)


def _assert_fields(gpu, ref, tol, what):
    for name, a, b in zip(FIELDS, gpu, ref):
        e = rel_l1(interior(a), interior(b))
        scale = np.abs(interior(b)).sum()
        if scale == 0:
            assert np.abs(interior(a)).max() == 0.0, f"{what} {name}: expected exact zeros"
            continue
        assert e <= tol, f"{what} {name}: rel L1 {e:.3e} > {tol:.1e}"


@pytest.mark.parametrize("ndirection", [1, 2, 3])
@pytest.mark.parametrize("case", ["sod", "grf"])
def test_single_sweep_fp64(oracle, ndirection, case):
    n = 16
    if case == "sod":
        state = sod_state(n, axis=ndirection - 1)
        prm = params_for((n, n, n))
    else:
        state = grf_state(n, seed=11)
        prm = params_for((n, n, n), cosmo=True)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.ppmsolver(ndirection)
        out = h.download()
    st.ppmsolver(s, ndirection)
    _assert_fields(out, st.f, 1e-13, f"{case} sweep {ndirection}")


@pytest.mark.parametrize("case,n,steps", [("sod", 32, 10), ("grf", 24, 10)])
def test_evolve_fp64(oracle, case, n, steps):
    if case == "sod":
        state = sod_state(n, axis=0)
        prm = params_for((n, n, n))
    else:
        state = grf_state(n, seed=3)
        prm = params_for((n, n, n), cosmo=True)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.evolve(steps, graph=True)
        out = h.download()
        g = h.get_scalars()
    fails = st.evolve(s, steps)
    assert fails == 0
    _assert_fields(out, st.f, FP64_TOL, f"{case} {steps} steps")
    assert abs(g.t - s.t) <= 1e-12 * abs(s.t)
    assert abs(g.dt - s.dt) <= 1e-10 * abs(s.dt)


def test_graph_matches_stream(oracle):
    n = 16
    state = grf_state(n, seed=5)
    prm = params_for((n, n, n), cosmo=True)
    outs = []
    for graph in (False, True):
        with _hydro(prm) as h:
            h.attach_state(*state)
            h.start_with_cfl()
            h.evolve(7, graph=graph)
            outs.append(h.download())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_conservation_fp64():
    """Mass and momentum are conserved to round-off on a periodic grid
    (static background: no expansion drag)."""
    n = 32
    state = grf_state(n, seed=9)
    prm = params_for((n, n, n), cosmo=False)
    with _hydro(prm) as h:
        h.attach_state(*state)
        h.start_with_cfl()
        h.evolve(5, graph=True)
        out = h.download()
    rho0, rho1 = interior(state[1]), interior(out[1])
    m0, m1 = rho0.sum(), rho1.sum()
    assert abs(m1 - m0) <= 1e-12 * m0
    for q in (2, 3, 4):
        mom0 = (rho0 * interior(state[q])).sum()
        mom1 = (rho1 * interior(out[q])).sum()
        assert abs(mom1 - mom0) <= 1e-11 * np.abs(rho0 * interior(state[q])).sum()


def test_drop_in_pointer_check():
    from hydropad_b200._lib import HydroError
    n = 16
    state = sod_state(n)
    prm = params_for((n, n, n))
    with _hydro(prm) as h:
        arrs = h.attach_state(*state)
        h.ppmsolver(1)
        h._host = [a.copy(order="F") for a in arrs]  # different host arrays
        with pytest.raises(HydroError, match="STATE_MISMATCH"):
            h.ppmsolver(2)


def test_mixed_close_to_fp64():
    n = 32
    state = grf_state(n, seed=21)
    prm = params_for((n, n, n), cosmo=True)
    outs = []
    for prec in ("fp64", "mixed"):
        with _hydro(prm, prec) as h:
            h.attach_state(*state)
            h.start_with_cfl()
            h.evolve(10, graph=True)
            outs.append(h.download())
    e = rel_l1(interior(outs[1][1]), interior(outs[0][1]))
    assert e <= 1e-5, e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_tiles_bitwise_identical(prec):
    """Every tile shape computes exactly the same cells (only speed differs)."""
    n = 24
    state = grf_state(n, seed=13)
    prm = params_for((n, n, n), cosmo=True)
    outs = []
    for t in range(num_tiles()):
        with _hydro(prm, prec) as h:
            h.attach_state(*state)
            h.set_tiles(t, t, t)
            h.start_with_cfl()
            h.evolve(3, graph=True)
            outs.append(h.download())
    for t in range(1, num_tiles()):
        for a, b in zip(outs[0], outs[t]):
            assert np.array_equal(a, b), t


def test_autotune_keeps_state():
    n = 32
    state = grf_state(n, seed=17)
    prm = params_for((n, n, n), cosmo=True)
    with _hydro(prm, "mixed") as h:
        h.attach_state(*state)
        before = h.download()
        tiles = h.autotune(reps=1)
        after = h.download()
    assert all(0 <= t < num_tiles() for t in tiles)
    for a, b in zip(before, after):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(24, 16, 20), (16, 32, 12)])
def test_evolve_fp64_non_cubic(oracle, shape):
    """Non-cubic boxes (dx = 1/max(N), the pencils of each axis have their
    own length): 6 steps within the FP64 gate of the oracle."""
    rng = np.random.Generator(np.random.PCG64(31))
    x, y, z = np.meshgrid(*[(np.arange(n) + 0.5) / n for n in shape], indexing="ij")
    rho = 1.0 + 0.4 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.1 * rng.random(shape)
    p = 0.6 + 0.3 * np.cos(2 * np.pi * z) + 0.1 * rng.random(shape)
    vel = [0.3 * np.sin(2 * np.pi * (x + 2 * y + 3 * z + q)) for q in range(3)]
    state = [np.asfortranarray(np.pad(a, NB, mode="wrap")) for a in (p, rho, *vel)]
    prm = params_for(shape)
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.evolve(6, graph=True)
        out = h.download()
    assert st.evolve(s, 6) == 0
    _assert_fields(out, st.f, FP64_TOL, f"non-cubic {shape}")


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_invalid_state_is_reported(prec):
    """A non-physical input (one cell with negative density) is caught by the
    device status word: the step returns an error instead of silently
    producing NaN, and the context stays usable."""
    from hydropad_b200._lib import HydroError
    n = 16
    state = [a.copy(order="F") for a in sod_state(n)]
    state[1][NB + 5, NB + 5, NB + 5] = -0.5
    prm = params_for((n, n, n))
    with _hydro(prm, prec) as h:
        s0 = h.get_scalars()
        h.attach_state(*state)
        h.start_with_cfl()
        with pytest.raises(HydroError, match="NAN|NEGATIVE"):
            h.evolve(1)
        # the context still runs a valid state once its clock is reset
        h.attach_state(*sod_state(n))
        h.set_scalars(s0)
        h.start_with_cfl()
        h.evolve(2)
        again = h.download()
    with _hydro(prm, prec) as h:
        h.attach_state(*sod_state(n))
        h.start_with_cfl()
        h.evolve(2)
        fresh = h.download()
    for a, b in zip(again, fresh):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(16, 16, 16), (24, 16, 20)])
def test_host_transfers_round_trip(shape):
    """attach_state / download / sync_to_host move whole ghosted planes
    through a device staging buffer: the interior comes back unchanged and
    the ghost layers hold the periodic copies (exchange_mesh for one rank)."""
    rng = np.random.Generator(np.random.PCG64(5))
    arrs = [np.asfortranarray(np.pad(1.0 + rng.random(shape), NB, mode="wrap")) for _ in range(5)]
    for a in arrs:  # junk in the ghosts: they must not be read
        a[:NB] = -7.0
    with _hydro(params_for(shape)) as h:
        host = h.attach_state(*arrs)
        out = h.download()
        synced = h.sync_to_host()
        dense = h.download(nbound=0)
    for a, o, s_, d in zip(arrs, out, synced, dense):
        inner = interior(a)
        assert np.array_equal(interior(o), inner)
        assert np.array_equal(o, np.pad(inner, NB, mode="wrap"))
        assert np.array_equal(s_, o)
        assert np.array_equal(d, inner)
    assert all(s_ is hh for s_, hh in zip(synced, host))


def test_config1_sod64(oracle):
    """The Sod configuration at its full size: 64^3, cour 0.8, 100 steps
    with the reference's nrot schedule, against the oracle after 10 and
    after 100 steps (the FP64 gate both times)."""
    n = 64
    state = sod_state(n, axis=0)
    prm = params_for((n, n, n))
    st = oracle.OracleState(*state)
    s = oracle.make_scalars(prm)
    oracle_first_dt(oracle, st, s)
    with _hydro(prm) as h:
        h.attach_state(*state)
        _copy_scalars(h, s)
        h.evolve(10, graph=True)
        out10 = h.download()
        h.evolve(90, graph=True)
        out100 = h.download()
        g = h.get_scalars()
    assert st.evolve(s, 10) == 0
    _assert_fields(out10, st.f, FP64_TOL, "Sod 64^3, 10 steps")
    assert st.evolve(s, 90) == 0
    _assert_fields(out100, st.f, FP64_TOL, "Sod 64^3, 100 steps")
    assert abs(g.t - s.t) <= 1e-12 * s.t


def test_config2_eds256_fp64_ten_steps(oracle):
    """The cosmological configuration at its full size (256^3): ten steps of
    the FP64 path against the oracle at the FP64 gate (1e-10 per field)."""
    n = 256
    state = grf_state(n, seed=12345)
    prm = params_for((n, n, n), cosmo=True)
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
    _assert_fields(out, st.f, FP64_TOL, "EdS 256^3, 10 steps")
    assert abs(g.t - s.t) <= 1e-12 * abs(s.t)


def test_config2_eds256_runs_to_z10():
    """The cosmological configuration runs from z = 50 to z = 10 (tstop,
    initialize_parameters.F90:85) and stops there: the step count and the
    final expansion factor of the FP64 and mixed paths."""
    n = 256
    state = grf_state(n, seed=12345)
    prm = params_for((n, n, n), cosmo=True)
    steps = {}
    for prec in ("fp64", "mixed"):
        with _hydro(prm, prec) as h:
            h.attach_state(*state)
            h.start_with_cfl()
            done = 0
            while done < 200:
                h.evolve(1, graph=True)
                done += 1
                g = h.get_scalars()
                if not g.told < prm.tstop:
                    break
            a_end = g.t ** (2.0 / 3.0)
            steps[prec] = g.nstep - 1
        assert abs(a_end - 1.0 / 11.0) <= 1e-9, (prec, a_end)
    assert all(50 <= v <= 200 for v in steps.values()), steps
    print(f"steps from z=50 to z=10 at 256^3: {steps}")
