"""Pin the C oracle against the golden vectors of the independent Python
restatement (tests/golden/gen_golden.py): one sweep per case, bit-exact --
the STENCIL sweep, and the non-STENCIL build's full-pencil solver for the
pencil_* cases."""
import glob
import os

import numpy as np
import pytest

from hydropad_b200.params import HydroParams

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def golden_cases():
    return [os.path.basename(p)[:-4] for p in GOLDEN]


def load_case(name):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    inp = [np.asfortranarray(a) for a in z["inp"]]
    out = [np.asfortranarray(a) for a in z["out"]]
    return z, inp, out


def oracle_scalars(oracle, z):
    shape = tuple(int(v) for v in z["shape"])
    prm = HydroParams(shape=shape, dmax=float(z["dmax"]))
    s = oracle.make_scalars(prm)
    s.dt = float(z["dt"])
    s.at = float(z["at"])
    s.dat = float(z["dat"])
    s.rat = 1.0 / s.at
    s.ath = float(z["ath"])
    s.rdtath = s.dt / s.ath
    return s


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_golden(oracle, name):
    z, inp, out = load_case(name)
    st = oracle.OracleState(*inp, gforce=z["gforce"] if "gforce" in z.files else None,
                            cho=z["cho"] if "cho" in z.files else None)
    s = oracle_scalars(oracle, z)
    if name.startswith("pencil"):  # the non-STENCIL build's full-pencil solver
        assert st.ppmsolver_pencil(s, int(z["nd"])) == 0
    else:
        assert st.ppmsolver(s, int(z["nd"])) == 0
    for q in range(5):
        a, b = st.f[q], out[q]
        assert np.array_equal(a, b), (name, q, np.abs(a - b).max())


def test_golden_set_present():
    assert len(GOLDEN) >= 18, "run tests/golden/gen_golden.py"


def test_pencil_peak_case_exercises_the_peaks():
    """pencil_peak_x must reach the full-pencil solver's density-peak paths:
    a cell above dmax x both x neighbours (pmean with cho3d) and a face
    window with rho(2) > dmax rho(1), rho(3) > dmax rho(4) (the fix)."""
    z, inp, _ = load_case("pencil_peak_x")
    r, dmax, cho = inp[1], float(z["dmax"]), z["cho"]
    cell = (r[1:-1] > dmax * r[:-2]) & (r[1:-1] > dmax * r[2:])
    assert cell.any() and np.isin(cho[1:-1][cell], (1.0, 2.0)).any()
    face = (r[1:-2] > dmax * r[:-3]) & (r[2:-1] > dmax * r[3:])
    assert face.any()


def test_gravity_cases_have_a_source():
    for name in ("grav_x", "grav_y", "grav_z"):
        z, _, _ = load_case(name)
        assert np.abs(z["gforce"]).max() > 0.1


def test_peak_case_exercises_the_fix():
    """The peak_y case must actually trigger the density-peak pressure fix
    (otherwise it would not pin the transposed gather)."""
    z, inp, _ = load_case("peak_y")
    rho = inp[1]
    dmax = float(z["dmax"])
    # some x-row quadruple with rho(2) > dmax rho(1) and rho(3) > dmax rho(4)
    r = rho
    hit = (r[1:-2] > dmax * r[:-3]) & (r[2:-1] > dmax * r[3:])
    assert hit.any()


@pytest.mark.parametrize("name", ["extreme_x", "extreme_y", "extreme_z"])
def test_extreme_cases_reach_every_pattern(name):
    """The extreme cases must pin the oracle on every wave pattern of
    riemannsolver.F90 (two shocks, shock + rarefaction, two rarefactions,
    vacuum), strong shocks included: the generator's tally of the faces."""
    z, _, out = load_case(name)
    two_shocks, shock_rare, two_rare, vacuum, strong_2s, strong_sr = (int(v) for v in z["patterns"])
    assert min(two_shocks, shock_rare, two_rare, vacuum) > 0, z["patterns"]
    assert strong_2s > 0 and strong_sr > 0, z["patterns"]
    assert all(np.isfinite(a).all() for a in out)


@pytest.mark.parametrize("name", ["cold_x", "cold_z"])
def test_cold_cases_reach_every_dual_energy_branch(name):
    """The cold cases must pin the oracle on every branch of the dual-energy
    switch of integrate.F90: internal energy replaced by total minus kinetic,
    pressure from total minus kinetic, pressure from the advected internal
    energy (the generator's tally of the cells)."""
    z, _, out = load_case(name)
    assert all(int(v) > 0 for v in z["dual"]), z["dual"]
    assert all(np.isfinite(a).all() for a in out)
