"""GPU: the write_var_mpi-compatible dump (raw REAL(4) interiors in Fortran
order, io/write_var_mpi.F90:36-65 with the names of main.F90:125-135)."""
import os

import numpy as np
import pytest

from tests.helpers import grf_state, params_for

pytestmark = pytest.mark.gpu

FILES = (("rho", 1), ("pressure", 0), ("vx", 2), ("vy", 3), ("vz", 4))


@pytest.mark.parametrize("shape", [(24, 24, 24), (16, 20, 24)])
def test_write_var_matches_fortran_real(tmp_path, shape):
    from hydropad_b200 import ics
    from hydropad_b200.api import Hydro
    prm = params_for(shape, cosmo=True)
    state = ics.grf_eds(shape[0], seed=5) if len(set(shape)) == 1 else None
    with Hydro(prm, precision="fp64") as h:
        if state is None:  # non-cubic: any smooth positive state
            x, y, z = np.meshgrid(*[np.arange(n) / n for n in shape], indexing="ij")
            rho = 1.0 + 0.3 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * z)
            p = 1.0 + 0.1 * np.cos(2 * np.pi * y)
            zero = 0.1 * np.sin(2 * np.pi * (x + y + z))
            state = [np.asfortranarray(np.pad(a, 3, mode="wrap")) for a in (p, rho, zero, 0 * zero, -zero)]
        h.attach_state(*state)
        h.start_with_cfl()
        h.evolve(2)
        ref = h.download(nbound=0)
        h.write_var(str(tmp_path))
        h.write_var(str(tmp_path), fp64=True)
    for name, q in FILES:
        raw = np.fromfile(os.path.join(tmp_path, f"{name}.bin"), dtype="<f4")
        assert raw.size == np.prod(shape)
        got = raw.reshape(shape, order="F")
        assert np.array_equal(got.view(np.uint32), ref[q].astype(np.float32).view(np.uint32)), name
        raw64 = np.fromfile(os.path.join(tmp_path, f"{name}.f64.bin"), dtype="<f8").reshape(shape, order="F")
        assert np.array_equal(raw64, ref[q]), name
