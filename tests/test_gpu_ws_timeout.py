"""Failure detection of the pipelined sweep (ppm_sweep_ws_kernel): its waits
on mbarriers are bounded.

A test-only environment switch (HP_TEST_WITHHOLD_NEWTON=1, read by the
launcher) makes the Newton warp of every CTA withhold the completion of its
first window.  The main warps' wait for it then runs out after its time
limit (2 s): the kernel ends through its abort flag (the other role's waits
see it), the status word says HP_ERR_TIMEOUT, and the context keeps working
-- a fresh attach and sweep give the same bits as a new context.  Nothing
faults or hangs: every wait involved is the bounded one.
"""
import time

import numpy as np
import pytest

from tests.helpers import grf_state, params_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ndirection", [1, 2])
def test_withheld_completion_times_out_and_context_recovers(monkeypatch, ndirection):
    from hydropad_b200._lib import HydroError
    from hydropad_b200.api import Hydro

    n = 32
    state = grf_state(n, seed=3)
    prm = params_for((n, n, n), cosmo=True)
    with Hydro(prm) as h:
        h.attach_state(*state)
        h.set_tiles(11, 11, 11)
        h.start_with_cfl()
        s0 = h.get_scalars()
        monkeypatch.setenv("HP_TEST_WITHHOLD_NEWTON", "1")
        t0 = time.time()
        with pytest.raises(HydroError, match="TIMEOUT"):
            h.ppmsolver(ndirection)
        assert time.time() - t0 < 60
        monkeypatch.delenv("HP_TEST_WITHHOLD_NEWTON")
        h.attach_state(*state)
        h.set_scalars(s0)
        h.ppmsolver(ndirection)
        again = h.download()
    with Hydro(prm) as h:
        h.attach_state(*state)
        h.set_tiles(11, 11, 11)
        h.start_with_cfl()
        h.ppmsolver(ndirection)
        fresh = h.download()
    for a, b in zip(again, fresh):
        assert np.array_equal(a, b)
