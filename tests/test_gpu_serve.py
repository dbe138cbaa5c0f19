"""GPU: the serving path against requests run alone, and the GPU initial
conditions against the host generator."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILES = (1, 1, 1)


@pytest.mark.parametrize("pool", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_serving_matches_alone(precision, pool):
    """Requests of different sizes and step counts, arriving while others
    run (members join and leave the batch at different nrot): every
    response is bitwise the request run alone through hp_evolve -- also
    when finished contexts are kept and reused for later requests."""
    from hydropad_b200.serve import GpuEngine, Request, Scheduler, box_bytes, run_alone
    reqs = [Request(0, 0.0, 32, 14, 101), Request(1, 0.0, 48, 9, 102), Request(2, 0.0, 32, 21, 103),
            Request(3, 0.0, 16 * 3, 6, 104), Request(4, 0.0, 32, 11, 105)]
    eng = GpuEngine(precision, capacity=3, tiles=TILES, graph=True,
                    pool_bytes=10 * box_bytes(48, precision) if pool else 0)
    try:
        # room for about two boxes: later requests wait and join mid-run
        sched = Scheduler(eng, budget_bytes=box_bytes(48, precision) + box_bytes(32, precision), capacity=3,
                          chunk=4, keep_results=True)
        eng.start_clock()
        st = sched.run(reqs)
        reused = eng.reused
    finally:
        eng.close()
    if pool:
        assert reused > 0
    assert sorted(c.rid for c in st.completed) == [r.rid for r in reqs]
    assert st.admission_stalls > 0
    for c in st.completed:
        ref = run_alone(reqs[c.rid], precision, tiles=TILES)
        for q, (a, b) in enumerate(zip(c.result, ref)):
            assert np.array_equal(a, b), f"request {c.rid} field {q}: max |d| {np.abs(a - b).max():.3e}"


def test_device_ics_match_host():
    from hydropad_b200 import ics
    n = 32
    host = ics.grf_eds(n, seed=9, spectral_index=-1.7, nb=0)
    dev = ics.grf_eds_device(n, seed=9, spectral_index=-1.7, device="cuda")
    for a, d in zip(host, dev):
        d = d.cpu().numpy().transpose(2, 1, 0)
        assert np.abs(a - d).max() <= 1e-12 * np.abs(a).max()


def test_attach_device_state_roundtrip():
    from hydropad_b200 import ics
    from hydropad_b200.api import Hydro
    from hydropad_b200.params import HydroParams
    n = 24
    dev = ics.grf_eds_device(n, seed=4, device="cuda")
    with Hydro(HydroParams(shape=(n, n, n), cosmo=True), precision="fp64") as h:
        h.attach_device(*dev)
        out = h.download(nbound=0)
    for a, d in zip(out, dev):
        assert np.array_equal(a, d.cpu().numpy().transpose(2, 1, 0))


def test_download_into_pinned_buffers():
    """The serving engine reads finished boxes back into pinned host arrays
    (download(out=...)): the same bits as a download into new arrays, with
    and without ghosts; arrays of another shape or order are refused."""
    from hydropad_b200 import ics
    from hydropad_b200.api import Hydro
    from hydropad_b200.params import HydroParams
    from hydropad_b200.serve import pinned_fields
    n = 20
    with Hydro(HydroParams(shape=(n, n, n), cosmo=True), precision="mixed") as h:
        h.attach_device(*ics.grf_eds_device(n, seed=6, device="cuda"))
        h.start_with_cfl()
        h.evolve(2)
        for nb in (0, 3):
            ref = h.download(nbound=nb)
            bufs = pinned_fields((n + 2 * nb,) * 3)
            out = h.download(nbound=nb, out=bufs)
            assert all(o is b for o, b in zip(out, bufs))
            for a, b in zip(out, ref):
                assert np.array_equal(a, b)
        with pytest.raises(ValueError):
            h.download(nbound=0, out=pinned_fields((n, n, n + 1)))
        with pytest.raises(ValueError):
            h.download(nbound=0, out=[np.zeros((n, n, n)) for _ in range(5)])  # C order
