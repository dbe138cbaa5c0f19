"""GPU: boxes advanced in a batch against the same boxes advanced alone.

Every member of a batch follows its own evolve_sys step (nrot, dt, nstep),
so with the same tiles the batched result must be bitwise identical to the
box advanced alone through hp_evolve -- for boxes of different sizes,
members joining and leaving between steps, and members at different nrot
(which split a sweep slot into several launches).  The alone path is itself
pinned to the oracle by test_gpu_parity.
"""
import numpy as np
import pytest

from tests.helpers import grf_state, params_for, sod_state

from hydropad_b200._lib import num_tiles  # noqa: E402

pytestmark = pytest.mark.gpu

TILES = (1, 1, 1)


def _box(kind, n, seed, precision):
    from hydropad_b200.api import Hydro
    if kind == "sod":
        state = sod_state(n, axis=seed % 3)
        prm = params_for((n, n, n))
    else:
        state = grf_state(n, seed=seed)
        prm = params_for((n, n, n), cosmo=True)
    h = Hydro(prm, precision=precision)
    h.attach_state(*state)
    h.set_tiles(*TILES)
    h.start_with_cfl()
    return h, state, prm


def _alone(kind, n, seed, precision, pre, steps):
    h, _, _ = _box(kind, n, seed, precision)
    with h:
        h.evolve(pre + steps)
        return h.download(), h.get_scalars()


def _same(a, b, what):
    for q, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"{what}: field {q} differs (max |d| = {np.abs(x - y).max():.3e})"


BOXES = [("grf", 16, 5), ("grf", 24, 6), ("sod", 32, 7), ("grf", 20, 8)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_alone(precision, graph):
    """Aligned members (one static plan per nrot, graphs when asked)."""
    from hydropad_b200.batch import Batch
    steps = 8
    with Batch(precision, capacity=8) as b:
        b.set_tiles(*TILES)
        boxes = [_box(k, n, s, precision)[0] for k, n, s in BOXES]
        for h in boxes:
            b.add(h)
        b.step(steps, graph=graph)
        assert b.synchronize() == [0] * len(boxes)
        for (k, n, s), h in zip(BOXES, boxes):
            ref, rs = _alone(k, n, s, precision, 0, steps)
            _same(h.download(), ref, f"{k}{n} {precision}")
            g = h.get_scalars()
            assert (g.nstep, g.t, g.dt) == (rs.nstep, rs.t, rs.dt)
        for h in boxes:
            b.remove(h)
            h.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_join_leave_staggered(precision):
    """Members at different nrot (advanced alone first), one joining late
    and one leaving early: dynamic plans with several launches per slot."""
    from hydropad_b200.batch import Batch
    pre = [0, 1, 2, 4]        # steps each box takes alone before joining
    join = [0, 0, 3, 0]       # batch step at which it joins
    leave = [9, 5, 9, 9]      # batch step after which it leaves
    total = 9
    boxes = []
    for (k, n, s), p in zip(BOXES, pre):
        h = _box(k, n, s, precision)[0]
        h.evolve(p)
        boxes.append(h)
    with Batch(precision, capacity=8) as b:
        b.set_tiles(*TILES)
        for t in range(total + 1):
            for i, h in enumerate(boxes):
                if join[i] == t:
                    b.add(h)
                if leave[i] == t and h in b.members:
                    b.synchronize()
                    b.remove(h)
            if t < total:
                b.step(1, graph=True)
        b.synchronize()
    for i, ((k, n, s), h) in enumerate(zip(BOXES, boxes)):
        batched = min(leave[i], total) - join[i]
        ref, rs = _alone(k, n, s, precision, pre[i], batched)
        with h:
            _same(h.download(), ref, f"{k}{n} {precision} pre={pre[i]} batched={batched}")
            assert h.get_scalars().nstep == rs.nstep


def test_batch_autotune_keeps_state():
    from hydropad_b200.batch import Batch
    with Batch("mixed", capacity=4) as b:
        boxes = [_box(k, n, s, "mixed")[0] for k, n, s in BOXES[:3]]
        before = [h.download() for h in boxes]
        for h in boxes:
            b.add(h)
        tiles = b.autotune(reps=1)
        assert all(0 <= t < num_tiles() for t in tiles)
        b.synchronize()
        for h, ref in zip(boxes, before):
            _same(h.download(), ref, "autotune")
        for h in boxes:
            b.remove(h)
            h.close()


def test_batch_rejects_mismatch():
    from hydropad_b200._lib import HydroError
    from hydropad_b200.batch import Batch
    with Batch("mixed", capacity=1) as b:
        h64 = _box("grf", 16, 1, "fp64")[0]
        with pytest.raises(HydroError):
            b.add(h64)          # precision differs
        h1 = _box("grf", 16, 2, "mixed")[0]
        h2 = _box("grf", 16, 3, "mixed")[0]
        b.add(h1)
        with pytest.raises(HydroError):
            b.add(h1)           # already a member
        with pytest.raises(HydroError):
            b.add(h2)           # over capacity
        b.remove(h1)
        for h in (h64, h1, h2):
            h.close()


def test_batch_density_peak_fix_matches_alone():
    """With dmax low enough for the density-peak fix (riemannsolver.F90:
    279-285) to act, batched y/z sweeps read the pre-pass values of their
    own pencils: bitwise equal to the boxes alone."""
    from hydropad_b200.api import Hydro
    from hydropad_b200.batch import Batch
    specs = [(24, 31), (16, 32), (20, 33)]
    steps = 4

    def make(n, seed, dmax):
        h = Hydro(params_for((n, n, n), cosmo=True, dmax=dmax), precision="fp64")
        h.attach_state(*grf_state(n, seed=seed))
        h.set_tiles(*TILES)
        h.start_with_cfl()
        return h

    alone, plain = [], []
    for n, seed in specs:
        for dmax, out in ((1.5, alone), (2e10, plain)):
            with make(n, seed, dmax) as h:
                h.evolve(steps)
                out.append(h.download())
    assert any(not np.array_equal(a[0], b[0]) for a, b in zip(alone, plain)), "the fix never acted"
    boxes = [make(n, seed, 1.5) for n, seed in specs]
    with Batch("fp64", capacity=4) as b:
        b.set_tiles(*TILES)
        for h in boxes:
            b.add(h)
        b.step(steps)
        b.synchronize()
        for h, ref in zip(boxes, alone):
            _same(h.download(), ref, "peak")
            b.remove(h)
            h.close()
