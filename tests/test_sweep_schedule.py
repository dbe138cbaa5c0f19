"""CPU emulation of the fused sweep's sliding-window schedule.

The kernel (hydropad_b200/csrc/hp_sweep.cuh) walks a periodic pencil of N
cells in iterations of T cells; each iteration runs the phases load, A, B,
C, D separated by barriers, passing per-cell results through rings of RING
slots, and updates the pencil in place.  This test replays that schedule
symbolically and checks, for every read, that the slot holds the intended
cell, that state reads see original (pre-sweep) values, that no phase reads
what another thread writes in the same phase, and that every cell is written
exactly once.  It covers all pencil lengths the kernel accepts for the tile
shapes it is compiled with.

lag=1 replays the non-STENCIL build's full-pencil solver (PENCIL): the walk
runs one cell further, the density-peak window of face f is cells
f-2..f+1, and stage D splits in two: D1 writes the new total energy of
cell e-4 to a ring, D2 (after a barrier) updates cell e-5 from its faces,
its state, its old neighbours' densities and the new total energies of
cells e-6..e-4 (0 beyond the pencil's ends).

early=True replays the mixed path's z sweeps: the cells of the next
iteration are loaded right after C2, before this iteration's D (which reads
the cell from global memory, not from the ring), C2 reads no state (the
density-peak values come from the pre-pass).  The save-area rule of the
plain schedule still holds: it takes a wrapped cell from the save area when
D of its iteration or an earlier one wrote it, and the save area then holds
it (written by an earlier load) whether D has run or not.
"""
import pytest

from tests.test_sweep_layout import tile_table

# (T, RING) of the compiled tiles, every axis
TILES = sorted({(T, ring) for _axis, _tile, _P, T, ring, _minb in tile_table()})


def emulate(N, T, R, lag=0, early=False):
    assert not (early and lag)
    glob = {c: ("orig", c) for c in range(N)}
    written = {}
    ring = {}
    A = {}
    LS = {}
    FS = {}
    save = {}
    right = {}
    SE = {}

    def wrap(c):
        return c % N

    def load(b):
        es = [b + tl for tl in range(T)]
        reads_save, writes = set(), {}
        for tl, e in enumerate(es):
            if -4 <= e <= N + 2:
                from_save = e >= N and (e + 4) // T > (e - N + 8 + lag) // T
                if from_save:
                    reads_save.add(e - N)
                    val = save[e - N]
                else:
                    val = glob[wrap(e)]
                assert val == ("orig", wrap(e)), (N, T, e, val)
                if 0 <= e < 3:
                    writes[("save", e)] = val
                writes[("ring", e % R)] = (e, val)
        for (kind, k), v in writes.items():
            assert not (kind == "save" and k in reads_save), "same-phase save race"
            (save if kind == "save" else ring)[k] = v

    b = -4
    if early:
        load(b)
    while b <= N + 3 + lag:
        es = [b + tl for tl in range(T)]
        # ---- load ----
        if not early:
            load(b)

        def state_ok(x):
            assert ring[x % R] == (x, ("orig", wrap(x))), (N, T, x, ring[x % R])

        # ---- A ----
        wr = {}
        for e in es:
            c = e - 1
            if -3 <= c <= N + 1:
                for x in (c - 1, c, c + 1):
                    state_ok(x)
                wr[c % R] = c
        A.update(wr)
        # ---- B ----
        wr = {}
        for tl, e in enumerate(es):
            c = e - 3
            if -1 <= c <= N:
                for x in range(c - 2, c + 3):
                    state_ok(x)
                for x in range(c - 2, c + 2):
                    assert A[x % R] == x
                wr[c % R] = c
                right[tl] = c
        LS.update(wr)
        # ---- C1: publish right states, classify ----
        wr = {}
        for tl, e in enumerate(es):
            f = e - 3
            if 0 <= f <= N:
                assert right[tl] == f
                wr[f % R] = ("right", f)
        assert len(wr) == len({v for v in wr.values()}), "ring slot collision"
        FS.update(wr)
        work = sorted(v[1] for v in wr.values())
        # ---- C2: any thread solves any face of the iteration ----
        wr = {}
        for f in work:
            assert LS[(f - 1) % R] == f - 1
            assert FS[f % R] == ("right", f)
            if not early:
                for x in range(f - 3, f + 1 + lag):  # the peak window (f-2..f+1 with lag)
                    state_ok(x)
            wr[f % R] = ("face", f)
        FS.update(wr)
        if early and b + T <= N + 3 + lag:
            load(b + T)  # the next iteration's cells, before this D
        # ---- D (lag: D1, barrier, D2) ----
        wr = {}
        if lag:
            wse = {}
            for e in es:
                d = e - 4
                if 0 <= d < N:
                    assert FS[d % R] == ("face", d) and FS[(d + 1) % R] == ("face", d + 1)
                    state_ok(d)
                    wse[d % R] = ("etot", d)
            SE.update(wse)
        for tl, e in enumerate(es):
            d = e - 4 - lag
            if 0 <= d < N:
                assert FS[d % R] == ("face", d), (N, T, d, FS[d % R])
                assert FS[(d + 1) % R] == ("face", d + 1)
                if early:
                    assert glob[d] == ("orig", d), (N, T, d, glob[d])  # D reads the cell from global memory
                else:
                    state_ok(d)
                if lag:
                    for x in (d - 1, d + 1):
                        state_ok(x)  # the old neighbours of the peak test
                    for x in (d - 1, d, d + 1):
                        if 0 <= x < N:
                            assert SE[x % R] == ("etot", x), (N, T, d, x, SE.get(x % R))
                wr[d] = ("new", d)
        for d, v in wr.items():
            assert d not in written
            written[d] = True
            glob[d] = v
        b += T
    assert sorted(written) == list(range(N))


def test_tiles_read():
    assert len(TILES) >= 5


@pytest.mark.parametrize("lag,early", [(0, False), (1, False), (0, True)])
@pytest.mark.parametrize("T,R", TILES)
def test_schedule_all_lengths(T, R, lag, early):
    for N in range(8, 200):
        emulate(N, T, R, lag, early)


@pytest.mark.parametrize("lag,early", [(0, False), (1, False), (0, True)])
def test_schedule_large_pencils(lag, early):
    for T, R in TILES:
        for N in (256, 511, 512, 1024):
            emulate(N, T, R, lag, early)
