"""CPU checks of the sweep kernel's thread and ring layouts, for every tile of
the compiled tile table (read from hydropad_b200/csrc/hp_sweep_launch.cuh).

The kernel (hp_sweep.cuh, SweepLayout) uses two thread layouts along y/z: the
load and the update hold 32 neighbouring pencils per warp at one cell; stages
A, B and C1 hold 32/T neighbouring pencils x the T cells of the window per
warp, so that their neighbour exchanges stay within a warp.  The pattern
sort stores the classifying thread's index and C2 decodes its pencil and
face with the same mapping.  These tests restate the index formulas and
check that

* each layout deals every (pencil, cell) of a window to exactly one thread;
* along x, and in stages A, B and C1 along y/z, a warp holds whole pencil
  windows (the condition for warp barriers between those stages);
* ring addresses of the cells alive at once are distinct;
* a warp's 4-byte ring accesses hit 32 distinct banks in both layouts
  (the padding of the y/z ring rows, the slot swizzle along x when a warp
  holds several pencils).
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def tile_table():
    src = open(os.path.join(ROOT, "hydropad_b200", "csrc", "hp_sweep_launch.cuh")).read()
    body = src[src.index("#define HP_TILE_TABLE(X)"):src.index("#define HP_TILE_CHECK")]
    return [tuple(int(v) for v in m) for m in re.findall(r"X\((\d+), (\d+), (\d+), (\d+), (\d+), (\d+)\)", body)]


class Layout:
    """Python restatement of SweepLayout<AXIS, P, T, RING>."""

    def __init__(self, axis, P, T, ring):
        self.axis, self.P, self.T, self.ring = axis, P, T, ring
        self.yz_warp = axis != 0 and 32 % T == 0 and P % (32 // T) == 0
        self.pw = 32 // T if self.yz_warp else 1
        if axis == 0:
            self.stride = ring
        else:
            self.stride = P + self.pw if self.yz_warp else P

    def idx(self, cell, tp):
        slot = cell & (self.ring - 1)
        if self.axis == 0:
            if self.T < 32:   # XOR swizzle of the k-th pencil of a warp
                slot ^= (tp & (32 // self.T - 1)) * self.T
            return tp * self.ring + slot
        return slot * self.stride + tp

    def load(self, t):   # (cell offset, pencil) of thread t in the load and the update
        return (t % self.T, t // self.T) if self.axis == 0 else (t // self.P, t % self.P)

    def stage(self, t):  # the same in stages A, B and C1 (wcell, wpencil)
        if self.axis == 0:
            return t % self.T, t // self.T
        if self.yz_warp:
            return (t & 31) // self.pw, (t >> 5) * self.pw + (t & 31) % self.pw
        return t // self.P, t % self.P


TILES = tile_table()


def test_table_read():
    assert len(TILES) == 3 * len({t[1] for t in TILES}) and len(TILES) >= 30


@pytest.mark.parametrize("axis,tile,P,T,ring,minb", TILES)
def test_layouts_deal_each_cell_once(axis, tile, P, T, ring, minb):
    L = Layout(axis, P, T, ring)
    n = P * T
    for f in (L.load, L.stage):
        seen = {f(t) for t in range(n)}
        assert seen == {(c, p) for c in range(T) for p in range(P)}


@pytest.mark.parametrize("axis,tile,P,T,ring,minb", TILES)
def test_warps_hold_whole_windows(axis, tile, P, T, ring, minb):
    L = Layout(axis, P, T, ring)
    if axis != 0 and not L.yz_warp:
        pytest.skip("this y/z tile keeps CTA barriers between the stages")
    assert 32 % T == 0
    for w in range(P * T // 32):
        cells = [L.stage(t) for t in range(32 * w, 32 * w + 32)]
        for p in {p for _, p in cells}:   # every cell of each of its pencils
            assert sorted(c for c, q in cells if q == p) == list(range(T))


@pytest.mark.parametrize("axis,tile,P,T,ring,minb", TILES)
def test_ring_slots_distinct(axis, tile, P, T, ring, minb):
    L = Layout(axis, P, T, ring)
    assert ring & (ring - 1) == 0 and ring >= T + 6
    b = 40
    live = range(b - 6, b + T)           # oldest cell read (peak fix, f-3) .. newest loaded
    addrs = {L.idx(c, p) for c in live for p in range(P)}
    assert len(addrs) == len(live) * P
    cells = L.stride * L.P if axis == 0 else L.stride * L.ring
    assert max(addrs) < cells


@pytest.mark.parametrize("axis,tile,P,T,ring,minb", TILES)
def test_ring_access_bank_conflict_free(axis, tile, P, T, ring, minb):
    L = Layout(axis, P, T, ring)
    for b in range(-4, 40):
        for w in range(P * T // 32):
            for f in ((L.load, L.stage) if L.yz_warp or axis == 0 else (L.load,)):
                banks = [L.idx(b + c, p) % 32 for t in range(32 * w, 32 * w + 32) for c, p in [f(t)]]
                if axis == 0 or f is L.stage or P >= 32:  # y/z loads with P = 16: two cells per warp
                    assert len(set(banks)) == 32, (axis, tile, b, w, f.__name__)
