"""CPU emulation of the pipelined sweep's schedule (ppm_sweep_ws_kernel).

The kernel (hydropad_b200/csrc/hp_sweep_ws.cuh) walks the windows of one or
more pencil groups per CTA.  For window s the main warp group waits for the
window's state (TMA) or loads it, passes a barrier (B1), issues the TMA of
window s+1, runs stages A, B, C1 (ordered within each warp), passes a
barrier (B2), publishes the window's Newton faces, solves its closed-form
faces, waits for the Newton faces of window s-1, passes a barrier (B3) and
updates window s-1.  The Newton warp group solves the faces of window s
between the publication of window s and the wait for them at B3 of window
s+1.  A TMA copy lands somewhere between its issue and its wait.

This test gives every access an interval on the line of the main group's
barrier instants (B1(s) = 10s, B2(s) = 10s+4, B3(s) = 10s+7; stages A, B,
C1 are sub-intervals of (B1, B2), ordered within the warp that holds the
pencil) and checks, for every ring slot, the save area and global memory:

* each read sees the value it needs (the cell or face it names, original
  state before the update, a solved face before the update reads it);
* no write overlaps (in time) a read or a write of the same location;
* every cell of every pencil group is updated exactly once, and every TMA
  box lies inside the pencil.

Faces are classified closed-form or Newton by a seeded coin, so both
solvers' intervals are exercised.  The slot functions are the kernel's
((cell + 4 + ro) mod ring, ro the group's ring offset).
"""
import random

import pytest


class Log:
    """Accesses per location: (kind, lo, hi, value, what, actor, seq).  Two
    accesses are ordered if their intervals do not overlap, or if they are
    made by the same actor (one thread), in program order."""

    def __init__(self):
        self.acc = {}
        self.seq = 0

    def add(self, loc, kind, lo, hi, value, what, actor=None):
        assert lo < hi, (loc, what)
        self.seq += 1
        self.acc.setdefault(loc, []).append((kind, lo, hi, value, what, actor, self.seq))

    @staticmethod
    def before(x, y):
        if x[5] is not None and x[5] == y[5]:
            return x[6] < y[6]
        return x[2] <= y[1]

    def check(self):
        for loc, accs in self.acc.items():
            writes = [a for a in accs if a[0] == "W"]
            for i, w in enumerate(writes):
                for w2 in writes[i + 1:]:
                    assert self.before(w, w2) or self.before(w2, w), ("write-write race", loc, w, w2)
            for a in accs:
                if a[0] != "R":
                    continue
                want = a[3]
                before = []
                for w in writes:
                    if self.before(w, a):
                        before.append(w)
                    elif not self.before(a, w):
                        raise AssertionError(("read-write race", loc, a, w))
                assert before, ("read of an unwritten location", loc, a)
                last = before[0]
                for w in before[1:]:
                    if self.before(last, w):
                        last = w
                assert last[3] == want, ("stale read", loc, a, last)


def emulate(N, T, groups, seed=0):
    """One pencil per group (the slot functions are injective in the
    pencil); returns the checked log."""
    rng = random.Random(seed)
    wpg = (N + 7) // T + 1
    nwin = groups * wpg
    log = Log()
    newton = {}  # (group, face) -> solved by the Newton group

    def win(s):
        j, w = divmod(s, wpg)
        b = -4 + w * T
        return j, w, b, (w >= 1 and b + T <= N), ((s - w) % 4) * T

    def st(c, ro):
        return ("st", (c + 4 + ro) % (4 * T))

    def ai(c, ro):
        return ("a", (c + 4 + ro) % (2 * T))

    def fi(c, ro):
        return ("f", (c + 4 + ro) % (4 * T))

    B1 = lambda s: 10 * s
    B2 = lambda s: 10 * s + 4
    B3 = lambda s: 10 * s + 7
    for j in range(groups):
        for c in range(N):
            log.add(("g", j, c), "W", -10, -9, ("orig", c), "initial state")
    updated = {}
    issued = {}
    for s in range(nwin + 1):
        if s < nwin:
            j, w, b, tma, ro = win(s)
            # ---- state of window s ----
            if not tma:
                lo, hi = B3(s - 1), B1(s)  # after this thread's update of window s-2
                for e in range(b, b + T):
                    if not -4 <= e <= N + 2:
                        continue
                    from_save = e >= N and w > (e - N + 8) // T + 1
                    c = e % N
                    if from_save:
                        log.add(("save", e - N), "R", lo, hi, (j, ("orig", c)), f"load {e} from save")
                    else:
                        log.add(("g", j, c), "R", lo, hi, ("orig", c), f"load {e}")
                        if 0 <= e < 3:
                            log.add(("save", e), "W", lo, hi, (j, ("orig", c)), f"save {e}")
                    log.add(st(e, ro), "W", lo, hi, (j, e), f"load {e}")
            else:
                lo, hi = issued.pop(s), B1(s)
                assert 0 <= b and b + T <= N
                for e in range(b, b + T):
                    log.add(("g", j, e), "R", lo, hi, ("orig", e), f"tma {e}")
                    log.add(st(e, ro), "W", lo, hi, (j, e), f"tma {e}")
            if s + 1 < nwin and win(s + 1)[3]:
                issued[s + 1] = B1(s) + 0.1
            # ---- A, B, C1 (warp-local order) ----
            for e in range(b, b + T):
                c = e - 1
                if -3 <= c <= N + 1:
                    for x in (c - 1, c, c + 1):
                        log.add(st(x, ro), "R", B1(s) + 1, B1(s) + 1.9, (j, x), f"A {c}")
                    log.add(ai(c, ro), "W", B1(s) + 1, B1(s) + 1.9, (j, c), f"A {c}")
            for e in range(b, b + T):
                c = e - 3
                if -1 <= c <= N:
                    for x in (c - 2, c - 1, c, c + 1):
                        log.add(ai(x, ro), "R", B1(s) + 2, B1(s) + 2.9, (j, x), f"B {c} flag")
                    for x in (c - 1, c, c + 1):
                        log.add(st(x, ro), "R", B1(s) + 2, B1(s) + 2.9, (j, x), f"B {c}")
                    log.add(("ls",) + fi(c, ro)[1:], "W", B1(s) + 2, B1(s) + 2.9, (j, c + 1), f"B {c}")
            for e in range(b, b + T):
                f = e - 3
                if 0 <= f <= N:
                    log.add(("ls",) + fi(f - 1, ro)[1:], "R", B1(s) + 3, B1(s) + 3.9, (j, f), f"C1 {f}")
                    log.add(("rs",) + fi(f, ro)[1:], "W", B1(s) + 3, B1(s) + 3.9, (j, f, "right"), f"C1 {f}")
                    nw = rng.random() < 0.4
                    newton[(j, f)] = nw
                    # closed forms: (B2(s), B3(s)); Newton: (B2(s), B3(s+1))
                    lo, hi = B2(s), (B3(s + 1) if nw else B3(s))
                    me = ("solver", j, f)
                    log.add(("ls",) + fi(f - 1, ro)[1:], "R", lo, hi, (j, f), f"C2 {f}", me)
                    log.add(("rs",) + fi(f, ro)[1:], "R", lo, hi, (j, f, "right"), f"C2 {f}", me)
                    for x in (f - 3, f - 2, f - 1, f):  # the density-peak gather along x
                        log.add(st(x, ro), "R", lo, hi, (j, x), f"peak {f}", me)
                    log.add(("rs",) + fi(f, ro)[1:], "W", lo, hi, (j, f, "solved"), f"C2 {f}", me)
        if s >= 1:
            j, w, b, tma, ro = win(s - 1)
            lo, hi = B3(s), B1(s + 1)
            for e in range(b, b + T):
                d = e - 4
                if 0 <= d < N:
                    for f in (d, d + 1):
                        log.add(("rs",) + fi(f, ro)[1:], "R", lo, hi, (j, f, "solved"), f"D {d}")
                    log.add(st(d, ro), "R", lo, hi, (j, d), f"D {d}")
                    log.add(("g", j, d), "W", lo, hi, ("new", d), f"D {d}", ("update", j, d))
                    assert (j, d) not in updated
                    updated[(j, d)] = s
    assert not issued, issued
    assert len(updated) == groups * N
    log.check()
    check_queue_protocol(nwin)
    return log


def check_queue_protocol(nwin):
    """The Newton queue of window s (row s mod 2: counts, chunk counter):
    filled by C1(s) in (B1(s), B2(s)); drained with atomics by the Newton
    warps in (B2(s), B3(s+1)) and by the main warps in (B2(s+1), B3(s+1));
    reset by thread 0 after the barrier B3(s+1) (in (B3(s+1), B1(s+2))).
    Every drain must end before the reset, and the reset before the next
    fill of the row (window s+2)."""
    fill = lambda s: (10 * s, 10 * s + 4)
    drains = lambda s: [(10 * s + 4, 10 * (s + 1) + 7), (10 * (s + 1) + 4, 10 * (s + 1) + 7)]
    reset = lambda s: (10 * (s + 1) + 7, 10 * (s + 2))
    for s in range(nwin):
        r = reset(s)
        assert fill(s)[1] <= min(d[0] for d in drains(s))
        for d in drains(s):
            assert d[1] <= r[0], ("drain after the reset", s, d, r)
        if s + 2 < nwin:
            assert r[1] <= fill(s + 2)[0], ("reset after the next fill", s)


# (T) of the compiled pipelined tiles: x T = 32, y/z T = 8 and 16
@pytest.mark.parametrize("T", [8, 16, 32])
@pytest.mark.parametrize("groups", [1, 2, 3, 5])
def test_ws_schedule(T, groups):
    for N in sorted({8, 9, 12, 16, 24, 31, 32, 33, 40, 48, 64, 100, 128, T + 3, 2 * T - 4, 2 * T + 5}):
        emulate(N, T, groups, seed=N * 31 + groups)


def test_ws_schedule_catches_a_shallow_ring():
    """The checker is not vacuous: a state ring of 3 windows instead of 4
    (the slot of window s+1 still being read) fails."""
    import tests.test_sweep_ws_schedule as m

    src_emulate = m.emulate

    def shallow(N, T, groups, seed=0):
        # re-run with the slot function of a 3-window ring
        wpg = (N + 7) // T + 1
        log = Log()
        for j in range(groups):
            for c in range(N):
                log.add(("g", j, c), "W", -10, -9, ("orig", c), "init")
        # window s reads cells of windows s-1 and s while s+1 lands in slot (s+1) mod 3
        T3 = 3 * T
        for s in range(1, groups * wpg - 1):
            w = s % wpg
            b = -4 + w * T
            for e in range(b - T, b + T):
                log.add(("st", (e + 4) % T3), "R", 10 * s + 1, 10 * s + 2, e, "read")
            for e in range(b + T, b + 2 * T):
                log.add(("st", (e + 4) % T3), "W", 10 * s + 0.1, 10 * s + 10, e, "tma")
        log.check()

    with pytest.raises(AssertionError):
        shallow(64, 8, 1)
    assert src_emulate is m.emulate


# (axis, P, T) of the compiled pipelined tiles (hp_sweep_launch.cuh, HP_WS_TILE_TABLE)
WS_TILES = [(0, 4, 32), (0, 8, 32), (1, 16, 8), (1, 16, 16), (2, 16, 8), (2, 16, 16)]


def ws_layout(axis, P, T):
    """The kernel's index functions (WsLayout): state ring, A ring, face ring."""
    kw = P * T
    kpw = 1 if axis == 0 else 32 // T
    kpad = 0 if axis == 0 else kpw

    def st(slot, tp):
        if axis == 0:
            return (slot // T) * kw + tp * T + slot % T
        i = slot * P + tp
        return i ^ (((i >> 4) & 7) << 1)

    def ring(slot, tp, nslots):
        return tp * nslots + slot if axis == 0 else slot * (P + kpad) + tp

    size_a = P * 2 * T if axis == 0 else 2 * T * (P + kpad)
    size_f = P * 4 * T if axis == 0 else 4 * T * (P + kpad)
    return st, ring, 4 * kw, size_a, size_f


@pytest.mark.parametrize("axis,P,T", WS_TILES)
def test_ws_layout_in_range_and_injective(axis, P, T):
    st, ring, n_st, n_a, n_f = ws_layout(axis, P, T)
    seen = set()
    for slot in range(4 * T):
        for tp in range(P):
            i = st(slot, tp)
            assert 0 <= i < n_st and i not in seen
            seen.add(i)
    for nslots, size in ((2 * T, n_a), (4 * T, n_f)):
        seen = set()
        for slot in range(nslots):
            for tp in range(P):
                i = ring(slot, tp, nslots)
                assert 0 <= i < size and i not in seen
                seen.add(i)


@pytest.mark.parametrize("axis,P,T", [t for t in WS_TILES if t[0] != 0])
def test_ws_tma_rows_match_swizzle(axis, P, T):
    """A y/z window lands by TMA as T rows of 16 doubles (128 bytes) with the
    128-byte swizzle: 16-byte chunk k of row r goes to chunk k ^ (r mod 8)
    (rows of one ring window start on 1024-byte boundaries).  st() must name
    the same element, and a warp's accesses in both thread layouts must hit
    each bank the minimal number of times (2 wavefronts for 32 doubles)."""
    st, _ring, _n, _a, _f = ws_layout(axis, P, T)
    for slot in range(4 * T):
        for tp in range(P):
            byte = slot * 128 + tp * 8
            chunk, row = (byte >> 4) & 7, (byte >> 7) & 7
            phys = (byte & ~0x70) | ((chunk ^ row) << 4)
            assert st(slot, tp) * 8 == phys
    kpw = 32 // T
    for w0 in range(0, 4 * T, T):
        # stages A/B/C1: a warp holds kpw pencils x T positions
        for pw in range(0, P, kpw):
            banks = {}
            for lane in range(32):
                slot, tp = w0 + lane // kpw, pw + lane % kpw
                b = (st(slot, tp) * 2) % 32
                for bb in (b, b + 1):
                    banks[bb] = banks.get(bb, 0) + 1
            assert max(banks.values()) <= 2
        # loads / update: 32 // P positions x P pencils
        for r0 in range(0, T, 32 // P):
            banks = {}
            for lane in range(32):
                slot, tp = w0 + r0 + lane // P, lane % P
                b = (st(slot, tp) * 2) % 32
                for bb in (b, b + 1):
                    banks[bb] = banks.get(bb, 0) + 1
            assert max(banks.values()) <= 2
