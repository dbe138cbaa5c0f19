"""CPU tests of the serving scheduler (continuous batching, HBM-budget
admission, latency accounting) against a CPU model of the GPU engine, and of
the serving trace generator."""
import math

import numpy as np
import pytest

from hydropad_b200.serve import Request, Scheduler, box_bytes, poisson_trace
from tests.serve_model import ModelEngine


def _trace(n=40, rate=200.0, seed=5):
    return poisson_trace(n, rate=rate, seed=seed, side_min=32, side_max=128, step_min=10, step_max=60)


def test_trace_statistics():
    tr = poisson_trace(4000, rate=200.0, seed=1)
    gaps = np.diff([r.arrival for r in tr])
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0
    sides = np.array([r.side for r in tr])
    assert sides.min() >= 32 and sides.max() <= 256 and np.all(sides % 16 == 0)
    # log-uniform: about as many sides below sqrt(32*256) ~ 90 as above
    assert 0.4 < np.mean(sides < math.sqrt(32 * 256)) < 0.6
    steps = np.array([r.steps for r in tr])
    assert steps.min() >= 50 and steps.max() <= 500
    assert len({r.seed for r in tr}) == len(tr)


def test_every_request_completes_with_its_steps():
    tr = _trace()
    eng = ModelEngine()
    st = Scheduler(eng, budget_bytes=box_bytes(128) * 4, capacity=8, chunk=4, keep_results=True).run(tr)
    assert sorted(c.rid for c in st.completed) == [r.rid for r in tr]
    by_id = {r.rid: r for r in tr}
    for c in st.completed:
        assert c.result == by_id[c.rid].steps            # ran exactly its step count
        assert c.done >= c.admitted >= c.arrival
    assert st.peak_resident_bytes <= box_bytes(128) * 4


def test_fifo_admission_and_stalls():
    # a budget of one big box: requests are admitted strictly in arrival order
    tr = [Request(i, 0.001 * i, side, 20, i) for i, side in enumerate([128, 32, 32, 128, 32])]
    eng = ModelEngine()
    st = Scheduler(eng, budget_bytes=box_bytes(128) + box_bytes(32), capacity=8, chunk=8).run(tr)
    order = [rid for what, rid, _ in eng.log if what == "create"]
    assert order == [0, 1, 2, 3, 4]
    assert st.admission_stalls > 0 and st.stall_seconds > 0
    assert len(st.completed) == len(tr)


def test_continuous_batching_shares_steps():
    # two requests that overlap in time run in the same batch steps
    tr = [Request(0, 0.0, 64, 40, 0), Request(1, 0.0, 64, 40, 1)]
    eng = ModelEngine()
    st = Scheduler(eng, budget_bytes=box_bytes(64) * 2, capacity=8, chunk=8).run(tr)
    assert st.steps_launched == 40
    assert abs(st.completed[0].done - st.completed[1].done) < 1e-12


def test_capacity_limits_members():
    tr = [Request(i, 0.0, 32, 16, i) for i in range(10)]
    eng = ModelEngine()

    seen = []
    orig_step = eng.step

    def step(k):
        seen.append(len(eng.members))
        orig_step(k)

    eng.step = step
    Scheduler(eng, budget_bytes=10 ** 12, capacity=3, chunk=16).run(tr)
    assert max(seen) == 3


def test_results_read_back_while_the_others_run():
    # request 0 ends with the first chunk: the scheduler detaches it and
    # enqueues request 1's next chunk before reading request 0 back
    tr = [Request(0, 0.0, 32, 8, 0), Request(1, 0.0, 32, 24, 1)]
    eng = ModelEngine()
    st = Scheduler(eng, budget_bytes=box_bytes(32) * 2, capacity=4, chunk=8).run(tr)
    ev = [e for e in eng.log if e[0] in ("step", "finish")]
    assert ev[0] == ("step", 8, 2) and ev[1] == ("step", 8, 1)
    assert ev[2][:2] == ("finish", 0)
    assert st.steps_launched == 24
    done = {c.rid: c.done for c in st.completed}
    assert done[0] < done[1]


def test_rejects_request_larger_than_budget():
    with pytest.raises(ValueError):
        Scheduler(ModelEngine(), budget_bytes=box_bytes(64), capacity=4).run([Request(0, 0.0, 128, 10, 0)])
