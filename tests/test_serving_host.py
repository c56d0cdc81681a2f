"""Host logic of the continuous-batching server (no GPU): admission under
the HBM budget, first-come-first-served order, iteration-level batching,
completion after exactly the requested steps, percentiles."""

import math

import pytest

from cutile.runtime.serving import (SolveKind, SolveRequest, StencilServer, _Active,
                                    percentile)


class FakeServer(StencilServer):
    """The scheduler with the device work replaced by bookkeeping."""

    def __init__(self, kinds, budget):
        super().__init__(kinds, budget_bytes=budget, device="cpu")
        self.iterations = []

    def _admit(self, req, res, now):
        res.admitted = now
        P = self.kinds[req.kind].nstate + 1
        return _Active(req=req, res=res, flat=None, bufs=[None] * P, desc=None, items=1,
                       nbytes=self.memory_of(req))

    def _iterate(self, active, stream):
        self.iterations.append(sorted(a.req.rid for a in active))

    def _stream(self):
        return None

    def _reserve(self):
        pass

    def _record(self, stream):
        import time

        return time.perf_counter()

    def _wait(self, mark):
        pass

    def _mark_time(self, mark, start, t_start):
        return t_start + (mark - start)

    def _done(self, mark):
        return True


KINDS = [SolveKind("heat2d", {}, 1), SolveKind("wave2d", {}, 2), SolveKind("lap7", {}, 1)]


def test_percentile_nearest_rank():
    v = list(range(1, 101))
    assert percentile(v, 50) == 50
    assert percentile(v, 99) == 99
    assert percentile(v, 100) == 100
    assert percentile([3.0], 99) == 3.0
    assert math.isnan(percentile([], 50))


def test_memory_counts_rotating_buffers_with_padded_rows():
    s = FakeServer(KINDS, 1e12)
    # 66 x 66 float64: rows 528 B -> 640 B, 66 rows = 42240 B -> 42240 (256-aligned)
    r = SolveRequest("heat2d", "float64", (66, 66), 10)
    assert s.memory_of(r) == 2 * 42240
    r = SolveRequest("wave2d", "float32", (66, 66), 10)
    assert s.memory_of(r) == 3 * (66 * 384)
    r = SolveRequest("lap7", "float32", (34, 34, 34), 10)
    assert s.memory_of(r) == 2 * (34 * 34 * 256)


def _mix(n=24):
    reqs = []
    for i in range(n):
        kind = ("heat2d", "wave2d", "lap7")[i % 3]
        shape = (34, 34, 34) if kind == "lap7" else (66 + 8 * (i % 5), 66)
        reqs.append(SolveRequest(kind, ("float32", "float64")[i % 2], shape, 3 + (i * 7) % 11,
                                 arrival=0.001 * i))
    return reqs


def test_budget_never_exceeded_and_fifo_admission():
    reqs = _mix()
    s = FakeServer(KINDS, 1)
    budget = 4 * max(s.memory_of(r) for r in reqs)
    s = FakeServer(KINDS, budget)
    res = s.run(reqs, realtime=False)
    assert all(used <= budget for _, _, used in s.stats.trace)
    assert s.stats.peak_bytes <= budget
    # admitted in arrival order
    adm = [(r.admitted, r.rid) for r in res]
    assert [rid for _, rid in sorted(adm)] == sorted(r.rid for r in reqs)
    order = sorted(res, key=lambda r: (r.admitted, r.rid))
    assert [r.rid for r in order] == list(range(len(reqs)))


def test_each_request_runs_exactly_its_steps_and_joins_running_batches():
    reqs = _mix()
    s = FakeServer(KINDS, 1)
    budget = 3 * max(s.memory_of(r) for r in reqs)
    s = FakeServer(KINDS, budget)
    res = s.run(reqs, realtime=False)
    for r in reqs:
        its = [k for k, act in enumerate(s.iterations) if r.rid in act]
        assert len(its) == r.steps, r.rid
        assert its == list(range(its[0], its[0] + r.steps))   # contiguous
    # continuous batching: some request joined while an earlier one was running
    joined = False
    for r in reqs:
        first = next(k for k, act in enumerate(s.iterations) if r.rid in act)
        if first > 0 and any(o < r.rid for o in s.iterations[first]):
            joined = True
    assert joined
    assert all(not math.isnan(x.completed) and x.completed >= x.admitted for x in res)


def test_oversized_request_is_rejected_not_blocking():
    reqs = _mix(6)
    big = SolveRequest("lap7", "float64", (514, 514, 514), 5, arrival=0.0)
    s = FakeServer(KINDS, 10 * max(FakeServer(KINDS, 1).memory_of(r) for r in reqs))
    res = s.run([big] + reqs, realtime=False)
    assert res[0].error is not None and s.stats.rejected == 1
    assert all(r.error is None for r in res[1:])


@pytest.mark.parametrize("budget_mult", [1, 2, 50])
def test_all_complete_for_any_budget_that_fits_the_largest(budget_mult):
    reqs = _mix(15)
    s = FakeServer(KINDS, 1)
    s = FakeServer(KINDS, budget_mult * max(s.memory_of(r) for r in reqs))
    res = s.run(reqs, realtime=False)
    assert all(r.error is None and r.completed >= r.admitted for r in res)
    assert s.stats.admitted == len(reqs)


class BusyGpuServer(FakeServer):
    """A GPU that stays busy for a few polls per iteration: the loop admits
    arrived requests while it waits."""

    def __init__(self, kinds, budget, busy_polls=3):
        super().__init__(kinds, budget)
        self.busy_polls = busy_polls
        self.polls = {}

    def _done(self, mark):
        n = self.polls.get(mark, 0)
        self.polls[mark] = n + 1
        return n >= self.busy_polls


def test_admission_while_the_gpu_runs_keeps_fifo_and_budget():
    reqs = [SolveRequest("heat2d", "float64", (66, 66), 3 + (i % 4), arrival=0.0) for i in range(20)]
    per = FakeServer(KINDS, 1e12).memory_of(reqs[0])
    s = BusyGpuServer(KINDS, 5 * per)
    s.admit_budget_s = 0.0        # the pre-iteration pass admits at most one
    res = s.run(reqs, realtime=False)
    assert all(r.error is None for r in res)
    assert s.stats.admitted == 20 and s.stats.peak_bytes <= 5 * per
    admitted = sorted(range(20), key=lambda i: (res[i].admitted, i))
    assert admitted == list(range(20))
    # every iteration ran at most five solves and each solve ran its steps
    assert max(len(it) for it in s.iterations) <= 5
    for r, q in zip(res, reqs):
        assert sum(r.rid in it for it in s.iterations) == q.steps
