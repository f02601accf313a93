"""Queue, admission and completion logic of the serving loop (CPU, fake engine).

The fake engine stands in for the GPU: it records every batched advance and
fails on request (allocation failure, malformed request) so that admission
control, cancellation and failure isolation are exercised without a device.
"""

from __future__ import annotations

import threading
import time

import pytest

from shearwave_b200.serve import ShearServer, latency_percentiles


class FakeEngine:
    def __init__(self, step_time=0.0):
        self.calls = []
        self.live = {}
        self.peak_bytes = 0
        self.step_time = step_time
        self.lock = threading.Lock()

    def footprint(self, p):
        if p.get("bz") is None:
            raise ValueError("At least one body-force component must be provided.")
        return p["fp"]

    def admit(self, p):
        if p.get("oom"):
            raise MemoryError("simulated allocation failure")
        if p.get("bad"):
            raise ValueError("malformed request")
        h = {"id": p["id"], "n": p["n_steps"], "fp": p["fp"], "done": 0}
        with self.lock:
            self.live[p["id"]] = h
            self.peak_bytes = max(self.peak_bytes, sum(x["fp"] for x in self.live.values()))
        return h

    @staticmethod
    def steps(h):
        return h["n"]

    def advance(self, handles, begins, clock, n):
        for h, b in zip(handles, begins):
            lit = clock - b
            assert 0 <= lit < h["n"]
            h["done"] = min(h["n"], lit + n)
        self.calls.append((clock, n, tuple(h["id"] for h in handles)))
        if self.step_time:
            time.sleep(self.step_time * n)

    @staticmethod
    def finish(h):
        assert h["done"] == h["n"]
        return ("result", h["id"])

    def release(self, h):
        with self.lock:
            del self.live[h["id"]]


class AsyncFakeEngine(FakeEngine):
    """Completion in the background, as on the GPU: a result becomes ready
    `copy_time` after finish_begin, and `mark` events complete `mark_time`
    after they are made; the engine records how far the loop runs ahead."""

    def __init__(self, step_time=0.0, copy_time=0.01, mark_time=0.003):
        super().__init__(step_time)
        self.copy_time = copy_time
        self.mark_time = mark_time
        self.ended = []
        self.outstanding = 0
        self.max_outstanding = 0

    def finish_begin(self, h):
        assert h["done"] == h["n"]
        return {"id": h["id"], "ready_at": time.perf_counter() + self.copy_time}

    @staticmethod
    def finish_ready(token):
        return time.perf_counter() >= token["ready_at"]

    def finish_end(self, h, token):
        dt = token["ready_at"] - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        self.ended.append(token["id"])
        return ("result", h["id"])

    def mark(self):
        self.outstanding += 1
        self.max_outstanding = max(self.max_outstanding, self.outstanding)
        return time.perf_counter() + self.mark_time

    def wait_mark(self, t):
        dt = t - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        self.outstanding -= 1


ENGINES = [FakeEngine, AsyncFakeEngine]


class _Arr:
    shape = (8, 8, 8)


def _req(i, n_steps=10, fp=1, **kw):
    return dict(bx=None, by=None, bz=_Arr(), n_steps=n_steps, id=i, fp=fp, **kw)


@pytest.mark.parametrize("engine", ENGINES)
def test_all_requests_complete_with_their_own_results(engine):
    eng = engine()
    with ShearServer(eng, hbm_budget=100, chunk_steps=4) as srv:
        futs = [srv.submit(_req(i, n_steps=5 + 3 * i)) for i in range(6)]
        res = [f.result(timeout=10) for f in futs]
    assert res == [("result", i) for i in range(6)]
    st = srv.stats()
    assert st["completed"] == 6 and st["failed"] == 0
    assert st["latency_s"]["p99"] >= st["latency_s"]["p50"] >= 0


@pytest.mark.parametrize("engine", ENGINES)
def test_admission_respects_the_memory_budget(engine):
    eng = engine()
    with ShearServer(eng, hbm_budget=10, chunk_steps=2) as srv:
        futs = [srv.submit(_req(i, n_steps=6, fp=4)) for i in range(5)]
        for f in futs:
            f.result(timeout=10)
    assert eng.peak_bytes <= 10  # never more than two 4-byte requests at once
    assert max(len(c[2]) for c in eng.calls) == 2


def test_oversize_request_is_refused_at_submission():
    srv = ShearServer(FakeEngine(), hbm_budget=10)
    with pytest.raises(MemoryError, match="budget"):
        srv.submit(_req(0, fp=11))
    assert srv.rejected == 1


def test_malformed_request_raises_before_queueing():
    srv = ShearServer(FakeEngine(), hbm_budget=10)
    with pytest.raises(ValueError, match="body-force"):
        srv.submit(dict(bx=None, by=None, bz=None, n_steps=3))


@pytest.mark.parametrize("engine", ENGINES)
def test_failures_stay_with_their_request(engine):
    eng = engine()
    with ShearServer(eng, hbm_budget=100, chunk_steps=3) as srv:
        ok1 = srv.submit(_req(0))
        oom = srv.submit(_req(1, oom=True))
        bad = srv.submit(_req(2, bad=True))
        ok2 = srv.submit(_req(3))
        assert ok1.result(timeout=10) == ("result", 0)
        assert ok2.result(timeout=10) == ("result", 3)
        with pytest.raises(MemoryError):
            oom.result(timeout=10)
        with pytest.raises(ValueError):
            bad.result(timeout=10)
    assert srv.stats()["failed"] == 2


def test_cancelled_request_is_never_admitted():
    eng = FakeEngine(step_time=0.002)
    srv = ShearServer(eng, hbm_budget=4, chunk_steps=2).start()
    first = srv.submit(_req(0, n_steps=40, fp=4))  # fills the budget
    queued = srv.submit(_req(1, fp=4))
    assert queued.cancel()
    assert first.result(timeout=10) == ("result", 0)
    srv.stop()
    assert all(1 not in c[2] for c in eng.calls)


def test_late_arrival_joins_running_solves():
    """Continuous batching: a request arriving mid-run overlaps with it."""
    eng = FakeEngine(step_time=0.002)
    with ShearServer(eng, hbm_budget=100, chunk_steps=5) as srv:
        long = srv.submit(_req(0, n_steps=200))
        time.sleep(0.05)
        late = srv.submit(_req(1, n_steps=10))
        late.result(timeout=10)
        assert not long.done()  # the late one finished while the long one still ran
        long.result(timeout=10)
    shared = [c for c in eng.calls if set(c[2]) == {0, 1}]
    assert shared, "the two requests never advanced in the same launch"


def test_latency_percentiles():
    p = latency_percentiles([0.1, 0.2, 0.3, 0.4])
    assert abs(p["p50"] - 0.25) < 1e-12 and p["n"] == 4
    assert latency_percentiles([])["p99"] is None


def test_async_completion_resolves_each_request_once_and_bounds_run_ahead():
    """Results are copied out while later chunks run; every request is
    resolved exactly once, and the loop is never more than two chunks (plus
    the one being enqueued) ahead of the device."""
    eng = AsyncFakeEngine(step_time=0.0005, copy_time=0.02)
    with ShearServer(eng, hbm_budget=100, chunk_steps=3) as srv:
        futs = [srv.submit(_req(i, n_steps=4 + 5 * (i % 3))) for i in range(9)]
        res = [f.result(timeout=10) for f in futs]
    assert res == [("result", i) for i in range(9)]
    assert sorted(eng.ended) == list(range(9))
    assert eng.max_outstanding <= 3
    assert srv.stats()["completed"] == 9


class AbandoningEngine(AsyncFakeEngine):
    """A device that abandoned one request's tiles: its result raises, as the
    real engine's finish_collect does for a timed-out solve (SW_ETIMEOUT)."""

    def finish_end(self, h, token):
        out = super().finish_end(h, token)
        if h["id"] == 2:
            raise RuntimeError("shear_fdtd: ... (SW_ETIMEOUT); the result is incomplete")
        return out


class AbandoningSyncEngine(FakeEngine):
    def finish(self, h):
        if h["id"] == 2:
            raise RuntimeError("shear_fdtd: ... (SW_ETIMEOUT); the result is incomplete")
        return super().finish(h)


@pytest.mark.parametrize("engine", [AbandoningEngine, AbandoningSyncEngine])
def test_device_failure_fails_that_request_only(engine):
    eng = engine()
    with ShearServer(eng, hbm_budget=100, chunk_steps=4) as srv:
        futs = [srv.submit(_req(i, n_steps=6 + i)) for i in range(5)]
        with pytest.raises(RuntimeError, match="SW_ETIMEOUT"):
            futs[2].result(timeout=10)
        others = [futs[i].result(timeout=10) for i in (0, 1, 3, 4)]
        # the server keeps serving after the failure
        late = srv.submit(_req(9, n_steps=3)).result(timeout=10)
    assert others == [("result", i) for i in (0, 1, 3, 4)]
    assert late == ("result", 9)
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 5
    assert not eng.live  # every request's memory was released


def test_admission_error_fails_that_request_only():
    """An unexpected error while admitting a request (a device call failing)
    fails that request; it never leaves its future unresolved."""

    class Broken(FakeEngine):
        def admit(self, p):
            if p["id"] == 1:
                raise RuntimeError("sw_fdtd_materials failed")
            return super().admit(p)

    with ShearServer(Broken(), hbm_budget=100, chunk_steps=4) as srv:
        futs = [srv.submit(_req(i)) for i in range(3)]
        with pytest.raises(RuntimeError, match="sw_fdtd_materials"):
            futs[1].result(timeout=10)
        assert futs[0].result(timeout=10) == ("result", 0)
        assert futs[2].result(timeout=10) == ("result", 2)


@pytest.mark.parametrize("engine", ENGINES)
def test_stream_without_results_counts_failures(engine):
    """A long stream that keeps no results reports how many requests failed
    and completes the rest."""
    from shearwave_b200.serve import poisson_arrivals, run_stream

    kinds = [dict(n_steps=4), dict(n_steps=7), dict(n_steps=3, bad=True)]
    problems = [_req(i, **kinds[i % 3]) for i in range(30)]
    arrivals = poisson_arrivals(2000.0, len(problems), seed=3)
    eng = engine()
    with ShearServer(eng, hbm_budget=100, chunk_steps=3) as srv:
        failed = run_stream(srv, problems, arrivals, timeout_s=10, keep=False)
    assert failed == 10
    st = srv.stats()
    assert st["completed"] == 20 and st["failed"] == 10
    assert not eng.live
