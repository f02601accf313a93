"""Continuous-batching request loop for shear_fdtd solves on one GPU.

Requests (dicts of ``shear_fdtd`` keyword arguments) arrive at any time.  A
background thread owns the GPU: at every chunk boundary it admits waiting
requests, in arrival order, while their device-memory footprint fits the
budget and a slot is free; it then advances every running solve together
(one batched launch per time step covers the tiles of all of them, each at
its own step offset); solves that finish are copied out, their futures
resolved and their memory returned to the budget.  Admission and completion
happen between launches, so a request never waits for a whole batch to
drain, and a solve's result is the same alone and in any mix: every cell of
a batched launch runs the same kernel code as a solve run alone.

The loop never waits for the GPU while it has work to give it: results are
copied out on a second stream and a future resolves once its copy has
landed, and the loop runs at most two chunks ahead of the GPU (so a new
request joins the launches within two chunks of its admission).

The queue, admission and bookkeeping are plain Python over an engine with
six methods (footprint, admit, advance, steps, finish, release), plus
optional ones for asynchronous completion (finish_begin, finish_ready,
finish_end) and run-ahead control (mark, wait_mark); the GPU engine drives
the CUDA library, and the test suite drives the same loop with a fake
engine on the CPU.
"""

from __future__ import annotations

import collections
import math
import threading
import time
from concurrent.futures import CancelledError, Future

import numpy as np

__all__ = ["GpuEngine", "ShearServer", "latency_percentiles"]


def latency_percentiles(lat_s) -> dict:
    """p50 / p95 / p99 / mean / max of a list of latencies (seconds)."""
    if not lat_s:
        return {"p50": None, "p95": None, "p99": None, "mean": None, "max": None, "n": 0}
    a = np.asarray(lat_s, dtype=np.float64)
    return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
            "p99": float(np.percentile(a, 99)), "mean": float(a.mean()), "max": float(a.max()),
            "n": int(a.size)}


class _Request:
    __slots__ = ("problem", "future", "t_arrive", "t_admit", "t_done", "footprint", "handle",
                 "begin", "rid", "token")

    def __init__(self, problem, rid):
        self.problem = problem
        self.future = Future()
        self.t_arrive = time.perf_counter()
        self.t_admit = None
        self.t_done = None
        self.footprint = 0
        self.handle = None
        self.begin = 0
        self.rid = rid
        self.token = None


class GpuEngine:
    """The CUDA engine: one ``_Solve`` per admitted request, batched steps."""

    def __init__(self, precision="mixed", return_device=False):
        import torch

        from . import _native
        from ._device import require_cuda

        self.torch = torch
        self.native = _native
        self.dev = require_cuda()
        self.precision = precision
        self.return_device = return_device
        self.stream = torch.cuda.Stream(device=self.dev)
        self.copy_stream = torch.cuda.Stream(device=self.dev)

    # -- sizes -------------------------------------------------------------
    @staticmethod
    def _shape(p):
        ref = p["bx"] if p["bx"] is not None else (p["by"] if p["by"] is not None else p["bz"])
        if ref is None:
            raise ValueError("At least one body-force component must be provided.")
        return tuple(int(s) for s in ref.shape[:3])

    def footprint(self, p) -> int:
        """Device bytes a request holds while it runs (state, materials,
        force patterns, outputs and the projection's scratch)."""
        nx, ny, nz = self._shape(p)
        pz = (nz + 7) // 8 * 8
        ncell = nx * ny * pz
        es = 8 if (p.get("opts") or {}).get("precision", self.precision) == "fp64" else 4
        nterms = 1 + len((p.get("opts") or {}).get("force_terms") or ())
        for b in (p["bx"], p["by"], p["bz"]):
            if b is not None and len(b.shape) == 4:  # 4-D forces: one pattern per step at most
                nterms = max(nterms, int(b.shape[3]) + nterms - 1)
        state = 3 * (3 if es == 8 else 9) * ncell * es
        coef = 2 * ncell * es
        pats = nterms * 3 * ncell * es
        outs = 2 * 3 * nx * ny * nz * es
        scratch = 8 * ncell * 8  # projection vectors (FP64), freed after admission
        return int(state + coef + pats + outs + scratch)

    # -- lifecycle ---------------------------------------------------------
    def on_thread_start(self):
        """Make this engine's device current on the serving thread."""
        self.torch.cuda.set_device(self.dev)
        self.native.call("sw_set_device", self.dev.index)

    def admit(self, p):
        from .solver import _project_inputs, _Solve

        with self.torch.cuda.stream(self.stream):
            opts = dict(p.get("opts") or {})
            opts.setdefault("precision", self.precision)
            kw = {k: p[k] for k in ("bx", "by", "bz", "rho", "mu", "dX", "dY", "dZ", "dT",
                                    "n_steps")}
            sv = _Solve(**kw, opts=opts, snapshot_stride=p.get("snapshot_stride"))
            if sv.needs_per_step_host(None):
                raise ValueError("the server runs batchable requests only (no 4-D forces, "
                                 "reproject_every, verbose, traces or direct kernels)")
            _project_inputs([sv])
            sv.build_terms()
            sv.mark_steps_begin()
            return sv

    @staticmethod
    def steps(handle) -> int:
        return handle.n_steps

    def advance(self, handles, begins, clock, nsteps):
        from .solver import _batch_steps

        with self.torch.cuda.stream(self.stream):
            groups = {}
            for h, b in zip(handles, begins):
                groups.setdefault(h.prec, []).append((h, b))
            for items in groups.values():
                _batch_steps([h.run for h, _ in items], [b for _, b in items], clock, nsteps)

    def finish(self, handle):
        with self.torch.cuda.stream(self.stream):
            return handle.finish(self.return_device)

    def finish_begin(self, handle):
        """Enqueue the output conversion and the copies to the host (on the
        copy stream); returns the token finish_end turns into the result."""
        with self.torch.cuda.stream(self.stream):
            return handle.finish_enqueue(self.return_device, self.copy_stream)

    @staticmethod
    def finish_ready(token) -> bool:
        return token["event"].query()

    def finish_end(self, handle, token):
        with self.torch.cuda.stream(self.stream):
            return handle.finish_collect(token)

    def mark(self):
        """An event after the work enqueued so far."""
        ev = self.torch.cuda.Event()
        ev.record(self.stream)
        return ev

    @staticmethod
    def wait_mark(ev):
        ev.synchronize()

    @staticmethod
    def release(handle):
        del handle


class ShearServer:
    """Continuous-batching server: ``submit(problem) -> Future``.

    ``hbm_budget``: device bytes the running requests may hold together
    (150 GB by default); ``max_active``: running requests at most;
    ``chunk_steps``: time steps between two admission / completion points.
    Use as a context manager or call :meth:`start` / :meth:`stop`.
    """

    def __init__(self, engine=None, *, hbm_budget=150e9, max_active=64, chunk_steps=50,
                 precision="mixed", return_device=False):
        self.engine = engine if engine is not None else GpuEngine(precision, return_device)
        self.hbm_budget = float(hbm_budget)
        self.max_active = int(max_active)
        self.chunk_steps = int(chunk_steps)
        self._pending = collections.deque()
        self._active = []
        self._finishing = []  # results being copied out
        self._marks = collections.deque()  # one event per chunk in flight
        self._cv = threading.Condition()
        self._stop = False
        self._thread = None
        self._clock = 0
        self._used = 0
        self._next_id = 0
        self.completed = []  # (rid, latency_s, queue_s, cell_steps)
        self.rejected = 0
        self.failed = 0
        self.busy_s = 0.0
        self._t_start = None
        self._error = None

    # -- public API --------------------------------------------------------
    def submit(self, problem) -> Future:
        """Queue one request; the future resolves to the shear_fdtd result."""
        fp = self.engine.footprint(problem)  # validates the force arguments
        if fp > self.hbm_budget:
            self.rejected += 1
            raise MemoryError(
                f"request needs {fp / 1e9:.2f} GB of device memory, above the "
                f"{self.hbm_budget / 1e9:.2f} GB budget")
        with self._cv:
            if self._stop:
                raise RuntimeError("server is stopped")
            req = _Request(problem, self._next_id)
            req.footprint = fp
            self._next_id += 1
            self._pending.append(req)
            self._cv.notify()
        return req.future

    def start(self):
        if self._thread is None:
            self._t_start = time.perf_counter()
            self._thread = threading.Thread(target=self._loop, name="shearwave-server",
                                            daemon=True)
            self._thread.start()
        return self

    def stop(self, wait=True):
        with self._cv:
            self._stop = True
            self._cv.notify()
        if wait and self._thread is not None:
            self._thread.join()
        if self._error is not None:
            raise self._error

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def stats(self) -> dict:
        lat = [c[1] for c in self.completed]
        queue = [c[2] for c in self.completed]
        cells = sum(c[3] for c in self.completed)
        wall = (time.perf_counter() - self._t_start) if self._t_start else 0.0
        return {"completed": len(self.completed), "rejected": self.rejected,
                "failed": self.failed, "latency_s": latency_percentiles(lat),
                "queue_s": latency_percentiles(queue),
                "gcell_steps_per_s": cells / wall / 1e9 if wall > 0 else None,
                "gcell_steps_per_busy_s": cells / self.busy_s / 1e9 if self.busy_s > 0 else None,
                "wall_s": wall}

    # -- the loop ------------------------------------------------------------
    def _loop(self):
        try:
            if hasattr(self.engine, "on_thread_start"):
                self.engine.on_thread_start()
            while True:
                with self._cv:
                    while (not self._stop and not self._pending and not self._active
                           and not self._finishing):
                        self._cv.wait(timeout=0.05)
                    if (self._stop and not self._pending and not self._active
                            and not self._finishing):
                        return
                self._admit()
                if not self._active:
                    self._collect(block=True)  # nothing left to overlap the copies with
                    if self._pending and not self._finishing:
                        time.sleep(0.001)  # waiting on memory held by no one: retry
                    continue
                t0 = time.perf_counter()
                self._advance()
                self._complete()
                self._collect(block=False)
                self.busy_s += time.perf_counter() - t0
        except BaseException as e:  # surface engine failures to every waiter
            self._error = e
            with self._cv:
                for r in list(self._pending) + self._active + self._finishing:
                    if not r.future.done():
                        r.future.set_exception(e)
                self._pending.clear()
                self._active = []
                self._finishing = []

    def _admit(self):
        while True:
            with self._cv:
                if not self._pending or len(self._active) >= self.max_active:
                    return
                req = self._pending[0]
                if req.future.cancelled():
                    self._pending.popleft()
                    continue
                if self._used + req.footprint > self.hbm_budget:
                    return  # wait for memory: keep arrival order
                self._pending.popleft()
                if not req.future.set_running_or_notify_cancel():
                    continue
            try:
                req.handle = self.engine.admit(req.problem)
            except Exception as e:  # bad request, no memory or a device error: fail it alone
                self.failed += 1
                req.future.set_exception(e)
                continue
            req.begin = self._clock
            req.t_admit = time.perf_counter()
            self._used += req.footprint
            self._active.append(req)

    def _advance(self):
        remaining = [self.engine.steps(r.handle) - (self._clock - r.begin) for r in self._active]
        n = max(1, min(self.chunk_steps, min(remaining)))
        self.engine.advance([r.handle for r in self._active], [r.begin for r in self._active],
                            self._clock, n)
        self._clock += n
        if hasattr(self.engine, "mark"):  # stay at most two chunks ahead of the GPU
            self._marks.append(self.engine.mark())
            while len(self._marks) > 2:
                self.engine.wait_mark(self._marks.popleft())

    def _complete(self):
        keep = []
        for r in self._active:
            if self._clock - r.begin < self.engine.steps(r.handle):
                keep.append(r)
                continue
            if hasattr(self.engine, "finish_begin"):
                r.token = self.engine.finish_begin(r.handle)
                self._finishing.append(r)
            else:
                try:
                    result = self.engine.finish(r.handle)
                except RuntimeError as e:  # this request's solve was abandoned on the device
                    self._fail(r, e)
                    continue
                self._resolve(r, result)
        self._active = keep

    def _collect(self, block: bool):
        """Resolve the requests whose results have reached the host (all of
        them when ``block``)."""
        left = []
        for r in self._finishing:
            if block or self.engine.finish_ready(r.token):
                try:
                    result = self.engine.finish_end(r.handle, r.token)
                except RuntimeError as e:  # this request's solve was abandoned on the device
                    self._fail(r, e)
                    continue
                self._resolve(r, result)
            else:
                left.append(r)
        self._finishing = left

    def _fail(self, r, exc):
        """Fail one request whose device work reported an error (the other
        requests of the mix keep running): its memory returns to the budget."""
        self.failed += 1
        self.engine.release(r.handle)
        r.handle = None
        r.token = None
        self._used -= r.footprint
        r.future.set_exception(exc)

    def _resolve(self, r, result):
        r.t_done = time.perf_counter()
        cells = _cell_steps(r.problem)
        self.completed.append((r.rid, r.t_done - r.t_arrive, r.t_admit - r.t_arrive, cells))
        self.engine.release(r.handle)
        r.handle = None
        r.token = None
        self._used -= r.footprint  # the request's memory returns to the budget
        r.future.set_result(result)


def _cell_steps(p) -> int:
    ref = p["bx"] if p["bx"] is not None else (p["by"] if p["by"] is not None else p["bz"])
    return int(math.prod(ref.shape[:3])) * int(p["n_steps"])


def poisson_arrivals(rate_hz: float, n: int, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of a Poisson process with the given mean rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=n))


def run_stream(server: ShearServer, problems, arrivals_s, timeout_s=None, keep=True):
    """Submit ``problems`` at ``arrivals_s`` (seconds from now) and wait for all.

    Returns the results in submission order (None for a cancelled request).
    With ``keep=False`` nothing holds on to a result once its request has
    finished (a long stream's outputs would not fit in host memory), and the
    return value is the number of requests that failed.
    """
    t0 = time.perf_counter()
    if not keep:
        left = threading.Semaphore(0)
        failed = [0]

        def done(f):
            if f.cancelled() or f.exception() is not None:
                failed[0] += 1
            left.release()

        n = 0
        for p, ta in zip(problems, arrivals_s):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            server.submit(p).add_done_callback(done)
            n += 1
        for _ in range(n):
            if not left.acquire(timeout=timeout_s):
                raise TimeoutError("request stream did not finish in time")
        return failed[0]
    futs = []
    for p, ta in zip(problems, arrivals_s):
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        futs.append(server.submit(p))
    out = []
    for f in futs:
        try:
            out.append(f.result(timeout=timeout_s))
        except CancelledError:
            out.append(None)
    return out
