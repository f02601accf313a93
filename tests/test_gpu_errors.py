"""Device-side failure detection of the step kernels, without a GPU fault.

Every wait of the TMA step kernels is bounded: when one runs out the CTA
stops, lets its copies in flight land, sets the timeout bit in the flags of
the solves whose tiles it had taken and not finished, and returns; later
launches skip a flagged solve.  These tests make a wait run out on purpose
with the descriptor's testing switch ``stall_test`` (the producer leaves the
first ring stage of each of that solve's tiles unarmed, so the consumers
wait on a barrier nothing completes) and a short wait budget
(``SW_TUNE_WAIT_BUDGET``).  Nothing faults or hangs: the call reports
``SW_ETIMEOUT`` for that solve only, the other solves of the batch come
back bit for bit equal to a clean run, and the library keeps working.
"""

from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# 2^14 units of 1024 cycles: about 8.5 ms at 1.965 GHz, far above any wait
# of a healthy pipeline (microseconds) and short enough for a test
SHORT_BUDGET = 1 << 14


@contextlib.contextmanager
def _wait_budget(units):
    import shearwave_b200._native as native

    lib = native.load()
    old = int(lib.sw_tune_get(native.SW_TUNE_WAIT_BUDGET))
    native.call("sw_tune_set", native.SW_TUNE_WAIT_BUDGET, int(units))
    try:
        yield
    finally:
        native.call("sw_tune_set", native.SW_TUNE_WAIT_BUDGET, old)


def _problems(n_steps=24):
    from shearwave_b200 import workloads as W

    # distinct x extents: the batch's tile queue runs the solves longest-x
    # first, so the smallest (the stalled one) comes last
    shapes = [(40, 30, 70), (28, 22, 40), (18, 20, 26)]
    return [W.problem_inclusions(sh, n_steps, seed=300 + i, tol=1e-9)
            for i, sh in enumerate(shapes)]


def _solves(probs, precision):
    from shearwave_b200 import solver as S

    keys = ("bx", "by", "bz", "rho", "mu", "dX", "dY", "dZ", "dT", "n_steps")
    return [S._Solve(**{k: p[k] for k in keys}, opts=dict(p["opts"], precision=precision))
            for p in probs]


def _status(sv):
    import shearwave_b200._native as native

    flags = C.c_int32(0)
    desc = sv.run.desc
    rc = native.load().sw_fdtd_status(C.byref(desc), C.byref(flags), None)
    return int(rc), int(flags.value)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_timeout_fails_that_solve_only(cuda, precision):
    import torch

    import shearwave_b200 as sw
    import shearwave_b200._native as native
    from shearwave_b200 import solver as S

    probs = _problems()
    clean = sw.shear_fdtd_batch(probs, precision=precision)
    victim = 2
    solves = _solves(probs, precision)
    solves[victim].run.stall_test = 1
    with _wait_budget(SHORT_BUDGET):
        handles = S._run_batch_group(solves, False, torch.cuda.Stream())
        torch.cuda.synchronize()
    for i, (sv, h) in enumerate(zip(solves, handles)):
        rc, flags = _status(sv)
        if i == victim:
            with pytest.raises(RuntimeError, match="SW_ETIMEOUT"):
                sv.finish_collect(h)
            assert rc == native.SW_ETIMEOUT
            assert flags & native.FLAG_TIMEOUT
        else:
            got = sv.finish_collect(h)
            assert rc == native.SW_OK and flags == 0
            for a, b in zip(got, clean[i]):
                assert np.array_equal(a, b)
    # the context stays usable: the same batch again gives the clean results
    again = sw.shear_fdtd_batch(probs, precision=precision)
    for res, ref in zip(again, clean):
        for a, b in zip(res, ref):
            assert np.array_equal(a, b)


def test_batch_errors_return_mode(cuda):
    """shear_fdtd_batch(errors="return") puts the failure in its slot."""
    import torch  # noqa: F401

    import shearwave_b200 as sw
    from shearwave_b200 import solver as S

    probs = _problems(n_steps=10)
    clean = sw.shear_fdtd_batch(probs)
    orig = S._Solve.__init__

    def init(self, *a, **kw):
        orig(self, *a, **kw)
        if self.shape == probs[2]["bz"].shape:
            self.run.stall_test = 1

    S._Solve.__init__ = init
    try:
        with _wait_budget(SHORT_BUDGET):
            got = sw.shear_fdtd_batch(probs, errors="return")
        with _wait_budget(SHORT_BUDGET):
            with pytest.raises(RuntimeError, match="SW_ETIMEOUT"):
                sw.shear_fdtd_batch(probs)
    finally:
        S._Solve.__init__ = orig
    assert isinstance(got[2], RuntimeError)
    for i in (0, 1):
        for a, b in zip(got[i], clean[i]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("precision,n_steps", [("mixed", 12), ("mixed", 80), ("fp64", 12),
                                               ("fp64", 80)])
def test_single_solve_timeout(cuda, precision, n_steps):
    """A lone solve (direct launches, and CUDA-graph replays from 64 steps on)."""
    import shearwave_b200 as sw
    import shearwave_b200._native as native
    from shearwave_b200 import solver as S

    p = _problems(n_steps)[1]
    sv = _solves([p], precision)[0]
    sv.run.stall_test = 1
    with _wait_budget(SHORT_BUDGET):
        with pytest.raises(RuntimeError, match="SW_ETIMEOUT"):
            S._solve_alone(sv, None, False)
    rc, flags = _status(sv)
    assert rc == native.SW_ETIMEOUT and flags & native.FLAG_TIMEOUT
    # a clean solve afterwards matches the same solve with the default budget
    ref = sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                        p["dZ"], p["dT"], p["n_steps"], dict(p["opts"], precision=precision))
    with _wait_budget(SHORT_BUDGET):
        got = sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                            p["dZ"], p["dT"], p["n_steps"], dict(p["opts"], precision=precision))
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
