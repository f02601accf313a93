"""Serving on the GPU: continuous batching gives every request the result it gets alone.

Requests of different grids, materials, pushes and lengths arrive while others
run; each future's (u, v) must equal the same problem run alone through
shear_fdtd bit for bit, and the server reports latency percentiles.
"""

from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems():
    from shearwave_b200 import workloads as W

    shapes = [(24, 20, 30), (16, 16, 16), (40, 12, 66), (20, 28, 18), (30, 30, 30), (12, 14, 90)]
    steps = [40, 25, 33, 60, 18, 45]
    probs = []
    for i, (sh, n) in enumerate(zip(shapes, steps)):
        p = W.problem_inclusions(sh, n, seed=200 + i, tol=1e-9)
        if i == 2:
            rng = np.random.default_rng(7)
            env = np.zeros(n, np.float32)
            env[5:12] = 1.0
            p["opts"]["force_terms"] = [((None, None, p["bz"][::-1].copy()), env)]
        probs.append(p)
    return probs


def _alone(p):
    import shearwave_b200 as sw

    return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"],
                         p["dT"], p["n_steps"], dict(p["opts"]))


@pytest.mark.parametrize("budget", [150e9, 3e7])
def test_served_results_equal_alone(cuda, budget):
    from shearwave_b200.serve import ShearServer

    probs = _problems()
    with ShearServer(hbm_budget=budget, chunk_steps=7) as srv:
        futs = []
        for p in probs:
            futs.append(srv.submit(p))
            time.sleep(0.01)  # staggered arrivals: later requests join running ones
        results = [f.result(timeout=120) for f in futs]
    st = srv.stats()
    assert st["completed"] == len(probs)
    assert st["latency_s"]["p99"] is not None
    for p, got in zip(probs, results):
        ref = _alone(p)
        for a, b in zip(got, ref):
            assert a.dtype == b.dtype and np.array_equal(a, b)


def test_server_rejects_requests_needing_the_host_between_steps(cuda):
    from shearwave_b200.serve import ShearServer

    p = _problems()[1]
    p = dict(p, opts=dict(p["opts"], reproject_every=5))
    with ShearServer(chunk_steps=5) as srv:
        f = srv.submit(p)
        with pytest.raises(ValueError, match="batchable"):
            f.result(timeout=60)
