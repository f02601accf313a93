"""Runs of the CPU oracle in worker processes, for the GPU parity tests.

TEST INFRASTRUCTURE: the oracle (oracle/shearwave_oracle.py) is the checker.
Large oracle runs (a whole benchmark configuration) take a minute or more of
single-threaded NumPy each, so the tests submit them to a process pool
started with the ``spawn`` method (a pool forked after CUDA has been
initialised can hang) and collect the results after their GPU runs.
"""

from __future__ import annotations

import concurrent.futures as cf
import multiprocessing as mp
import os

import numpy as np


def _f64(v):
    return v.astype(np.float64) if isinstance(v, np.ndarray) else v


def oracle_fdtd(p: dict, *, force_terms=None, snapshot_stride=None, callback_every=None):
    """FP64 oracle run of a problem dict (shearwave_b200.workloads format).

    Returns ``(u, v)`` or ``(u, v, snaps)``; with ``callback_every`` the
    oracle's callback records ``(it, u copy)`` every that many steps and the
    list is returned as a last element.
    """
    from oracle import shearwave_oracle as O

    opts = {k: _f64(v) for k, v in p["opts"].items() if k != "force_terms"}
    terms = force_terms
    if terms is None and p["opts"].get("force_terms"):
        terms = p["opts"]["force_terms"]
    if terms is not None:
        terms = [(tuple(None if b is None else _f64(b) for b in tb), _f64(env))
                 for tb, env in terms]
    seen = []
    cb = None
    if callback_every:
        def cb(it, u):
            if it % callback_every == 0:
                seen.append((it, u.copy()))
    out = O.shear_fdtd(*(None if p[k] is None else _f64(p[k]) for k in ("bx", "by", "bz")),
                       _f64(p["rho"]), _f64(p["mu"]), p["dX"], p["dY"], p["dZ"], p["dT"],
                       p["n_steps"], opts=opts, callback=cb, dtype=np.float64,
                       snapshot_stride=snapshot_stride, force_terms=terms)
    if callback_every:
        return (*out, seen)
    return out


def oracle_projection(fx, fy, fz, h, tol, max_iters):
    """FP64 oracle projection; returns the three components and the CG stats."""
    from oracle import shearwave_oracle as O

    st = O.CGStats()
    out = O.project_vector_field(*(np.asarray(f, np.float64) for f in (fx, fy, fz)), h, h, h,
                                 tol, max_iters, dtype=np.float64, stats=st)
    return out, {"iters": st.iters, "reason": st.reason}


def make_pool(workers: int | None = None) -> cf.ProcessPoolExecutor:
    n = workers or max(1, min(8, (os.cpu_count() or 2) - 1))
    return cf.ProcessPoolExecutor(max_workers=n, mp_context=mp.get_context("spawn"))
