"""Autotuner for the launch shape of the step kernels.

The step kernels' results do not depend on how the grid is cut into tiles
or how many time steps a launch fuses (every cell runs the same
arithmetic), only their speed does.  Five process-wide knobs of the CUDA
library set the cut (enum ``sw_tune_knob``):

* ``ctas_per_sm`` — resident step CTAs per SM (1 or 2): one CTA per SM
  leaves each CTA the whole SM's bandwidth share, two hide more latency;
* ``batch_tiles_per_cta`` — launches fed by a tile queue (batches, and
  one solve whose tiles would not fill the GPU in whole waves) cut x into
  chunks so that about this many tiles fall to each CTA (more tiles balance
  better, each chunk re-reads two halo planes);
* ``xchunk`` — planes per x chunk for every launch (0 = automatic; 32 in
  batched two-step launches);
* ``tile_shape`` — the mixed step kernel's (z, y) tile: 0 picks, per grid,
  whichever of 64 x 8 and 32 x 16 covers the plane with fewer cells; 1 and
  2 force one;
* ``steps_per_pass`` — time steps per launch of mixed solves that leave
  ``opts["steps_per_pass"]`` at 0: 0 keeps the library's choice (two),
  1 or 2 force it.

:func:`autotune` times a shortened copy of a workload (one problem through
``shear_fdtd``, or a batch through ``shear_fdtd_batch``) under each
candidate setting with CUDA events around the step loop, keeps the fastest,
applies it, and records it in a JSON cache keyed by the workload's shape
class, from which :func:`apply_cached` restores it in a later process.
"""

from __future__ import annotations

import contextlib
import itertools
import json
import math
import os
from pathlib import Path

from . import _native

KNOBS = {"ctas_per_sm": 0, "batch_tiles_per_cta": 1, "xchunk": 2, "tile_shape": 3,
         "steps_per_pass": 4}

__all__ = ["KNOBS", "get_knobs", "set_knobs", "knobs", "workload_key", "autotune",
           "apply_cached", "default_cache_path", "fused_batch_candidates"]


def get_knobs() -> dict:
    """Current knob values."""
    lib = _native.load()
    return {k: int(lib.sw_tune_get(v)) for k, v in KNOBS.items()}


def set_knobs(**values) -> None:
    """Set knobs by name (``ctas_per_sm=1``, ...); ValueError on a bad value."""
    for k, v in values.items():
        if k not in KNOBS:
            raise ValueError(f"unknown knob {k!r}; knobs are {sorted(KNOBS)}")
        try:
            _native.call("sw_tune_set", KNOBS[k], int(v))
        except _native.NativeError as e:
            raise ValueError(str(e)) from None


@contextlib.contextmanager
def knobs(**values):
    """Set knobs for the duration of a ``with`` block."""
    old = get_knobs()
    set_knobs(**values)
    try:
        yield
    finally:
        set_knobs(**old)


def _shape(p):
    ref = p["bx"] if p["bx"] is not None else (p["by"] if p["by"] is not None else p["bz"])
    return tuple(int(s) for s in ref.shape[:3])


def workload_key(problems, precision="mixed") -> str:
    """Shape class of a workload: precision, batch size and total cells (to a
    power of two), and for one problem its grid rounded to 16 cells."""
    if isinstance(problems, dict):
        problems = [problems]
    cells = sum(math.prod(_shape(p)) for p in problems)
    if len(problems) == 1:
        g = "x".join(str(16 * max(1, (s + 8) // 16)) for s in _shape(problems[0]))
        return f"{precision}:single:{g}"
    return f"{precision}:batch{len(problems)}:2^{round(math.log2(max(cells, 1)))}"


def default_cache_path() -> Path:
    root = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(root) / "shearwave_b200" / "tune.json"


def _shorten(p, steps):
    """Copy of problem ``p`` with at most ``steps`` time steps (envelopes cut)."""
    n = min(int(p["n_steps"]), int(steps))
    q = dict(p, n_steps=n)
    opts = dict(p.get("opts") or {})
    if opts.get("env_t") is not None:
        opts["env_t"] = opts["env_t"][:n]
    if opts.get("force_terms"):
        opts["force_terms"] = [(f, None if e is None else e[:n]) for f, e in opts["force_terms"]]
    q["opts"] = opts
    q.pop("snapshot_stride", None)
    return q


def _time_steps(problems, precision) -> float:
    """Gcell-steps/s of the step loop (CUDA events inside the solver); one
    problem runs through shear_fdtd, several through shear_fdtd_batch."""
    from .solver import shear_fdtd, shear_fdtd_batch

    batch = [dict(p, opts=dict(p["opts"], precision=precision, info={})) for p in problems]
    if len(batch) == 1:
        q = batch[0]
        shear_fdtd(q["bx"], q["by"], q["bz"], q["rho"], q["mu"], q["dX"], q["dY"], q["dZ"],
                   q["dT"], q["n_steps"], q["opts"], return_device=True)
    else:
        shear_fdtd_batch(batch, return_device=True)
    t_ms = max(q["opts"]["info"]["t_steps_ms"] for q in batch)
    cells = sum(math.prod(_shape(q)) * q["n_steps"] for q in batch)
    return cells / (t_ms / 1e3) / 1e9


def _candidates(n_problems):
    """Default sweep: two steps per pass (whose tiles are fixed), then one step
    per pass under each tile shape x tiles per CTA (batches) or x chunk (one
    solve), at two CTAs per SM (one CTA per SM measured slower everywhere)."""
    fused = [dict(ctas_per_sm=2, batch_tiles_per_cta=8, xchunk=0, tile_shape=0,
                  steps_per_pass=2)]
    if n_problems > 1:
        return fused + [dict(ctas_per_sm=2, batch_tiles_per_cta=b, xchunk=0, tile_shape=t,
                             steps_per_pass=1)
                        for t, b in itertools.product((0, 1, 2), (4, 8, 16))]
    return fused + [dict(ctas_per_sm=2, xchunk=x, batch_tiles_per_cta=8, tile_shape=t,
                         steps_per_pass=1)
                    for t, x in itertools.product((0, 1, 2), (0, 32, 64))]


def fused_batch_candidates(xchunks=(0, 16, 24, 48, 64)):
    """Two steps per pass with each of ``xchunks`` planes per x chunk (0: the
    library's 32).  The sweep a long batch should use: the two-step kernel
    wins once the board sits at its power cap, which a shortened tuning run
    does not reach, so the one-step shapes are left out of it."""
    return [dict(ctas_per_sm=2, batch_tiles_per_cta=8, xchunk=x, tile_shape=0,
                 steps_per_pass=2) for x in xchunks]


def autotune(problems, *, precision="mixed", steps=64, repeats=2, candidates=None,
             cache=None, apply=True) -> dict:
    """Sweep knob settings on ``problems`` (a problem dict or a list) and keep
    the fastest.

    Each candidate runs a copy of the workload cut to ``steps`` time steps,
    ``repeats`` times after one warm-up run; its score is the best
    Gcell-steps/s of the step loop.  ``cache`` (a path, or True for
    :func:`default_cache_path`) records the winner under
    :func:`workload_key`.  Returns ``{"key", "best", "gcell_steps_per_s",
    "results"}``; the winner is applied when ``apply``.
    """
    if isinstance(problems, dict):
        problems = [problems]
    short = [_shorten(p, steps) for p in problems]
    cands = list(candidates) if candidates is not None else _candidates(len(short))
    old = get_knobs()
    results = []
    try:
        for c in cands:
            set_knobs(**c)
            _time_steps(short, precision)  # warm-up: tables, attributes, caches
            g = max(_time_steps(short, precision) for _ in range(max(1, repeats)))
            results.append({"knobs": dict(c), "gcell_steps_per_s": g})
    finally:
        set_knobs(**old)
    best = max(results, key=lambda r: r["gcell_steps_per_s"])
    key = workload_key(problems, precision)
    if apply:
        set_knobs(**best["knobs"])
    if cache:
        path = default_cache_path() if cache is True else Path(cache)
        path.parent.mkdir(parents=True, exist_ok=True)
        data = json.loads(path.read_text()) if path.exists() else {}
        data[key] = {"knobs": best["knobs"], "gcell_steps_per_s": best["gcell_steps_per_s"]}
        path.write_text(json.dumps(data, indent=1, sort_keys=True))
    return {"key": key, "best": best["knobs"], "gcell_steps_per_s": best["gcell_steps_per_s"],
            "results": results}


def apply_cached(problems, *, precision="mixed", cache=True) -> dict | None:
    """Apply the cached winner for this workload's key; returns it, or None."""
    path = default_cache_path() if cache is True else Path(cache)
    if not path.exists():
        return None
    entry = json.loads(path.read_text()).get(workload_key(problems, precision))
    if entry is None:
        return None
    set_knobs(**entry["knobs"])
    return entry["knobs"]
