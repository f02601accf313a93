"""Parity at the benchmark's own configurations, against the FP64 oracle.

The golden fixtures pin the oracle to the reference on small grids; these
tests carry that pin to the configurations the benchmark is quoted on, by
running the FP64 oracle itself at their real sizes (in spawned worker
processes, while the GPU works):

* configuration 0 exactly: 64^3, homogeneous medium with viscosity, a
  Gaussian push for the first 5 steps, nT = 500, CG tolerance 1e-10,
  snapshots every 10 steps -- the plain FP64 form within 1e-10 on u, v and
  every snapshot, the mixed form within 1e-4; and its projected force, whose
  divergence residual (max|div f_S| / max|div f|) must agree to 1e-10;
* the three smallest solves of the configuration-3 batch at their real grids
  and step counts, run through the batched path;
* a three-push problem (the ``env_t`` term plus two ``force_terms``) against
  the SUM of three oracle runs with one push each: the scheme and the
  projection are linear in the force, so this pins the multi-term path to
  the reference's own single-push runs;
* ``callback(it, u)`` against the oracle's callback sequence
  (src/shearwave/solver.py:228-229).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2
from oracle_pool import make_pool, oracle_fdtd, oracle_projection

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    with make_pool() as ex:
        yield ex


def _run(p, precision, **kw):
    import shearwave_b200 as sw

    return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                         p["dZ"], p["dT"], p["n_steps"], dict(p["opts"], precision=precision),
                         snapshot_stride=p.get("snapshot_stride"), **kw)


def test_config0_full_size(cuda, pool):
    from shearwave_b200 import workloads as W

    p = W.problem_c0()
    assert p["bz"].shape == (64, 64, 64) and p["n_steps"] == 500
    assert p["snapshot_stride"] == 10 and p["opts"]["poisson_tol"] == 1e-10
    fut = pool.submit(oracle_fdtd, p, snapshot_stride=10)
    u64, v64, s64 = _run(p, "fp64")
    u32, v32, s32 = _run(p, "mixed")
    u_ref, v_ref, s_ref = fut.result()
    assert s64.shape == s_ref.shape == (50, 64, 64, 64, 3)
    assert rel_l2(u64, u_ref) <= 1e-10
    assert rel_l2(v64, v_ref) <= 1e-10
    assert rel_l2(s64, s_ref) <= 1e-10
    for k in range(0, 50, 7):
        assert rel_l2(s64[k], s_ref[k]) <= 1e-10
    assert rel_l2(u32, u_ref) <= 1e-4
    assert rel_l2(v32, v_ref) <= 1e-4
    assert rel_l2(s32, s_ref) <= 1e-4


def test_config0_projection_divergence_residual(cuda, pool):
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O
    from shearwave_b200 import workloads as W

    p = W.problem_c0()
    z = np.zeros_like(p["bz"], dtype=np.float64)
    bz = p["bz"].astype(np.float64)
    fut = pool.submit(oracle_projection, z, z, bz, p["dX"], 1e-10, 2000)
    info = {}
    got = sw.project_vector_field(z, z, bz, p["dX"], p["dY"], p["dZ"], 1e-10, 2000, info=info)
    ref, st = fut.result()
    assert info["iters"] == st["iters"]
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= 1e-10
    h = p["dX"]
    div_in = np.max(np.abs(O.divergence_center(z, z, bz, h, h, h)))

    def residual(f):
        return np.max(np.abs(O.divergence_center(*f, h, h, h))) / div_in

    r_gpu, r_ref = residual(got), residual(ref)
    assert r_gpu <= 1e-8
    assert abs(r_gpu - r_ref) <= 1e-10


def _c3_smallest(k=3):
    from shearwave_b200 import workloads as W

    probs = W.batch_c3()
    return sorted(probs, key=W.cell_steps)[:k]


def test_config3_smallest_solves(cuda, pool):
    """The three smallest configuration-3 solves, batched, against the oracle."""
    import shearwave_b200 as sw

    probs = _c3_smallest()
    futs = [pool.submit(oracle_fdtd, p) for p in probs]
    got64 = sw.shear_fdtd_batch(probs, precision="fp64")
    got32 = sw.shear_fdtd_batch(probs, precision="mixed")
    for p, r64, r32, fut in zip(probs, got64, got32, futs):
        u_ref, v_ref = fut.result()
        assert rel_l2(r64[0], u_ref) <= 1e-10, p["name"]
        assert rel_l2(r64[1], v_ref) <= 1e-10, p["name"]
        assert rel_l2(r32[0], u_ref) <= 1e-4, p["name"]
        assert rel_l2(r32[1], v_ref) <= 1e-4, p["name"]


def test_three_pushes_equal_sum_of_single_push_runs(cuda, pool):
    """force_terms against the sum of one oracle run per push (linearity)."""
    from shearwave_b200 import workloads as W

    shape, n = (30, 26, 44), 90
    p = W.problem_inclusions(shape, n, seed=7, tol=1e-10)
    L = np.array(shape) * W.H
    rng = np.random.default_rng(8)
    pushes = [(p["bz"], p["opts"]["env_t"])]
    for k in range(2):
        c = (0.25 + 0.5 * rng.uniform(0.0, 1.0, 3)) * L
        pushes.append((W.gaussian_push(shape, c), W._envelope(n, 10, start=12 + 25 * k)))
    single = []
    for bz, env in pushes:
        q = dict(p, bz=bz, opts=dict(p["opts"], env_t=env))
        single.append(pool.submit(oracle_fdtd, q))
    multi = dict(p, opts=dict(p["opts"],
                              force_terms=[((None, None, bz), env) for bz, env in pushes[1:]]))
    u64, v64 = _run(multi, "fp64")
    u32, v32 = _run(multi, "mixed")
    parts = [f.result() for f in single]
    u_ref = sum(r[0] for r in parts)
    v_ref = sum(r[1] for r in parts)
    assert rel_l2(u64, u_ref) <= 1e-10
    assert rel_l2(v64, v_ref) <= 1e-10
    assert rel_l2(u32, u_ref) <= 1e-4
    assert rel_l2(v32, v_ref) <= 1e-4


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_callback_sequence(cuda, pool, precision, tol):
    """callback(it, u) sees the same steps and displacements as the reference's."""
    from shearwave_b200 import workloads as W

    p = W.problem_inclusions((18, 16, 22), 25, seed=11, tol=1e-10)
    p["opts"]["vel_damp"] = 0.01
    fut = pool.submit(oracle_fdtd, p, callback_every=1)
    seen = []

    def cb(it, u):
        seen.append((it, np.array(u, copy=True)))

    u, v = _run(p, precision, callback=cb)
    u_ref, v_ref, ref_seen = fut.result()
    assert [it for it, _ in seen] == [it for it, _ in ref_seen] == list(range(25))
    for (_, a), (_, b) in zip(seen, ref_seen):
        if np.any(b):
            assert rel_l2(a, b) <= tol
        else:
            assert not np.any(a)
    assert rel_l2(u, seen[-1][1]) == 0.0
    assert rel_l2(u, u_ref) <= tol and rel_l2(v, v_ref) <= tol
