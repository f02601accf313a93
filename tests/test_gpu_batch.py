"""Batched solves (shear_fdtd_batch) against solves run alone.

Every cell of a batched launch goes through the same kernel code as a solve
run alone, and the batched CG keeps each solve's own tiles, partial sums and
stopping rule, so a solve's result must be bit-identical alone and in the
batch.  One batched solve is also checked against the FP64 oracle.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _problems():
    from shearwave_b200 import workloads as W

    shapes = [(20, 18, 26), (33, 12, 70), (16, 16, 16), (9, 40, 21), (24, 24, 130)]
    steps = [30, 12, 45, 20, 33]
    probs = []
    for i, (sh, n) in enumerate(zip(shapes, steps)):
        p = W.problem_inclusions(sh, n, seed=100 + i, tol=1e-9)
        if i == 1:
            p["opts"]["vel_damp"] = 0.02
        if i == 2:
            p["snapshot_stride"] = 9
        if i == 3:
            p["opts"]["eta"] = 0.0
        probs.append(p)
    return probs


def _alone(p, precision):
    import shearwave_b200 as sw

    return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"],
                         p["dT"], p["n_steps"], dict(p["opts"], precision=precision),
                         snapshot_stride=p.get("snapshot_stride"))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_alone_bitwise(cuda, precision):
    import shearwave_b200 as sw

    probs = _problems()
    got = sw.shear_fdtd_batch(probs, precision=precision)
    for p, res in zip(probs, got):
        ref = _alone(p, precision)
        assert len(res) == len(ref)
        for a, b in zip(res, ref):
            assert a.dtype == b.dtype and a.shape == b.shape
            assert np.array_equal(a, b)


def test_batch_member_against_oracle(cuda):
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O

    probs = _problems()
    got = sw.shear_fdtd_batch(probs, precision="fp64")
    p = probs[0]
    o64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) else v)
           for k, v in p["opts"].items()}
    ref = O.shear_fdtd(None, None, p["bz"].astype(np.float64), p["rho"].astype(np.float64),
                       p["mu"].astype(np.float64), p["dX"], p["dY"], p["dZ"], p["dT"],
                       p["n_steps"], opts=o64, dtype=np.float64)
    assert rel_l2(got[0][0], ref[0]) <= 1e-10
    assert rel_l2(got[0][1], ref[1]) <= 1e-10


def test_batch_with_host_stepped_member(cuda):
    """A member needing per-step host work (reprojection) runs alone inside the batch call."""
    import shearwave_b200 as sw

    probs = _problems()[:3]
    probs[1] = dict(probs[1], opts=dict(probs[1]["opts"], reproject_every=5))
    got = sw.shear_fdtd_batch(probs, precision="mixed")
    ref = _alone(probs[1], "mixed")
    for a, b in zip(got[1], ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_long_batch_replays_graphs_bitwise(cuda, precision):
    """Runs of >= 64 steps with the same solves running replay CUDA graphs of
    the batched launches (one host call per 32 steps); the results stay bit
    for bit those of the solves run alone, and the host makes far fewer
    enqueue calls than kernels run."""
    import shearwave_b200 as sw
    import shearwave_b200._native as native
    from shearwave_b200 import workloads as W

    probs = [W.problem_inclusions(sh, 300, seed=40 + i, tol=1e-9)
             for i, sh in enumerate([(22, 20, 30), (18, 26, 24), (30, 16, 20)])]
    k0, h0 = native.launch_count(), native.host_enqueue_count()
    got = sw.shear_fdtd_batch(probs, precision=precision)
    kernels, enqueues = native.launch_count() - k0, native.host_enqueue_count() - h0
    # 288 of the 300 steps run as 9 graph replays: >= 9 x 16 kernels without a host call
    assert kernels - enqueues >= 140, (kernels, enqueues)
    for p, res in zip(probs, got):
        ref = _alone(p, precision)
        for a, b in zip(res, ref):
            assert np.array_equal(a, b)


def test_pushes_and_snapshots_inside_replayed_runs_bitwise(cuda):
    """Push and snapshot tiles (force terms from the shared term buffer,
    snapshot writes) inside graph-replayed runs of the two-step kernel: a
    push from step 100, snapshots every 6 steps on one solve, none on the
    others; every solve still matches its lone run bit for bit."""
    import shearwave_b200 as sw
    from shearwave_b200 import workloads as W

    probs = [W.problem_inclusions(sh, 300, seed=60 + i, tol=1e-9)
             for i, sh in enumerate([(22, 20, 30), (18, 26, 24), (30, 16, 20)])]
    env = np.zeros(300, np.float32)
    env[100:104] = np.linspace(1.0, 0.25, 4)
    probs[0]["opts"]["force_terms"] = [((None, None, 0.5 * probs[0]["bz"][::-1]), env)]
    probs[1]["snapshot_stride"] = 6
    got = sw.shear_fdtd_batch(probs, precision="mixed")
    for p, res in zip(probs, got):
        ref = _alone(p, "mixed")
        assert len(res) == len(ref)
        for a, b in zip(res, ref):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("nterms", [5, 33])
def test_many_force_terms_at_one_step_bitwise(cuda, nterms):
    """Several force terms active at the same steps: up to 32 go through the
    two-step kernel's shared term buffer, more make that solve run one step
    per launch; either way the batched solve matches its lone run bit for
    bit."""
    import shearwave_b200 as sw
    from shearwave_b200 import workloads as W

    probs = [W.problem_inclusions(sh, 200, seed=80 + i, tol=1e-9)
             for i, sh in enumerate([(20, 18, 24), (16, 22, 20)])]
    rng = np.random.default_rng(nterms)
    terms = []
    for k in range(nterms):
        env = np.zeros(200, np.float32)
        env[100 + k % 3:104 + k % 3] = rng.uniform(0.1, 1.0, 4).astype(np.float32)
        terms.append(((None, None, rng.uniform(-1, 1) * probs[0]["bz"]), env))
    probs[0]["opts"]["force_terms"] = terms
    got = sw.shear_fdtd_batch(probs, precision="mixed")
    for p, res in zip(probs, got):
        ref = _alone(p, "mixed")
        for a, b in zip(res, ref):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_4d_force_streamed_from_the_device(cuda, precision):
    """4-D forces: the non-zero slices are projected up front (batched CG)
    and streamed as patterns; bit for bit the per-step host projection of the
    reference's loop (solver.py:198-199), which a zero byte budget forces;
    the solve also joins a batch unchanged."""
    import shearwave_b200 as sw
    from shearwave_b200 import workloads as W

    p = W.problem_inclusions((20, 16, 24), 30, seed=77, tol=1e-9)
    t = np.arange(30, dtype=np.float32)
    env = (np.sin(0.3 * t) * (t < 18)).astype(np.float32)
    b4 = (p["bz"][..., None] * env[None, None, None, :]).astype(np.float32)
    opts = {k: v for k, v in p["opts"].items() if k != "env_t"}
    q = dict(p, bz=b4, opts=opts)
    args = (None, None, b4, p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"], p["dT"], 30)
    streamed = sw.shear_fdtd(*args, dict(opts, precision=precision))
    host = sw.shear_fdtd(*args, dict(opts, precision=precision, force_stream_bytes=0))
    for a, b in zip(streamed, host):
        assert np.array_equal(a, b)
    batched = sw.shear_fdtd_batch([q, _problems()[0]], precision=precision)
    for a, b in zip(batched[0], streamed):
        assert np.array_equal(a, b)
