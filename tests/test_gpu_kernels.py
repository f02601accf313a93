"""Step kernels against each other and against the FP64 oracle on awkward grids.

Grids are chosen to hit tile edges (z tiles of 64 / 32 cells, y tiles of 8
rows), short and long x chunks, non-multiple-of-8 z pitches and grids with
a single interior plane.  Tolerances: the TMA-staged and direct-load kernels
compute the same expression per cell, so they agree to FP rounding (rel L2
<= 1e-12 in FP64, <= 1e-6 in FP32); the FP64 form matches the oracle to
rel L2 <= 1e-10 and the mixed form to <= 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GRIDS = [(5, 7, 9), (17, 13, 11), (3, 20, 70), (40, 9, 133), (12, 33, 65)]


def _problem(shape, seed, n_steps=24):
    rng = np.random.default_rng(seed)
    h = (0.5e-3, 0.6e-3, 0.45e-3)
    rho = (1000.0 * (1 + 0.05 * rng.uniform(-1, 1, shape))).astype(np.float32)
    mu = (3e3 * np.exp(rng.uniform(-1, 1, shape))).astype(np.float32)
    eta = rng.uniform(0.2, 1.0, shape).astype(np.float32)
    ax = [(np.arange(n) - (n - 1) / 2.0) * hh for n, hh in zip(shape, h)]
    x, y, z = np.meshgrid(*ax, indexing="ij")
    bz = (1e3 * np.exp(-(x**2 + y**2) / (2 * 1e-3**2) - z**2 / (2 * 2e-3**2))).astype(np.float32)
    bx = (200 * np.exp(-((x - 5e-4) ** 2 + y**2 + z**2) / (2 * 1e-3**2))).astype(np.float32)
    env = np.zeros(n_steps, np.float32)
    env[:6] = np.linspace(1.0, 0.5, 6)
    iu = (1e-7 * rng.standard_normal((*shape, 3))).astype(np.float32)
    opts = {"eta": eta, "env_t": env, "vel_damp": 0.01, "poisson_tol": 1e-10,
            "poisson_max_iters": 4 * max(shape), "initial_u": iu}
    return dict(bx=bx, by=None, bz=bz, rho=rho, mu=mu, dX=h[0], dY=h[1], dZ=h[2], dT=4e-6,
                n_steps=n_steps), opts


def _run(p, opts, **kw):
    import shearwave_b200 as sw

    o = dict(opts, **kw)
    return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"],
                         p["dT"], p["n_steps"], o, snapshot_stride=6)


@pytest.mark.parametrize("shape", GRIDS)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tma_matches_direct_kernel(cuda, shape, precision):
    p, opts = _problem(shape, seed=sum(shape))
    a = _run(p, opts, precision=precision, step_kernel="tma")
    b = _run(p, opts, precision=precision, step_kernel="direct")
    tol = 1e-12 if precision == "fp64" else 1e-6
    for x, y in zip(a, b):
        assert rel_l2(x, y) <= tol


@pytest.mark.parametrize("xchunk", [1, 2, 7, 1000])
def test_xchunk_does_not_change_results(cuda, xchunk):
    p, opts = _problem((30, 18, 70), seed=3)
    ref = _run(p, opts, precision="fp64", xchunk=0)
    got = _run(p, opts, precision="fp64", xchunk=xchunk)
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("shape", GRIDS[:4])
def test_against_oracle(cuda, shape):
    from oracle import shearwave_oracle as O

    p, opts = _problem(shape, seed=7 + shape[0])
    o64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) else v) for k, v in opts.items()}
    ref = O.shear_fdtd(p["bx"].astype(np.float64), None, p["bz"].astype(np.float64),
                       p["rho"].astype(np.float64), p["mu"].astype(np.float64), p["dX"], p["dY"],
                       p["dZ"], p["dT"], p["n_steps"], opts=o64, dtype=np.float64,
                       snapshot_stride=6)
    g64 = _run(p, opts, precision="fp64")
    g32 = _run(p, opts, precision="mixed")
    for r, a, b in zip(ref, g64, g32):
        assert rel_l2(a, r) <= 1e-10
        assert rel_l2(b, r) <= 1e-4


FUSED_GRIDS = [(5, 7, 9), (17, 13, 11), (3, 20, 70), (40, 9, 133), (12, 33, 65), (70, 16, 64),
               (9, 71, 37)]


@pytest.mark.parametrize("shape", FUSED_GRIDS)
@pytest.mark.parametrize("kahan", [True, False])
@pytest.mark.parametrize("tile_shape", [1, 2])
def test_two_steps_per_pass_matches_one(cuda, shape, kahan, tile_shape):
    """The fused two-step kernel reproduces two one-step launches bit for bit
    (both use the same per-cell arithmetic; with the compensated sum the
    one-step kernel runs both), with either tile shape (tile_shape 1: 64-wide
    level-1 rows, one per warp; 2: 32-wide, two rows per warp).

    Odd n_steps (the last step runs alone), snapshots every 5 steps (both
    parities of the fused pair), pushes, damping and viscosity.
    """
    p, opts = _problem(shape, seed=11 + sum(shape), n_steps=25)
    opts = dict(opts, kahan=kahan)
    import shearwave_b200 as sw
    from shearwave_b200 import tune

    def run(spp):
        return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                             p["dZ"], p["dT"], p["n_steps"],
                             dict(opts, precision="mixed", steps_per_pass=spp),
                             snapshot_stride=5)

    with tune.knobs(tile_shape=tile_shape):
        a, b = run(2), run(1)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_two_steps_per_pass_without_viscosity(cuda):
    p, opts = _problem((30, 20, 90), seed=5, n_steps=16)
    opts = dict(opts, eta=0.0)
    import shearwave_b200 as sw

    outs = [sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"], p["dZ"],
                          p["dT"], p["n_steps"], dict(opts, steps_per_pass=spp))
            for spp in (2, 1)]
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("precision,spp", [("mixed", 1), ("mixed", 2), ("fp64", 0)])
def test_cuda_graph_replay_matches_direct_launches(cuda, precision, spp):
    """Long step runs replay an instantiated graph; results are bit-identical."""
    import shearwave_b200 as sw

    p, opts = _problem((20, 18, 40), seed=9, n_steps=137)

    def run(graph):
        return sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                             p["dZ"], p["dT"], p["n_steps"],
                             dict(opts, precision=precision, steps_per_pass=spp,
                                  cuda_graph=graph), snapshot_stride=None)

    for x, y in zip(run(True), run(False)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_unstable_run_is_flagged(cuda, precision):
    """An unstable dT (viscous number 240, limit 2) overflows within 300 steps
    in both forms; the solve reports it (info["nonfinite"] and a
    RuntimeWarning), alone and batched."""
    import warnings

    import numpy as np

    import shearwave_b200 as sw
    from shearwave_b200 import workloads as W

    shape = (20, 18, 22)
    bz = W.gaussian_push(shape, [(n - 1) / 2 * W.H for n in shape])
    n = 300
    env = np.zeros(n, np.float32)
    env[:5] = 1
    opts = {"eta": 5.0, "env_t": env, "poisson_tol": 1e-8, "poisson_max_iters": 200,
            "precision": precision}
    for batched in (False, True):
        info = {}
        o = dict(opts, info=info)
        with warnings.catch_warnings(record=True) as rec:
            warnings.simplefilter("always")
            if batched:
                p = dict(bx=None, by=None, bz=bz, rho=1000.0, mu=3e3, dX=W.H, dY=W.H, dZ=W.H,
                         dT=1e-3, n_steps=n, opts=o)
                sw.shear_fdtd_batch([p, dict(p, opts=dict(opts))])
            else:
                sw.shear_fdtd(None, None, bz, 1000.0, 3e3, W.H, W.H, W.H, 1e-3, n, o)
        assert info["nonfinite"], batched
        assert any(issubclass(w.category, RuntimeWarning) for w in rec), batched
    # and a stable run is not flagged
    info = {}
    sw.shear_fdtd(None, None, bz, 1000.0, 3e3, W.H, W.H, W.H, 1e-6, n, dict(opts, info=info))
    assert not info["nonfinite"]


@pytest.mark.parametrize("tile_shape", [0, 1, 2])
def test_two_steps_per_pass_batched(cuda, tile_shape):
    """A batch run with two steps per pass (solves of different lengths, so
    one-step launches fill the odd ends) equals each solve run alone with one
    step per launch, bit for bit, whichever tile shape the launches use."""
    import shearwave_b200 as sw
    from shearwave_b200 import tune

    probs = []
    for k, (shape, n) in enumerate([((30, 20, 90), 16), ((17, 13, 11), 9), ((40, 9, 133), 21),
                                    ((9, 71, 37), 12)]):
        p, opts = _problem(shape, seed=40 + k, n_steps=n)
        probs.append(dict(p, opts=dict(opts, precision="mixed", steps_per_pass=2)))
    with tune.knobs(tile_shape=tile_shape):
        batch = sw.shear_fdtd_batch(probs)
    for p, got in zip(probs, batch):
        alone = sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                              p["dZ"], p["dT"], p["n_steps"], dict(p["opts"], steps_per_pass=1))
        for x, y in zip(got, alone):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("shape", [(3, 4, 97), (6, 5, 70), (4, 9, 33)])
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_stencil_operators_on_long_rows_bitexact(cuda, shape, dt):
    """The operator and strain kernels walk the grid one (x, y) row per warp
    with the lanes along z; rows longer than a warp (several passes per lane,
    a ragged last pass) give the oracle's bits."""
    import oracle.shearwave_oracle as orc
    import shearwave_b200 as sw

    rng = np.random.default_rng(sum(shape))
    h = (0.5e-3, 0.7e-3, 0.9e-3)
    a, b, c = (rng.standard_normal(shape).astype(dt) for _ in range(3))
    assert np.array_equal(sw.laplacian_center(a, *h), orc.laplacian_center(a, *h))
    assert np.array_equal(sw.divergence_center(a, b, c, *h), orc.divergence_center(a, b, c, *h))
    for g, r in zip(sw.gradient_center(a, *h), orc.gradient_center(a, *h)):
        assert np.array_equal(g, r)
    eps = sw.compute_strain_tensor(a, b, c, *h)
    assert np.array_equal(eps, orc.compute_strain_tensor(a, b, c, *h))
    u = np.stack([a, b, c], axis=-1)
    eps2, inv2 = sw.compute_strain_fields(u, *h)
    assert np.array_equal(eps2, eps)
    ref_inv = orc.compute_strain_invariants(eps)
    for k, v in inv2.items():
        assert np.array_equal(v, ref_inv[k]), k
