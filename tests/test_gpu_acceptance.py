"""The reference's own acceptance tests, restated against the CUDA path.

pinton-lab/shearwave ships four test modules whose checks are analytic
(known answers and physical invariants, no fixtures).  Each test here
restates one of them -- same setup, same quantity, same threshold, cited by
file and line -- and runs it through ``shearwave_b200`` (both forms where the
reference's own run is FP32).  The reference's JAX-only snapshot tests are
re-targeted: the JAX solver is replaced by this package's
``snapshot_stride`` path and the NumPy callback side by the CPU oracle (the
reference's NumPy loop restated, in float32 as it ships).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECISIONS = ["mixed", "fp64"]


# ---------------------------------------------------------------------------
# tests/test_divergence_free.py:72-111 -- the stepped displacement stays
# solenoidal until the wall signal arrives; reproject_every keeps it so
# ---------------------------------------------------------------------------
DIV_TOL = 1e-4  # tests/test_divergence_free.py:27


def _div_curl_ratio(u, d):
    """RMS(div u) / RMS(|curl u|) over the inner half-cube, 2h central
    differences (one-sided at the edges), as tests/test_divergence_free.py:30-42."""
    jac = [np.gradient(np.asarray(u[..., c], np.float64), d, d, d, edge_order=1)
           for c in range(3)]
    div = jac[0][0] + jac[1][1] + jac[2][2]
    curl = np.sqrt((jac[2][1] - jac[1][2]) ** 2 + (jac[0][2] - jac[2][0]) ** 2
                   + (jac[1][0] - jac[0][1]) ** 2)
    n = u.shape[0]
    inner = (slice(n // 4, n - n // 4),) * 3
    return float(np.sqrt(np.mean(div[inner] ** 2)) / np.sqrt(np.mean(curl[inner] ** 2)))


def _cube_push(n=32, d=1.0e-3, mu=4580.0, rho=1000.0):
    """Axial Gaussian push (sigma 2.5 voxels, 300 N/m^3 on bx) at the centre of
    an n^3 cube, dt = 0.1 d / (c_s sqrt 3) (tests/test_divergence_free.py:45-55)."""
    ax = (np.arange(n) - (n - 1) / 2) * d
    x, y, z = np.meshgrid(ax, ax, ax, indexing="ij")
    bx = (300.0 * np.exp(-(x**2 + y**2 + z**2) / (2 * (2.5 * d) ** 2))).astype(np.float32)
    cs = math.sqrt(mu / rho)
    dt = 0.1 * d / (cs * math.sqrt(3.0))
    return bx, mu, rho, d, dt, d / (cs * dt)


def _ratios(n, arrivals, opts, precision, every=20):
    import shearwave_b200 as sw

    bx, mu, rho, d, dt, steps_per_voxel = _cube_push(n)
    n_steps = int(arrivals * (n // 4) * steps_per_voxel)
    env = np.zeros(n_steps, np.float32)
    env[: max(1, n_steps // 3)] = 1.0
    out = []

    def cb(it, u):
        if it % every == every - 1:
            out.append((it, _div_curl_ratio(u, d)))

    sw.shear_fdtd(bx, None, None, rho, mu, d, d, d, dt, n_steps,
                  opts={**opts, "env_t": env, "precision": precision}, callback=cb)
    assert out, "run too short to sample"
    return [r for _, r in out]


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("damped", [False, True])
def test_point_force_stays_solenoidal(cuda, precision, damped):
    """tests/test_divergence_free.py:72-84: half the wall-arrival time."""
    opts = {"vel_damp": 0.02 if damped else 0.0, "eta": 0.5 if damped else 0.0}
    assert max(_ratios(32, 0.5, opts, precision)) < DIV_TOL


@pytest.mark.parametrize("precision", PRECISIONS)
def test_wall_injects_divergence(cuda, precision):
    """tests/test_divergence_free.py:87-93: after arrival the wall signal dominates."""
    assert max(_ratios(32, 1.5, {"vel_damp": 0.02, "eta": 0.5}, precision)) > 1e-2


@pytest.mark.parametrize("precision", PRECISIONS)
def test_reproject_every_bounds_divergence(cuda, precision):
    """tests/test_divergence_free.py:96-102: reproject_every=20 for 3 arrival times."""
    opts = {"vel_damp": 0.02, "eta": 0.5, "reproject_every": 20}
    assert max(_ratios(32, 3.0, opts, precision)) < DIV_TOL


# ---------------------------------------------------------------------------
# tests/test_projection_static.py:45-129 -- projection and static-solve KATs
# ---------------------------------------------------------------------------
def _unit_grid(n=32):
    """tests/test_projection_static.py:26-34: linspace(0, 1, n) axes, d = 1/n."""
    ax = np.linspace(0.0, 1.0, n, dtype=np.float32)
    mask = np.zeros((n, n, n), np.float32)
    mask[1:-1, 1:-1, 1:-1] = 1.0
    return n, 1.0 / n, ax[:, None, None], ax[None, :, None], ax[None, None, :], mask


def _max_div(f, d, mask):
    from oracle import shearwave_oracle as O

    return float(np.max(np.abs(O.divergence_center(*f, d, d, d) * mask)))


def _energy(f, mask):
    return float(np.sum((f[0] ** 2 + f[1] ** 2 + f[2] ** 2) * mask))


METHODS = ["cg", "spectral"]


@pytest.mark.parametrize("method", METHODS)
def test_projection_removes_pure_gradient(cuda, method):
    """tests/test_projection_static.py:45-54."""
    import shearwave_b200 as sw

    n, d, x, y, z, mask = _unit_grid()
    psi = (np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)).astype(
        np.float32) * np.ones((n, n, n), np.float32)
    g = [a.astype(np.float32) for a in sw.gradient_center(psi, d, d, d)]
    out = sw.project_vector_field(*g, d, d, d, 1e-9, 5000, method=method)
    assert _energy(out, mask) / _energy(g, mask) < 1e-3


@pytest.mark.parametrize("method", METHODS)
def test_projection_preserves_solenoidal_field(cuda, method):
    """tests/test_projection_static.py:57-70: f = curl(a_x, 0, a_z)."""
    import shearwave_b200 as sw

    n, d, x, y, z, mask = _unit_grid()
    a_x = (np.sin(2 * np.pi * y) * np.sin(2 * np.pi * z)).astype(np.float32) * np.ones_like(x)
    a_z = (np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y)).astype(np.float32) * np.ones_like(z)
    gx = sw.gradient_center(a_x, d, d, d)
    gz = sw.gradient_center(a_z, d, d, d)
    f = [gz[1].astype(np.float32), (gx[2] - gz[0]).astype(np.float32),
         (-gx[1]).astype(np.float32)]
    out = sw.project_vector_field(*f, d, d, d, 1e-9, 5000, method=method)
    assert _energy(out, mask) / _energy(f, mask) > 0.98


@pytest.mark.parametrize("method", METHODS)
def test_projection_output_is_divergence_free(cuda, method):
    """tests/test_projection_static.py:73-83: a tapered blob."""
    import shearwave_b200 as sw

    n, d, x, y, z, mask = _unit_grid()
    blob = np.exp(-(((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) / (2 * 0.08**2))).astype(
        np.float32) * np.ones((n, n, n), np.float32)
    zero = np.zeros_like(blob)
    before = _max_div((zero, zero, blob), d, mask)
    out = sw.project_vector_field(zero, zero, blob, d, d, d, 1e-9, 5000, method=method)
    assert _max_div(out, d, mask) < 1e-3 * before


def test_static_solver_recovers_manufactured_solution(cuda):
    """tests/test_projection_static.py:86-105: mu lap(u) = -bz for a sine bump."""
    import shearwave_b200 as sw

    n, d, x, y, z, mask = _unit_grid()
    mu = 1000.0
    u_true = (np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)).astype(
        np.float32) * np.ones((n, n, n), np.float32)
    lap = np.zeros_like(u_true)
    c = u_true[1:-1, 1:-1, 1:-1]
    lap[1:-1, 1:-1, 1:-1] = (
        (u_true[2:, 1:-1, 1:-1] - 2 * c + u_true[:-2, 1:-1, 1:-1]) / d**2
        + (u_true[1:-1, 2:, 1:-1] - 2 * c + u_true[1:-1, :-2, 1:-1]) / d**2
        + (u_true[1:-1, 1:-1, 2:] - 2 * c + u_true[1:-1, 1:-1, :-2]) / d**2)
    u = sw.elastic_solve_static((-mu * lap).astype(np.float32), d, d, d, mu, tol=1e-8,
                                max_iters=5000)
    assert np.max(np.abs(u)) > 0.0
    assert np.max(np.abs((u - u_true) * mask)) / np.max(np.abs(u_true * mask)) < 1e-3


@pytest.mark.parametrize("seed", [0, 1])
def test_projection_backend_parity_is_divergence_free(cuda, seed):
    """tests/test_projection_static.py:108-129, re-targeted: the CUDA path
    against the NumPy algorithm (the oracle) instead of JAX against NumPy."""
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O

    n, d, x, y, z, mask = _unit_grid(24)
    rng = np.random.default_rng(seed)
    taper = (np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)).astype(np.float32)
    f = [rng.standard_normal((n, n, n)).astype(np.float32) * taper for _ in range(3)]
    ref = O.project_vector_field(*(a.copy() for a in f), d, d, d, 1e-8, 5000)
    got = sw.project_vector_field(*(a.copy() for a in f), d, d, d, 1e-8, 5000)
    assert np.max(np.abs(ref[0] - got[0])) / (np.max(np.abs(ref[0])) + 1e-20) < 1e-2
    div_in = _max_div(f, d, mask)
    assert _max_div(ref, d, mask) < 1e-2 * div_in
    assert _max_div(got, d, mask) < 1e-2 * div_in


# ---------------------------------------------------------------------------
# tests/test_strain.py:19-149 -- strain tensor and invariant KATs
# ---------------------------------------------------------------------------
def test_strain_uniform_displacement_is_zero(cuda):
    """tests/test_strain.py:22-34."""
    import shearwave_b200 as sw

    n, h = 20, 1e-3
    one = np.ones((n, n, n), np.float64)
    eps = sw.compute_strain_tensor(3.0 * one, -1.0 * one, 0.5 * one, h, h, h)
    assert eps.shape == (n, n, n, 6)
    np.testing.assert_allclose(eps[2:-2, 2:-2, 2:-2, :], 0.0, atol=1e-14)


def test_strain_linear_uniaxial(cuda):
    """tests/test_strain.py:36-54: u_x = a x gives eps_xx = a."""
    import shearwave_b200 as sw

    n, h, a = 20, 1e-3, 0.01
    ux = np.zeros((n, n, n), np.float64)
    ux[:] = (np.arange(n) * h)[:, None, None] * a
    eps = sw.compute_strain_tensor(ux, np.zeros_like(ux), np.zeros_like(ux), h, h, h)
    np.testing.assert_allclose(eps[2:-2, 2:-2, 2:-2, 0], a, rtol=1e-10)
    for k in range(1, 6):
        np.testing.assert_allclose(eps[2:-2, 2:-2, 2:-2, k], 0.0, atol=1e-14)


def test_strain_pure_shear_xy(cuda):
    """tests/test_strain.py:56-76: u_x = b y, u_y = b x give gamma_xy = 2 b."""
    import shearwave_b200 as sw

    n, h, b = 20, 1e-3, 0.005
    ux = np.zeros((n, n, n), np.float64)
    uy = np.zeros_like(ux)
    ux[:] = b * (np.arange(n) * h)[None, :, None]
    uy[:] = b * (np.arange(n) * h)[:, None, None]
    eps = sw.compute_strain_tensor(ux, uy, np.zeros_like(ux), h, h, h)
    np.testing.assert_allclose(eps[2:-2, 2:-2, 2:-2, 5], 2.0 * b, rtol=1e-10)
    for k in range(3):
        np.testing.assert_allclose(eps[2:-2, 2:-2, 2:-2, k], 0.0, atol=1e-14)


def test_strain_input_errors(cuda):
    """tests/test_strain.py:78-88 (messages)."""
    import shearwave_b200 as sw

    z = np.zeros((10, 10, 10))
    with pytest.raises(ValueError, match="same shape"):
        sw.compute_strain_tensor(z, np.zeros((10, 10, 11)), z, 1e-3, 1e-3, 1e-3)
    with pytest.raises(ValueError, match="positive"):
        sw.compute_strain_tensor(z, z, z, -1e-3, 1e-3, 1e-3)


def test_invariants_pure_dilation(cuda):
    """tests/test_strain.py:95-112."""
    import shearwave_b200 as sw

    eps = np.zeros((10, 10, 10, 6))
    eps[..., :3] = 0.01
    inv = sw.compute_strain_invariants(eps)
    np.testing.assert_allclose(inv["volumetric"], 0.01, rtol=1e-12)
    for k in ("deviatoric", "von_mises", "max_shear"):
        np.testing.assert_allclose(inv[k], 0.0, atol=1e-14)


def test_invariants_pure_shear(cuda):
    """tests/test_strain.py:114-125."""
    import shearwave_b200 as sw

    eps = np.zeros((10, 10, 10, 6))
    eps[..., 5] = 0.02
    inv = sw.compute_strain_invariants(eps)
    np.testing.assert_allclose(inv["volumetric"], 0.0, atol=1e-14)
    assert np.all(inv["deviatoric"] > 0) and np.all(inv["von_mises"] > 0)


def test_invariants_uniaxial_von_mises(cuda):
    """tests/test_strain.py:127-143: von Mises of uniaxial e is 2e/3."""
    import shearwave_b200 as sw

    eps = np.zeros((10, 10, 10, 6))
    eps[..., 0] = 0.03
    inv = sw.compute_strain_invariants(eps)
    np.testing.assert_allclose(inv["von_mises"][5, 5, 5], 0.03 * 2.0 / 3.0, rtol=1e-10)


def test_invariants_last_dim_error(cuda):
    """tests/test_strain.py:145-149."""
    import shearwave_b200 as sw

    with pytest.raises(ValueError, match="Voigt"):
        sw.compute_strain_invariants(np.zeros((5, 5, 5, 3)))


# ---------------------------------------------------------------------------
# tests/test_snapshot_stride.py:73-210 -- snapshots, re-targeted
# ---------------------------------------------------------------------------
def _chirp_problem(nx=16, ny=12, nz=16, n_steps=24):
    """tests/test_snapshot_stride.py:18-52: a chirp-modulated Gaussian push."""
    rho, mu, h = 1000.0, 4000.0, 2.0e-4
    dT = 0.15 * h / (math.sqrt(mu / rho) * math.sqrt(3.0))
    xg, yg, zg = np.meshgrid(np.arange(nx) - nx // 2, np.arange(ny) - ny // 2,
                             np.arange(nz) - nz // 2, indexing="ij")
    b3 = np.exp(-0.5 * ((xg / 3.0) ** 2 + (yg / 3.0) ** 2 + (zg / 3.0) ** 2)).astype(np.float32)
    b3 = b3 / np.max(b3) * np.float32(0.03)
    t = np.arange(n_steps, dtype=np.float32)
    env = (np.sin(2.0 * np.pi * 0.07 * t) * (1.0 + 0.5 * np.cos(2.0 * np.pi * 0.19 * t))).astype(
        np.float32)
    b4 = (b3[..., None] * env[None, None, None, :]).astype(np.float32)
    opts = {"vel_damp": 0.0, "poisson_tol": 5e-5, "poisson_max_iters": 120, "verbose": False}
    grid = {"rho": rho, "mu": mu, "dX": h, "dY": h, "dZ": h, "dT": dT, "n_steps": n_steps}
    return b3, env, b4, opts, grid


def _oracle_callback_snapshots(b4, opts, grid, stride):
    """The reference's NumPy path collecting snapshots through its callback
    (tests/test_snapshot_stride.py:55-70), in float32 as it ships."""
    from oracle import shearwave_oracle as O

    snaps = []

    def cb(it, u):
        if (it + 1) % stride == 0:
            snaps.append(np.array(u, copy=True))

    u, _v = O.shear_fdtd(None, None, b4, grid["rho"], grid["mu"], grid["dX"], grid["dY"],
                         grid["dZ"], grid["dT"], grid["n_steps"], opts=opts, callback=cb)
    return u, np.stack(snaps)


@pytest.mark.parametrize("stride", [4, 6])
def test_snapshot_stride_matches_callback_4d(cuda, stride):
    """tests/test_snapshot_stride.py:73-92."""
    import shearwave_b200 as sw

    _b3, _env, b4, opts, grid = _chirp_problem()
    u_np, np_snaps = _oracle_callback_snapshots(b4, opts, grid, stride)
    u, _v, snaps = sw.shear_fdtd_jax(None, None, b4, opts={**opts, "jit": True},
                                     snapshot_stride=stride, **grid)
    assert snaps.shape == (grid["n_steps"] // stride, *u_np.shape)
    scale = float(np.max(np.abs(u_np))) + 1e-30
    assert np.max(np.abs(np_snaps - snaps)) < 1e-3 * scale
    assert np.max(np.abs(u_np - u)) < 1e-3 * scale


def test_snapshot_stride_matches_callback_separable(cuda):
    """tests/test_snapshot_stride.py:95-111."""
    import shearwave_b200 as sw

    b3, env, b4, opts, grid = _chirp_problem()
    u_np, np_snaps = _oracle_callback_snapshots(b4, opts, grid, 6)
    u, _v, snaps = sw.shear_fdtd_jax(None, None, b3, opts={**opts, "jit": True, "env_t": env},
                                     snapshot_stride=6, **grid)
    assert snaps.shape == (grid["n_steps"] // 6, *u_np.shape)
    scale = float(np.max(np.abs(u_np))) + 1e-30
    assert np.max(np.abs(np_snaps - snaps)) < 1e-3 * scale
    assert np.max(np.abs(u_np - u)) < 1e-3 * scale


def test_snapshot_stride_separable_matches_4d(cuda):
    """tests/test_snapshot_stride.py:114-137."""
    import shearwave_b200 as sw

    b3, env, b4, opts, grid = _chirp_problem()
    _u, _v, s4 = sw.shear_fdtd_jax(None, None, b4, opts={**opts, "jit": True},
                                   snapshot_stride=6, **grid)
    _u, _v, ss = sw.shear_fdtd_jax(None, None, b3, opts={**opts, "jit": True, "env_t": env},
                                   snapshot_stride=6, **grid)
    assert s4.shape == ss.shape
    assert np.max(np.abs(s4 - ss)) < 1e-5 * (float(np.max(np.abs(s4))) + 1e-30)


def test_snapshot_stride_device_arrays(cuda):
    """tests/test_snapshot_stride.py:140-156: device outputs are torch CUDA tensors."""
    import torch

    import shearwave_b200 as sw

    b3, env, _b4, opts, grid = _chirp_problem()
    out = sw.shear_fdtd_jax(None, None, b3, opts={**opts, "jit": True, "env_t": env},
                            snapshot_stride=6, return_device=True, **grid)
    assert len(out) == 3
    assert all(isinstance(t, torch.Tensor) and t.is_cuda for t in out)


def test_snapshot_stride_errors_and_default_contract(cuda):
    """tests/test_snapshot_stride.py:159-210."""
    import shearwave_b200 as sw

    b3, env, _b4, opts, grid = _chirp_problem()
    o = {**opts, "jit": True, "env_t": env}
    with pytest.raises(ValueError, match=r"multiple of snapshot_stride"):
        sw.shear_fdtd_jax(None, None, b3, opts=o, snapshot_stride=5, **grid)
    with pytest.raises(ValueError, match=r"positive integer"):
        sw.shear_fdtd_jax(None, None, b3, opts=o, snapshot_stride=0, **grid)
    with pytest.raises(ValueError, match=r"not both supported"):
        sw.shear_fdtd_jax(None, None, b3, opts=o, snapshot_stride=6, return_traces=True,
                          trace_indices=([0], [0], [0]), **grid)
    b3, env, _b4, opts, grid = _chirp_problem(n_steps=12)
    assert len(sw.shear_fdtd_jax(None, None, b3, opts={**opts, "env_t": env}, **grid)) == 2
