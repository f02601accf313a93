"""Seeded synthetic shear_fdtd problems with the shapes of the benchmark configs.

The reference publishes no benchmark dataset; these generators stand in for
it with the documented shapes, sizes and value distributions:

* ``c0`` 64^3 homogeneous medium, centred Gaussian axial push, nT=500;
* ``c1`` 192^3 heterogeneous medium (rho +-5 %, 12 seeded spherical
  inclusions), seeded push location, nT=2000, snapshot stride 10;
* ``c2`` 256x256x384 layered medium (5 mm stiff slab over soft tissue with
  smooth +-10 % variation), 8 seeded sparse pushes, nT=4000;
* ``c3`` 48 independent solves with seeded grids 64^3 .. 160x160x224 and
  nT in [500, 3000];
* ``c4`` serving requests: log-uniform grids 64^3 .. 256^3, 1 or 4 pushes,
  nT in [500, 4000].

Explicit viscous time stepping is stable only for
``dT * eta * 12 / (rho h^2) <= 2``; configs drawing eta up to 5 Pa s at
h = 0.5 mm therefore clamp dT per instance to
``min(dT, 0.9 rho_min h^2 / (6 eta_max))`` (and to the elastic CFL limit).
A problem is a dict of ``shear_fdtd`` keyword arguments (numpy float32
arrays) plus ``name``.
"""

from __future__ import annotations

import math

import numpy as np

H = 0.5e-3  # grid spacing of every config [m]


def _f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def _coords(shape, h=H):
    ax = [np.arange(n) * h for n in shape]
    return np.meshgrid(*ax, indexing="ij")


def gaussian_push(shape, centre, sig_lat=1.5e-3, sig_ax=5e-3, amp=1e3, h=H):
    """Axial (z) Gaussian body force centred at ``centre`` (metres from cell 0)."""
    x, y, z = _coords(shape, h)
    cx, cy, cz = centre
    r2 = ((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig_lat**2) + (z - cz) ** 2 / (2 * sig_ax**2)
    return _f32(amp * np.exp(-r2))


def inclusion_medium(rng, shape, n_inc=12, h=H):
    """rho +-5 % noise; 12 spheres (radius 2-8 mm, mu log-uniform 1-20 kPa, eta 0.5-5).

    Spheres are painted in order (later ones overwrite earlier ones); each is
    evaluated on its bounding box only.
    """
    L = np.array(shape) * h
    rho = _f32(1000.0 * (1.0 + rng.uniform(-0.05, 0.05, shape)))
    mu = np.full(shape, 3e3, dtype=np.float32)
    eta = np.full(shape, 1.0, dtype=np.float32)
    for _ in range(n_inc):
        c = rng.uniform(0.0, 1.0, 3) * L
        r = rng.uniform(2e-3, 8e-3)
        mu_i = math.exp(rng.uniform(math.log(1e3), math.log(2e4)))
        eta_i = rng.uniform(0.5, 5.0)
        lo = [max(0, int(math.floor((c[a] - r) / h)) - 1) for a in range(3)]
        hi = [min(shape[a], int(math.ceil((c[a] + r) / h)) + 2) for a in range(3)]
        if any(hi[a] <= lo[a] for a in range(3)):
            continue
        ax = [np.arange(lo[a], hi[a]) * h - c[a] for a in range(3)]
        d2 = (ax[0][:, None, None] ** 2 + ax[1][None, :, None] ** 2 + ax[2][None, None, :] ** 2)
        inside = d2 < r * r
        box = tuple(slice(lo[a], hi[a]) for a in range(3))
        mu[box][inside] = np.float32(mu_i)
        eta[box][inside] = np.float32(eta_i)
    return rho, mu, eta


def stable_dt(rho, mu, eta, dt_max, cfl=None, h=H):
    """dT clamped by the viscous limit (and the elastic CFL number when given)."""
    rho_min = float(np.min(rho))
    eta_max = float(np.max(eta)) if np.ndim(eta) else float(eta)
    dt = dt_max
    if eta_max > 0:
        dt = min(dt, 0.9 * rho_min * h * h / (6.0 * eta_max))
    if cfl is not None:
        cs_max = math.sqrt(float(np.max(mu)) / rho_min)
        dt = min(dt, cfl * h / (cs_max * math.sqrt(3.0)))
    return dt


def _envelope(n_steps, on=10, start=0):
    env = np.zeros(n_steps, np.float32)
    env[start:start + on] = 1.0
    return env


def problem_c0():
    shape = (64, 64, 64)
    c = [(n - 1) / 2 * H for n in shape]
    bz = gaussian_push(shape, c)
    n_steps = 500
    return {
        "name": "c0", "bx": None, "by": None, "bz": bz, "rho": 1000.0, "mu": 2000.0,
        "dX": H, "dY": H, "dZ": H, "dT": 20e-6, "n_steps": n_steps,
        "opts": {"eta": 1.0, "env_t": _envelope(n_steps, 5), "poisson_tol": 1e-10,
                 "poisson_max_iters": 2000},
        "snapshot_stride": 10,
    }


def problem_inclusions(shape, n_steps, seed, stride=None, tol=1e-10, cfl=None):
    """A config-1 style problem on ``shape`` (also used by c3 and c4)."""
    rng = np.random.default_rng(seed)
    rho, mu, eta = inclusion_medium(rng, shape)
    L = np.array(shape) * H
    centre = (0.25 + 0.5 * rng.uniform(0.0, 1.0, 3)) * L
    bz = gaussian_push(shape, centre)
    dT = stable_dt(rho, mu, eta, 10e-6, cfl=cfl)
    p = {
        "name": f"inclusions{shape}", "bx": None, "by": None, "bz": bz, "rho": rho, "mu": mu,
        "dX": H, "dY": H, "dZ": H, "dT": dT, "n_steps": int(n_steps),
        "opts": {"eta": eta, "env_t": _envelope(n_steps, 10), "poisson_tol": tol,
                 "poisson_max_iters": 3 * max(shape)},
    }
    if stride:
        p["snapshot_stride"] = stride
    return p


def problem_c1(seed=0, n_steps=2000, shape=(192, 192, 192)):
    p = problem_inclusions(shape, n_steps, seed, stride=10)
    p["name"] = "c1"
    return p


def problem_c2(seed=0, n_steps=4000, shape=(256, 256, 384), n_push=8):
    """Config 2: a 5 mm stiff slab (z in [2.5, 7.5) mm; mu 500 kPa, eta 2, rho
    1900) over soft tissue (mu 2 kPa, eta 1, rho 1040), every map scaled by
    (1 + 0.1 s) with s Gaussian-filtered white noise (sigma 4 voxels, max
    |s| = 1); 8 pushes (sigma 1 mm lateral, 4 mm axial, 1e3 N/m^3) centred in
    the soft region, each on for 20 steps (100 us) from a start in
    [0, nT/4); dT 5 us.
    """
    from scipy.ndimage import gaussian_filter

    rng = np.random.default_rng(seed)
    nz = shape[2]
    zc = (np.arange(nz) + 0.5) * H
    slab = (zc >= 2.5e-3) & (zc < 7.5e-3)
    mu = np.where(slab, 500e3, 2e3)[None, None, :] * np.ones(shape)
    eta = np.where(slab, 2.0, 1.0)[None, None, :] * np.ones(shape)
    rho = np.where(slab, 1900.0, 1040.0)[None, None, :] * np.ones(shape)
    sm = gaussian_filter(rng.standard_normal(shape).astype(np.float32), sigma=4.0)
    sm /= np.max(np.abs(sm))
    var = 1.0 + 0.1 * sm
    mu, eta, rho = _f32(mu * var), _f32(eta * var), _f32(rho * var)
    L = np.array(shape) * H
    pushes = []
    for _ in range(n_push):
        c = np.array([rng.uniform(0.25, 0.75) * L[0], rng.uniform(0.25, 0.75) * L[1],
                      rng.uniform(9e-3, L[2] - 4e-3)])
        start = int(rng.integers(0, max(1, n_steps // 4)))
        pushes.append((gaussian_push(shape, c, sig_lat=1e-3, sig_ax=4e-3),
                       _envelope(n_steps, 20, start)))
    opts = {"eta": eta, "env_t": pushes[0][1], "poisson_tol": 1e-10,
            "poisson_max_iters": 3 * max(shape),
            "force_terms": [((None, None, b), env) for b, env in pushes[1:]]}
    return {"name": "c2", "bx": None, "by": None, "bz": pushes[0][0], "rho": rho, "mu": mu,
            "dX": H, "dY": H, "dZ": H, "dT": 5e-6, "n_steps": int(n_steps), "opts": opts}


def batch_c3(seed=0, n=48, shrink=1.0):
    """48 seeded instances: grids U(64,160) x U(64,160) x U(64,224), nT U[500,3000].

    ``shrink`` scales grid extents and nT down (for quick tests).
    """
    probs = []
    for i in range(n):
        rng = np.random.default_rng(1000 * seed + i)
        shape = (int(round(rng.uniform(64, 160) * shrink)), int(round(rng.uniform(64, 160) * shrink)),
                 int(round(rng.uniform(64, 224) * shrink)))
        shape = tuple(max(8, s) for s in shape)
        n_steps = max(10, int(round(int(rng.integers(500, 3001)) * shrink)))
        p = problem_inclusions(shape, n_steps, 1000 * seed + i, cfl=0.2)
        p["name"] = f"c3[{i}]"
        probs.append(p)
    return probs


def problem_c4(rng):
    """One serving request (config 4): log-uniform cubic grid, 1 or 4 pushes."""
    n = int(round(math.exp(rng.uniform(math.log(64), math.log(256)))))
    shape = (n, n, n)
    n_steps = int(rng.integers(500, 4001))
    seed = int(rng.integers(0, 2**31 - 1))
    p = problem_inclusions(shape, n_steps, seed, cfl=0.2)
    if rng.uniform() < 0.5:
        # 4 pushes at seeded locations and start steps: extra separable terms
        r2 = np.random.default_rng(seed + 1)
        L = np.array(shape) * H
        terms = []
        for k in range(3):
            c = (0.25 + 0.5 * r2.uniform(0.0, 1.0, 3)) * L
            start = int(r2.integers(0, max(1, n_steps // 4)))
            terms.append(((None, None, gaussian_push(shape, c)), _envelope(n_steps, 10, start)))
        p["opts"]["force_terms"] = terms
    p["name"] = f"c4[{n}^3,{n_steps}]"
    return p


def cell_steps(p) -> int:
    """Cell-steps of one problem: nx*ny*nz*nT."""
    ref = p["bx"] if p["bx"] is not None else (p["by"] if p["by"] is not None else p["bz"])
    nx, ny, nz = ref.shape[:3]
    return int(nx) * int(ny) * int(nz) * int(p["n_steps"])
