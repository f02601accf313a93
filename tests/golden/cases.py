"""Seeded input cases shared by the golden-fixture generator and the tests.

Every input array is drawn in float64 and rounded to float32 once, so the
float32 run and the float64 run of a case see exactly the same values.
"""

from __future__ import annotations

import math

import numpy as np


def _f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def _axes(shape, h):
    """Cell-centre coordinates (metres), centred on the grid (indexing ij)."""
    ax = [(np.arange(n) - (n - 1) / 2.0) * hh for n, hh in zip(shape, h)]
    return np.meshgrid(*ax, indexing="ij")


def gaussian_push(shape, h, centre=(0.0, 0.0, 0.0), sig_lat=1.5e-3, sig_ax=5e-3, amp=1e3):
    """Axial (z) push: lateral sigma in x/y, axial sigma in z (config-0 shape)."""
    x, y, z = _axes(shape, h)
    cx, cy, cz = centre
    r2 = ((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig_lat**2) + (z - cz) ** 2 / (2 * sig_ax**2)
    return _f32(amp * np.exp(-r2))


def smooth_random(rng, shape, passes=2):
    """Random field smoothed by repeated 3-point box filters, peak 1."""
    a = rng.standard_normal(shape)
    for _ in range(passes):
        for ax in range(3):
            a = (np.roll(a, 1, ax) + a + np.roll(a, -1, ax)) / 3.0
    return a / np.max(np.abs(a))


CASES: dict[str, dict] = {
    "ops_a": {"kind": "operators", "shape": (9, 11, 13), "h": (0.5e-3, 0.7e-3, 0.9e-3), "seed": 3},
    "strain_a": {"kind": "strain", "shape": (12, 10, 14), "h": (1e-3, 1.1e-3, 0.9e-3), "seed": 4},
    "proj_taper_s0": {"kind": "projection", "n": 20, "h": 1.0 / 20, "tol": 1e-8,
                      "max_iters": 5000, "seed": 0, "field": "taper"},
    "proj_taper_s1": {"kind": "projection", "n": 20, "h": 1.0 / 20, "tol": 1e-8,
                      "max_iters": 5000, "seed": 1, "field": "taper"},
    "proj_blob": {"kind": "projection", "n": 22, "h": 0.5e-3, "tol": 1e-10,
                  "max_iters": 3000, "seed": 2, "field": "blob"},
    "static_a": {"kind": "static", "n": 16, "h": 1.0 / 16, "mu": 1000.0, "tol": 1e-8,
                 "max_iters": 5000},
    "fdtd_c0": {"kind": "fdtd", "shape": (16, 14, 20), "dX": 0.5e-3, "dY": 0.5e-3, "dZ": 0.5e-3,
                "dT": 20e-6, "n_steps": 60, "stride": 20, "seed": 0, "physics": "c0"},
    "fdtd_hetero": {"kind": "fdtd", "shape": (18, 16, 20), "dX": 0.5e-3, "dY": 0.45e-3,
                    "dZ": 0.55e-3, "dT": 10e-6, "n_steps": 50, "stride": 25, "seed": 5,
                    "physics": "hetero"},
    "fdtd_4d": {"kind": "fdtd", "shape": (16, 12, 16), "dX": 2e-4, "dY": 2e-4, "dZ": 2e-4,
                "dT": 0.15 * 2e-4 / (math.sqrt(4000.0 / 1000.0) * math.sqrt(3.0)),
                "n_steps": 24, "stride": 6, "seed": 0, "physics": "chirp4d"},
    "fdtd_reproject": {"kind": "fdtd", "shape": (14, 14, 14), "dX": 1e-3, "dY": 1e-3,
                       "dZ": 1e-3, "dT": 0.1 * 1e-3 / (math.sqrt(4.58) * math.sqrt(3.0)),
                       "n_steps": 30, "stride": 10, "seed": 0, "physics": "reproject"},
    "fdtd_initial": {"kind": "fdtd", "shape": (12, 14, 10), "dX": 0.5e-3, "dY": 0.5e-3,
                     "dZ": 0.5e-3, "dT": 10e-6, "n_steps": 15, "stride": 5, "seed": 7,
                     "physics": "initial"},
    # radiation force: a focused tone burst recorded on a small grid; the
    # auto gate (None), an explicit slice and an index array
    "arf_auto": {"kind": "radiation", "shape": (10, 9, 12), "nt": 48, "f0": 1.0e6, "seed": 11,
                 "gate": None},
    "arf_slice": {"kind": "radiation", "shape": (7, 8, 9), "nt": 40, "f0": 0.5e6, "seed": 12,
                  "gate": (6, 30, 2)},
    "arf_index": {"kind": "radiation", "shape": (6, 5, 11), "nt": 70, "f0": 2.0e6, "seed": 13,
                  "gate": [3, 4, 5, 9, 17, 33, 34, 60]},
    # validate_wavespeed.py at its default size (float32 reference run only:
    # the script runs the reference as shipped)
    "wavespeed_default": {"kind": "wavespeed", "f32_only": True},
}


def radiation_inputs(case, dtype):
    """Pressure and particle-velocity records (nx, ny, nz, nt), sound speed,
    density and attenuation maps, and the gate of one radiation-force case."""
    nx, ny, nz = case["shape"]
    nt = case["nt"]
    rng = np.random.default_rng(case["seed"])
    x, y, z = np.meshgrid(np.linspace(-1, 1, nx), np.linspace(-1, 1, ny), np.linspace(-1, 1, nz),
                          indexing="ij")
    t = np.arange(nt)
    burst = np.sin(2 * np.pi * 0.11 * t) * np.exp(-0.5 * ((t - 0.45 * nt) / (0.15 * nt)) ** 2)
    focus = np.exp(-2.0 * (x**2 + y**2) - 0.7 * z**2)[..., None]
    delay = (0.8 * z[..., None] * 4.0).astype(np.int64)
    p = 1e5 * focus * np.take(burst, np.clip(t[None, None, None, :] - delay, 0, nt - 1))
    p = p * (1.0 + 0.05 * rng.standard_normal(p.shape))
    rc = 1500.0 * (1.0 + 0.03 * rng.uniform(-1, 1, (nx, ny, nz)))
    rho = 1000.0 * (1.0 + 0.05 * rng.uniform(-1, 1, (nx, ny, nz)))
    alpha = 0.5 + 0.3 * rng.uniform(0, 1, (nx, ny, nz))
    v = [p / (rho * rc)[..., None] * w for w in (0.2 * x[..., None], 0.1 * y[..., None],
                                                  np.ones_like(z)[..., None])]
    v = [a * (1.0 + 0.05 * rng.standard_normal(a.shape)) for a in v]
    c = lambda a: _f32(a).astype(dtype)  # noqa: E731
    g = case["gate"]
    gate = None if g is None else (slice(*g) if isinstance(g, tuple) else np.asarray(g))
    return {"p": c(p), "vx": c(v[0]), "vy": c(v[1]), "vz": c(v[2]), "c": c(rc), "rho": c(rho),
            "alpha": c(alpha), "f0": case["f0"], "gate": gate}


def operator_inputs(case, dtype):
    rng = np.random.default_rng(case["seed"])
    return tuple(_f32(rng.standard_normal(case["shape"])).astype(dtype) for _ in range(3))


def strain_inputs(case, dtype):
    rng = np.random.default_rng(case["seed"])
    return tuple(_f32(1e-6 * smooth_random(rng, case["shape"])).astype(dtype) for _ in range(3))


def projection_inputs(case, dtype):
    n, h = case["n"], case["h"]
    rng = np.random.default_rng(case["seed"])
    if case["field"] == "taper":
        t = np.linspace(0.0, 1.0, n)
        taper = (np.sin(np.pi * t)[:, None, None] * np.sin(np.pi * t)[None, :, None]
                 * np.sin(np.pi * t)[None, None, :])
        f = [_f32(rng.standard_normal((n, n, n)) * taper) for _ in range(3)]
    else:
        bz = gaussian_push((n, n, n), (h, h, h), centre=(0.3e-3, -0.2e-3, 0.5e-3),
                           sig_lat=1.2e-3, sig_ax=2.5e-3)
        f = [np.zeros_like(bz), np.zeros_like(bz), bz]
    return tuple(a.astype(dtype) for a in f)


def static_inputs(case):
    n, d, mu = case["n"], case["h"], case["mu"]
    t = np.linspace(0.0, 1.0, n)
    u = (np.sin(np.pi * t)[:, None, None] * np.sin(np.pi * t)[None, :, None]
         * np.sin(np.pi * t)[None, None, :])
    u = _f32(u)
    lap = np.zeros_like(u)
    lap[1:-1, 1:-1, 1:-1] = sum(
        (np.roll(u, -1, ax) - 2 * u + np.roll(u, 1, ax))[1:-1, 1:-1, 1:-1] / d**2
        for ax in range(3)
    )
    return _f32(-mu * lap)


def fdtd_inputs(case, dtype):
    """Inputs of one shear_fdtd call: forces, materials and opts (arrays in ``dtype``)."""
    shape = case["shape"]
    h = (case["dX"], case["dY"], case["dZ"])
    n_steps = case["n_steps"]
    rng = np.random.default_rng(case["seed"])
    phys = case["physics"]
    c = lambda a: None if a is None else np.asarray(a).astype(dtype)  # noqa: E731
    opts: dict = {}
    bx = by = bz = None
    if phys == "c0":
        bz = gaussian_push(shape, h)
        env = np.zeros(n_steps, np.float32)
        env[:5] = 1.0
        rho, mu = 1000.0, 2000.0
        opts.update(eta=1.0, env_t=env, poisson_tol=1e-10, poisson_max_iters=2000)
    elif phys == "hetero":
        x, y, z = _axes(shape, h)
        rho = _f32(1000.0 * (1.0 + rng.uniform(-0.05, 0.05, shape)))
        mu = np.full(shape, 3e3)
        eta = np.full(shape, 1.0)
        for _ in range(2):
            cen = rng.uniform(-2e-3, 2e-3, 3)
            r = rng.uniform(1e-3, 2.5e-3)
            inside = (x - cen[0]) ** 2 + (y - cen[1]) ** 2 + (z - cen[2]) ** 2 < r * r
            mu[inside] = math.exp(rng.uniform(math.log(1e3), math.log(2e4)))
            eta[inside] = rng.uniform(0.5, 2.5)
        mu, eta = _f32(mu), _f32(eta)
        bx = gaussian_push(shape, h, centre=(1e-3, 0, 0), sig_lat=1e-3, sig_ax=2e-3, amp=300.0)
        by = gaussian_push(shape, h, centre=(0, -1e-3, 0.5e-3), sig_lat=1e-3, sig_ax=2e-3,
                           amp=-200.0)
        bz = gaussian_push(shape, h, centre=(-0.5e-3, 0.5e-3, 0), sig_lat=1.2e-3, sig_ax=3e-3)
        env = np.zeros(n_steps, np.float32)
        env[:8] = _f32(np.sin(np.pi * (np.arange(8) + 0.5) / 8.0))
        opts.update(eta=eta, env_t=env, vel_damp=0.02, poisson_tol=1e-10,
                    poisson_max_iters=2000)
    elif phys == "chirp4d":
        nx, ny, nz = shape
        xg, yg, zg = np.meshgrid(np.arange(nx) - nx // 2, np.arange(ny) - ny // 2,
                                 np.arange(nz) - nz // 2, indexing="ij")
        b3 = np.exp(-0.5 * ((xg / 3.0) ** 2 + (yg / 3.0) ** 2 + (zg / 3.0) ** 2))
        b3 = _f32(0.03 * b3 / np.max(b3))
        t = np.arange(n_steps, dtype=np.float64)
        env = _f32(np.sin(2 * np.pi * 0.07 * t) * (1.0 + 0.5 * np.cos(2 * np.pi * 0.19 * t)))
        bz = _f32(b3[..., None].astype(np.float64) * env[None, None, None, :].astype(np.float64))
        rho, mu = 1000.0, 4000.0
        opts.update(vel_damp=0.0, poisson_tol=5e-5, poisson_max_iters=120)
    elif phys == "reproject":
        bx = gaussian_push(shape, h, sig_lat=2.5e-3, sig_ax=2.5e-3, amp=300.0)
        env = np.zeros(n_steps, np.float32)
        env[: n_steps // 3] = 1.0
        rho, mu = 1000.0, 4580.0
        opts.update(eta=0.5, vel_damp=0.02, env_t=env, reproject_every=10, poisson_tol=1e-8,
                    poisson_max_iters=1000)
    elif phys == "initial":
        bz = np.zeros(shape, np.float32)
        env = np.ones(n_steps, np.float32)
        rho, mu = 1000.0, 2500.0
        iu = np.stack([1e-6 * smooth_random(rng, shape) for _ in range(3)], axis=-1)
        iv = np.stack([1e-4 * smooth_random(rng, shape) for _ in range(3)], axis=-1)
        opts.update(eta=0.8, env_t=env, initial_u=_f32(iu).astype(dtype),
                    initial_v=_f32(iv).astype(dtype), poisson_tol=1e-10, poisson_max_iters=500)
    else:  # pragma: no cover - guarded by CASES
        raise KeyError(phys)
    if isinstance(rho, np.ndarray):
        rho = c(rho)
    if isinstance(mu, np.ndarray):
        mu = c(mu)
    if isinstance(opts.get("eta"), np.ndarray):
        opts["eta"] = c(opts["eta"])
    if "env_t" in opts:
        opts["env_t"] = np.asarray(opts["env_t"]).astype(dtype)
    return {"bx": c(bx), "by": c(by), "bz": c(bz), "rho": rho, "mu": mu, "opts": opts}
