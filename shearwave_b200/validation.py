"""Physics acceptance checks on the GPU solver, headless.

Two checks from the reference's validation scripts, restated for this
package (no plots, no movie frames; results come back as dicts):

* :func:`wavespeed_recovery` — validation/validate_wavespeed.py:21-205: a
  divergence-free initial velocity (the curl of a Hann-tapered Gaussian
  vector potential) launches shear waves; z-displacement traces at sensors
  along x give arrival times (peak |du_z/dt| after half the expected
  travel time), and a straight-line fit of distance against arrival time
  recovers the shear speed, to compare with sqrt(mu/rho).  The traces come
  from the solver's on-device trace recorder (``trace_indices``), not from a
  per-step host callback.
* :func:`quasistatic` — validation/validate_quasistatic.py:21-108: a constant
  shear-projected body force with strong velocity damping drives the time
  loop to the static solution of mu L7(u) = -b, which
  :func:`elastic_solve_static` computes directly; the check is their
  relative L2 difference (the script passes below 5e-2).
"""

from __future__ import annotations

import math

import numpy as np

from .solver import elastic_solve_static, hann1d, project_body_force_to_shear, shear_fdtd

__all__ = ["wavespeed_setup", "wavespeed_recovery", "quasistatic", "arrival_analysis"]


def _centred_grid(nx, ny, nz):
    return np.meshgrid(np.arange(nx) - nx // 2, np.arange(ny) - ny // 2,
                       np.arange(nz) - nz // 2, indexing="ij")


def _tapered_gaussian(nx, ny, nz, sig_xy, sig_z):
    xg, yg, zg = _centred_grid(nx, ny, nz)
    g = np.exp(-0.5 * ((xg / sig_xy) ** 2 + (yg / sig_xy) ** 2 + (zg / sig_z) ** 2))
    g = g.astype(np.float32)
    g /= np.max(g)
    return g * (hann1d(nx)[:, None, None] * hann1d(ny)[None, :, None] * hann1d(nz)[None, None, :])


def arrival_analysis(traces, dT, distances, cs_expected):
    """Arrival time per sensor and fitted speed from displacement traces.

    ``traces`` (n_sensors, n_steps) of u_z.  The velocity proxy is the
    first difference / dT; a sensor's arrival is the step of its largest
    |velocity| at or after half the expected travel time
    (validate_wavespeed.py:160-192).  Returns arrival times, per-sensor
    speeds, their mean and the slope of a least-squares line through
    (arrival time, distance).
    """
    traces = np.asarray(traces, dtype=np.float64)
    distances = np.asarray(distances, dtype=np.float64)
    n_steps = traces.shape[1]
    vel = np.diff(traces, axis=1) / dT
    t_after = (np.arange(1, n_steps) * dT)  # time of each velocity sample
    arrival_idx = np.full(len(distances), np.nan)
    for i, dist in enumerate(distances):
        first = int(np.searchsorted(t_after, 0.5 * dist / cs_expected))
        if first >= vel.shape[1]:
            continue
        arrival_idx[i] = first + int(np.argmax(np.abs(vel[i, first:])))
    arrival_t = (arrival_idx + 1) * dT
    ok = np.isfinite(arrival_idx)
    speeds = np.full(len(distances), np.nan)
    speeds[ok] = distances[ok] / arrival_t[ok]
    c_fit = float(np.polyfit(arrival_t[ok], distances[ok], 1)[0]) if ok.sum() >= 2 else math.nan
    return {"arrival_idx": arrival_idx, "arrival_times": arrival_t, "speeds": speeds,
            "mean_speed": float(np.nanmean(speeds)) if ok.any() else math.nan,
            "c_fit": c_fit}


def wavespeed_setup(*, nX=180, nY=60, nZ=180, dX=2.0e-4, rho=1000.0, cs_target=2.0, CFL=0.2,
                    Tmax=6.0e-3, amplitude=3e-5, sensor_offsets=None, eta=0.5, sigma_xy=None,
                    vel_damp=None) -> dict:
    """Inputs of the wavespeed check (validate_wavespeed.py:79-142): zero
    force, an initial velocity equal to the curl of psi = amplitude x a
    Hann-tapered Gaussian (v = (-dpsi/dz, 0, dpsi/dx)), sensors on the x
    axis through the grid centre."""
    mu = rho * cs_target**2
    dT = CFL * dX / (cs_target * math.sqrt(3.0))
    n_steps = int(math.ceil(Tmax / dT))
    big = max(nX, nZ) > 150
    if sigma_xy is None:
        sigma_xy = 5.0 if big else 3.0
    psi = amplitude * _tapered_gaussian(nX, nY, nZ, sigma_xy, sigma_xy)
    dpsi_dx, _, dpsi_dz = np.gradient(psi, dX, dX, dX, edge_order=2)
    vx0 = -dpsi_dz.astype(np.float32)
    v0 = np.stack([vx0, np.zeros_like(vx0), dpsi_dx.astype(np.float32)], axis=-1)
    if sensor_offsets is None:
        sensor_offsets = [18, 30, 42, 54, 66, 78] if big else [12, 18, 24, 30, 36, 42]
    offs = np.asarray(sensor_offsets, dtype=int)
    ix = nX // 2 + offs
    opts = {"vel_damp": vel_damp if vel_damp is not None else (0.001 if big else 0.002),
            "poisson_tol": 5e-5, "poisson_max_iters": 400, "initial_v": v0, "eta": eta,
            "env_t": np.zeros(n_steps, np.float32)}
    return {"bz": np.zeros((nX, nY, nZ), np.float32), "rho": rho, "mu": mu, "dX": dX, "dT": dT,
            "n_steps": n_steps, "opts": opts, "sensor_offsets": offs,
            "sensor_distances": offs * dX, "cs_target": cs_target,
            "trace_indices": (ix, np.full_like(ix, nY // 2), np.full_like(ix, nZ // 2))}


def wavespeed_recovery(*, precision="mixed", **setup) -> dict:
    """Shear-speed recovery from an impulse (validate_wavespeed.py:21-205);
    keyword arguments of :func:`wavespeed_setup` change the set-up."""
    s = wavespeed_setup(**setup)
    opts = dict(s["opts"], precision=precision)
    _, _, traces = shear_fdtd(None, None, s["bz"], s["rho"], s["mu"], s["dX"], s["dX"], s["dX"],
                              s["dT"], s["n_steps"], opts, trace_indices=s["trace_indices"],
                              return_traces=True)
    res = arrival_analysis(traces, s["dT"], s["sensor_distances"], s["cs_target"])
    res.update({k: s[k] for k in ("dT", "n_steps", "sensor_offsets", "sensor_distances",
                                  "cs_target")})
    res["traces"] = np.asarray(traces)
    return res


def quasistatic(*, nX=72, nY=48, nZ=72, dX=2.0e-4, rho=1000.0, cs=2.0, CFL=0.5, Tmax=7e-4,
                b_amp=0.02, vel_damp=0.05, precision="mixed") -> dict:
    """Damped time loop against the static solve (validate_quasistatic.py:21-108).

    The reference passes the projected force as a 4-D array repeated over
    every step (re-projected each step); here the same constant force goes
    in once as a 3-D field, which the solver projects once — the identical
    force at every step.
    """
    mu = rho * cs**2
    dT = CFL * dX / (cs * math.sqrt(3.0))
    n_steps = int(math.ceil(Tmax / dT))
    b0 = b_amp * _tapered_gaussian(nX, nY, nZ, 8.0, 6.0)
    bx, by, bz = project_body_force_to_shear(b0, dX, dX, dX, tol=5e-5, max_iters=400)
    opts = {"vel_damp": vel_damp, "poisson_tol": 5e-5, "poisson_max_iters": 400,
            "precision": precision}
    u, v = shear_fdtd(bx, by, bz, rho, mu, dX, dX, dX, dT, n_steps, opts)
    u_static = elastic_solve_static(bz, dX, dX, dX, mu, tol=1e-6, max_iters=1500)
    uz = np.asarray(u)[..., 2].astype(np.float64)
    us = np.asarray(u_static, dtype=np.float64)
    rel = float(np.linalg.norm(uz - us) / max(np.linalg.norm(us), np.finfo(np.float32).eps))
    return {"rel_err": rel, "max_abs_diff": float(np.max(np.abs(uz - us))),
            "v_norm": float(np.linalg.norm(np.asarray(v, dtype=np.float64))),
            "n_steps": n_steps, "dT": dT}
