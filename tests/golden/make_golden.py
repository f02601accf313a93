"""Generate the golden fixtures under tests/golden/ by running the reference itself.

Point ``SHEARWAVE_REF_SRC`` at the ``src`` directory of a pinton-lab/shearwave
checkout (the directory that holds the ``shearwave`` package) and run:

    SHEARWAVE_REF_SRC=<checkout>/src python tests/golden/make_golden.py [case ...]

Each case is run twice through the reference's own NumPy code:

* ``f32`` - the reference exactly as shipped (float32 fields, float64 CG);
* ``f64`` - the same code with its module-level ``np`` replaced by a proxy
  whose ``float32`` attribute is ``numpy.float64``, so every float32 cast in
  ``solver.py`` widens to float64 (the FP64 oracle of the hot path).

Inputs are regenerated from the seeds and parameters stored in each ``.npz``
by ``tests/golden/cases.py``; outputs are stored as produced.  The fixtures
pin ``oracle/shearwave_oracle.py`` (CPU tests) and the CUDA path (GPU tests).
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import cases  # noqa: E402

REF_SRC = os.environ.get("SHEARWAVE_REF_SRC")
if not REF_SRC or not (Path(REF_SRC) / "shearwave" / "solver.py").is_file():
    sys.exit("make_golden.py: set SHEARWAVE_REF_SRC to the src directory of a "
             "pinton-lab/shearwave checkout (it must contain shearwave/solver.py)")
sys.path.insert(0, REF_SRC)
import shearwave.radiation_force as ref_arf  # noqa: E402
import shearwave.solver as ref_solver  # noqa: E402
import shearwave.strain as ref_strain  # noqa: E402


class _Widened(types.ModuleType):
    """numpy with float32 widened to float64 (the FP64 oracle technique)."""

    def __getattr__(self, name):
        return getattr(np, name)


_WIDE = _Widened("numpy_widened")
_WIDE.float32 = np.float64


class _precision:
    """Context manager that swaps the reference solver's numpy module."""

    def __init__(self, wide: bool):
        self.wide = wide

    def __enter__(self):
        if self.wide:
            ref_solver.np = _WIDE

    def __exit__(self, *exc):
        ref_solver.np = np


class _CGCounter:
    """Counts the reference CG's operator applications through one operator."""

    def __init__(self, op: str = "gradient_center"):
        self.calls = 0
        self.op = op
        self._orig = getattr(ref_solver, op)

    def __enter__(self):
        def wrapped(*a, **k):
            self.calls += 1
            return self._orig(*a, **k)

        setattr(ref_solver, self.op, wrapped)
        return self

    def __exit__(self, *exc):
        setattr(ref_solver, self.op, self._orig)


def _run_fdtd(case: dict, wide: bool):
    inp = cases.fdtd_inputs(case, np.float64 if wide else np.float32)
    stride = case.get("stride")
    snaps = []

    def cb(it, u):
        if stride and (it + 1) % stride == 0:
            snaps.append(np.array(u, copy=True))

    with _precision(wide):
        u, v = ref_solver.shear_fdtd(
            inp["bx"], inp["by"], inp["bz"], inp["rho"], inp["mu"],
            case["dX"], case["dY"], case["dZ"], case["dT"], case["n_steps"],
            opts=inp["opts"], callback=cb,
        )
    out = {"u": u, "v": v}
    if stride:
        out["snaps"] = np.stack(snaps)
    return out


def _run_projection(case: dict, wide: bool):
    dt = np.float64 if wide else np.float32
    fx, fy, fz = cases.projection_inputs(case, dt)
    d = case["h"]
    with _precision(wide), _CGCounter() as cnt:
        ox, oy, oz = ref_solver.project_vector_field(
            fx.copy(), fy.copy(), fz.copy(), d, d, d, case["tol"], case["max_iters"],
        )
    # one apply_a for the initial residual, one gradient for f - grad(phi)
    return {"fx": ox, "fy": oy, "fz": oz, "apply_calls": np.int64(cnt.calls)}


def _run_operators(case: dict, wide: bool):
    dt = np.float64 if wide else np.float32
    a, b, c = cases.operator_inputs(case, dt)
    h = case["h"]
    with _precision(wide):
        lap = ref_solver.laplacian_center(a, *h)
        div = ref_solver.divergence_center(a, b, c, *h)
        gx, gy, gz = ref_solver.gradient_center(a, *h)
    return {"lap": lap, "div": div, "gx": gx, "gy": gy, "gz": gz}


def _run_strain(case: dict, wide: bool):
    dt = np.float64 if wide else np.float32
    ux, uy, uz = cases.strain_inputs(case, dt)
    h = case["h"]
    eps = ref_strain.compute_strain_tensor(ux, uy, uz, *h)
    inv = ref_strain.compute_strain_invariants(eps)
    return {"eps": eps, **{f"inv_{k}": v for k, v in inv.items()}}


def _run_static(case: dict, wide: bool):
    bz = cases.static_inputs(case)
    d = case["h"]
    with _precision(wide), _CGCounter("laplacian_center") as cnt:
        u = ref_solver.elastic_solve_static(
            bz.astype(np.float64 if wide else np.float32), d, d, d, case["mu"],
            tol=case["tol"], max_iters=case["max_iters"],
        )
    return {"u": u, "apply_calls": np.int64(cnt.calls)}


def _run_radiation(case: dict, wide: bool):
    """radiation_force.py has no float32 casts: f32 runs float32 records and
    maps, f64 the same values in float64."""
    r = cases.radiation_inputs(case, np.float64 if wide else np.float32)
    b = ref_arf.compute_radiation_force(r["p"], r["c"], r["rho"], r["alpha"], r["f0"],
                                        gate=r["gate"])
    bx, by, bz = ref_arf.compute_radiation_force_velocity(
        r["p"], r["vx"], r["vy"], r["vz"], r["c"], r["rho"], r["alpha"], r["f0"], gate=r["gate"])
    return {"b": b, "bx": bx, "by": by, "bz": bz}


def _run_wavespeed(case: dict, wide: bool):
    """validation/validate_wavespeed.py:21-205 at its defaults, through the
    reference's shear_fdtd with a per-step callback recording u_z at the
    sensors; the arrival analysis is shearwave_b200.validation's restatement
    of the script's (the script itself needs matplotlib)."""
    sys.path.insert(0, str(HERE.parents[1]))
    from shearwave_b200 import validation as V

    s = V.wavespeed_setup()
    traces = np.zeros((len(s["sensor_offsets"]), s["n_steps"]), np.float32)
    ix, iy, iz = s["trace_indices"]

    def cb(it, u):
        traces[:, it] = u[ix, iy, iz, 2]

    ref_solver.shear_fdtd(None, None, s["bz"], s["rho"], s["mu"], s["dX"], s["dX"], s["dX"],
                          s["dT"], s["n_steps"], opts=s["opts"], callback=cb)
    r = V.arrival_analysis(traces, s["dT"], s["sensor_distances"], s["cs_target"])
    return {"traces": traces, "arrival_idx": r["arrival_idx"], "c_fit": np.float64(r["c_fit"])}


RUNNERS = {
    "fdtd": _run_fdtd,
    "projection": _run_projection,
    "operators": _run_operators,
    "strain": _run_strain,
    "static": _run_static,
    "radiation": _run_radiation,
    "wavespeed": _run_wavespeed,
}


def main(names=None) -> None:
    """Regenerate every fixture, or only the named cases."""
    for name, case in cases.CASES.items():
        if names and name not in names:
            continue
        payload = {"case": np.array(repr(case))}
        for tag, wide in (("f32", False),) + ((("f64", True),) if not case.get("f32_only")
                                               else ()):
            out = RUNNERS[case["kind"]](case, wide)
            for k, v in out.items():
                payload[f"{tag}_{k}"] = np.asarray(v)
        path = HERE / f"{name}.npz"
        np.savez_compressed(path, **payload)
        print(f"{path.name}: {path.stat().st_size / 1024:.1f} KiB")


if __name__ == "__main__":
    main(sys.argv[1:])
