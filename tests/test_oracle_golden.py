"""Pin the CPU oracle against fixtures produced by running the reference itself.

tests/golden/make_golden.py ran pinton-lab/shearwave's own NumPy code (float32
as shipped, and float64 through the widened-numpy proxy) on the cases of
tests/golden/cases.py.  The oracle must reproduce every output bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from conftest import load_golden
from oracle import shearwave_oracle as O

PREC = [("f32", np.float32), ("f64", np.float64)]


def _oracle_outputs(case: dict, dt):
    kind = case["kind"]
    if kind == "fdtd":
        inp = cases.fdtd_inputs(case, dt)
        u, v, s = O.shear_fdtd(inp["bx"], inp["by"], inp["bz"], inp["rho"], inp["mu"],
                               case["dX"], case["dY"], case["dZ"], case["dT"], case["n_steps"],
                               opts=inp["opts"], dtype=dt, snapshot_stride=case["stride"])
        return {"u": u, "v": v, "snaps": s}
    if kind == "projection":
        f = cases.projection_inputs(case, dt)
        d = case["h"]
        st = O.CGStats()
        o = O.project_vector_field(*[a.copy() for a in f], d, d, d, case["tol"],
                                   case["max_iters"], dtype=dt, stats=st)
        return {"fx": o[0], "fy": o[1], "fz": o[2], "apply_calls": np.int64(st.iters + 2)}
    if kind == "operators":
        a, b, c = cases.operator_inputs(case, dt)
        h = case["h"]
        gx, gy, gz = O.gradient_center(a, *h)
        return {"lap": O.laplacian_center(a, *h), "div": O.divergence_center(a, b, c, *h),
                "gx": gx, "gy": gy, "gz": gz}
    if kind == "strain":
        ux, uy, uz = cases.strain_inputs(case, dt)
        e = O.compute_strain_tensor(ux, uy, uz, *case["h"])
        inv = O.compute_strain_invariants(e)
        return {"eps": e, **{f"inv_{k}": v for k, v in inv.items()}}
    if kind == "static":
        bz = cases.static_inputs(case)
        d = case["h"]
        return {"u": O.elastic_solve_static(bz.astype(dt), d, d, d, case["mu"], tol=case["tol"],
                                            max_iters=case["max_iters"], dtype=dt)}
    if kind == "radiation":
        r = cases.radiation_inputs(case, dt)
        b = O.compute_radiation_force(r["p"], r["c"], r["rho"], r["alpha"], r["f0"], r["gate"])
        bx, by, bz = O.compute_radiation_force_velocity(r["p"], r["vx"], r["vy"], r["vz"], r["c"],
                                                        r["rho"], r["alpha"], r["f0"], r["gate"])
        return {"b": b, "bx": bx, "by": by, "bz": bz}
    raise KeyError(kind)


@pytest.mark.parametrize("tag,dt", PREC)
@pytest.mark.parametrize("name", sorted(k for k, c in cases.CASES.items()
                                        if c["kind"] != "wavespeed"))
def test_oracle_matches_reference_bitwise(name, tag, dt):
    case = cases.CASES[name]
    gold = load_golden(name)
    out = _oracle_outputs(case, dt)
    for key, val in out.items():
        ref = gold[f"{tag}_{key}"]
        val = np.asarray(val)
        if key == "apply_calls":
            assert int(val) == int(ref), (name, tag, key)
            continue
        assert val.dtype == ref.dtype, (name, tag, key, val.dtype, ref.dtype)
        assert val.shape == ref.shape, (name, tag, key)
        assert np.array_equal(val, ref), (name, tag, key)


def test_golden_cases_are_all_present():
    for name, case in cases.CASES.items():
        gold = load_golden(name)
        assert any(k.startswith("f32_") for k in gold)
        assert case.get("f32_only") or any(k.startswith("f64_") for k in gold)


def test_oracle_cg_stopping_rule_counts():
    """The oracle CG reports the same number of operator applications as the reference."""
    gold = load_golden("proj_blob")
    case = cases.CASES["proj_blob"]
    f = cases.projection_inputs(case, np.float64)
    st = O.CGStats()
    d = case["h"]
    O.project_vector_field(*f, d, d, d, case["tol"], case["max_iters"], dtype=np.float64, stats=st)
    assert st.reason == "converged"
    assert st.iters + 2 == int(gold["f64_apply_calls"])
