"""CUDA path against fixtures produced by the reference itself (tests/golden).

Tolerances:
* plain FP64 form vs the FP64 reference run: relative L2 <= 1e-10 on u, v,
  snapshots and projected forces (the FP64 parity bar);
* mixed FP32 form vs the FP64 reference run: relative L2 <= 1e-4;
* operators and strain: bit-exact against the reference in float32 and float64.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 1e-4

FDTD = sorted(k for k, c in cases.CASES.items() if c["kind"] == "fdtd")
PROJ = sorted(k for k, c in cases.CASES.items() if c["kind"] == "projection")


def _run_fdtd(name, precision, dt):
    import shearwave_b200 as sw

    case = cases.CASES[name]
    inp = cases.fdtd_inputs(case, dt)
    opts = dict(inp["opts"], precision=precision)
    info = {}
    opts["info"] = info
    u, v, s = sw.shear_fdtd(inp["bx"], inp["by"], inp["bz"], inp["rho"], inp["mu"], case["dX"],
                            case["dY"], case["dZ"], case["dT"], case["n_steps"], opts,
                            snapshot_stride=case["stride"])
    return u, v, s, info


@pytest.mark.parametrize("name", FDTD)
def test_fdtd_fp64_matches_reference_fp64(cuda, name):
    gold = load_golden(name)
    u, v, s, info = _run_fdtd(name, "fp64", np.float64)
    assert u.dtype == np.float64 and v.dtype == np.float64
    assert u.shape == gold["f64_u"].shape
    assert not info["nonfinite"]
    assert rel_l2(u, gold["f64_u"]) <= FP64_TOL
    assert rel_l2(v, gold["f64_v"]) <= FP64_TOL
    assert rel_l2(s, gold["f64_snaps"]) <= FP64_TOL
    # shell stays exactly zero
    for a in (u, v):
        assert not a[0].any() and not a[-1].any() and not a[:, 0].any() and not a[:, :, -1].any()


@pytest.mark.parametrize("name", FDTD)
def test_fdtd_mixed_within_budget_of_reference_fp64(cuda, name):
    gold = load_golden(name)
    u, v, s, info = _run_fdtd(name, "mixed", np.float32)
    assert u.dtype == np.float32
    assert rel_l2(u, gold["f64_u"]) <= MIXED_TOL
    assert rel_l2(v, gold["f64_v"]) <= MIXED_TOL
    assert rel_l2(s, gold["f64_snaps"]) <= MIXED_TOL


@pytest.mark.parametrize("name", PROJ)
def test_projection_fp64_matches_reference(cuda, name):
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O

    case = cases.CASES[name]
    gold = load_golden(name)
    f = cases.projection_inputs(case, np.float64)
    d = case["h"]
    info = {}
    out = sw.project_vector_field(*f, d, d, d, case["tol"], case["max_iters"], info=info)
    assert info["reason"] == "converged"
    # same number of CG updates as the reference (applies = updates + 2)
    assert info["iters"] + 2 == int(gold["f64_apply_calls"])
    for k, o in zip(("fx", "fy", "fz"), out):
        assert o.dtype == np.float64
        assert rel_l2(o, gold[f"f64_{k}"]) <= FP64_TOL
    # divergence of the projected field agrees with the reference's, relative
    # to the input divergence
    m = O.shell_mask(out[0].shape, np.float64)
    div_in = O.divergence_center(*[a * m for a in f], d, d, d) * m
    div_gpu = O.divergence_center(*out, d, d, d) * m
    div_ref = O.divergence_center(gold["f64_fx"], gold["f64_fy"], gold["f64_fz"], d, d, d) * m
    assert np.linalg.norm(div_gpu - div_ref) / np.linalg.norm(div_in) <= FP64_TOL
    assert np.abs(div_gpu).max() <= 1e-6 * np.abs(div_in).max()


@pytest.mark.parametrize("name", PROJ)
def test_projection_fp32_inputs(cuda, name):
    import shearwave_b200 as sw

    case = cases.CASES[name]
    gold = load_golden(name)
    f = cases.projection_inputs(case, np.float32)
    d = case["h"]
    out = sw.project_vector_field(*f, d, d, d, case["tol"], case["max_iters"])
    for k, o in zip(("fx", "fy", "fz"), out):
        assert o.dtype == np.float32
        assert rel_l2(o, gold[f"f64_{k}"]) <= 1e-5
        assert rel_l2(o, gold[f"f32_{k}"]) <= 1e-5


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("f64", np.float64)])
def test_operators_bitexact(cuda, tag, dt):
    import shearwave_b200 as sw

    case = cases.CASES["ops_a"]
    gold = load_golden("ops_a")
    a, b, c = cases.operator_inputs(case, dt)
    h = case["h"]
    lap = sw.laplacian_center(a, *h)
    div = sw.divergence_center(a, b, c, *h)
    gx, gy, gz = sw.gradient_center(a, *h)
    for k, val in (("lap", lap), ("div", div), ("gx", gx), ("gy", gy), ("gz", gz)):
        ref = gold[f"{tag}_{k}"]
        assert val.dtype == ref.dtype
        assert np.array_equal(val, ref), k


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("f64", np.float64)])
def test_strain_bitexact(cuda, tag, dt):
    import shearwave_b200 as sw

    case = cases.CASES["strain_a"]
    gold = load_golden("strain_a")
    ux, uy, uz = cases.strain_inputs(case, dt)
    eps = sw.compute_strain_tensor(ux, uy, uz, *case["h"])
    assert eps.dtype == gold[f"{tag}_eps"].dtype
    assert np.array_equal(eps, gold[f"{tag}_eps"])
    inv = sw.compute_strain_invariants(eps)
    for k, val in inv.items():
        ref = gold[f"{tag}_inv_{k}"]
        assert val.dtype == ref.dtype, k
        assert np.array_equal(val, ref), k
    # fused post-pass on an AoS displacement gives the same numbers
    u = np.stack([ux, uy, uz], axis=-1)
    eps2, inv2 = sw.compute_strain_fields(u, *case["h"])
    assert np.array_equal(eps2, eps)
    for k in inv:
        assert np.array_equal(inv2[k], inv[k]), k


def test_static_solve_matches_reference(cuda):
    """elastic_solve_static (solver.py:569-625) against the reference's fixture."""
    import shearwave_b200 as sw

    case = cases.CASES["static_a"]
    gold = load_golden("static_a")
    bz = cases.static_inputs(case)
    d = case["h"]
    info = {}
    u64 = sw.elastic_solve_static(bz.astype(np.float64), d, d, d, case["mu"], tol=case["tol"],
                                  max_iters=case["max_iters"], info=info)
    assert u64.dtype == np.float64
    assert info["reason"] == "converged"
    assert info["iters"] + 1 == int(gold["f64_apply_calls"])  # + the initial residual
    assert rel_l2(u64, gold["f64_u"]) <= FP64_TOL
    u32 = sw.elastic_solve_static(bz, d, d, d, case["mu"], tol=case["tol"],
                                  max_iters=case["max_iters"])
    assert u32.dtype == np.float32
    assert rel_l2(u32, gold["f64_u"]) <= 1e-6
