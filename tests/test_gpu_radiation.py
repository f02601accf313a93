"""Radiation-force producers on the GPU against the reference's own outputs
(tests/golden/arf_*.npz, made by running src/shearwave/radiation_force.py).

The reference averages float32 records in float32 (numpy pairwise sums);
the kernels sum in FP64, so float32 results agree to a few float32 ulps
(relative L2 <= 1e-6) and float64 results to 1e-12.  The auto gate picks
the same time indices.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

ARF = sorted(k for k, c in cases.CASES.items() if c["kind"] == "radiation")
TOL = {"f32": 1e-6, "f64": 1e-12}


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("f64", np.float64)])
@pytest.mark.parametrize("name", ARF)
def test_radiation_force_matches_reference(cuda, name, tag, dt):
    from shearwave_b200 import compute_radiation_force, compute_radiation_force_velocity

    gold = load_golden(name)
    r = cases.radiation_inputs(cases.CASES[name], dt)
    b = compute_radiation_force(r["p"], r["c"], r["rho"], r["alpha"], r["f0"], gate=r["gate"])
    assert b.dtype == gold[f"{tag}_b"].dtype and b.shape == gold[f"{tag}_b"].shape
    assert rel_l2(b, gold[f"{tag}_b"]) <= TOL[tag]
    out = compute_radiation_force_velocity(r["p"], r["vx"], r["vy"], r["vz"], r["c"], r["rho"],
                                           r["alpha"], r["f0"], gate=r["gate"])
    for k, o in zip(("bx", "by", "bz"), out):
        assert o.dtype == gold[f"{tag}_{k}"].dtype
        assert rel_l2(o, gold[f"{tag}_{k}"]) <= TOL[tag], k


def test_auto_gate_matches_reference_rule(cuda):
    from shearwave_b200.radiation import auto_gate

    r = cases.radiation_inputs(cases.CASES["arf_auto"], np.float32)
    env = (r["p"].astype(np.float64) ** 2).mean(axis=(0, 1, 2))
    want = np.nonzero(env >= 0.1 * env.max())[0]
    assert np.array_equal(auto_gate(r["p"]), want)


def test_scalar_maps_and_device_inputs(cuda):
    """Scalar maps broadcast; torch CUDA records give torch results."""
    import torch

    from oracle import shearwave_oracle as O
    from shearwave_b200 import compute_radiation_force

    r = cases.radiation_inputs(cases.CASES["arf_slice"], np.float64)
    want = O.compute_radiation_force(r["p"], 1540.0, 1000.0, 0.5, r["f0"], r["gate"])
    got = compute_radiation_force(torch.from_numpy(r["p"]).cuda(), 1540.0, 1000.0, 0.5, r["f0"],
                                  gate=r["gate"])
    assert isinstance(got, torch.Tensor) and got.is_cuda
    assert rel_l2(got.cpu().numpy(), want) <= 1e-12


def test_gate_errors(cuda):
    from shearwave_b200 import compute_radiation_force

    r = cases.radiation_inputs(cases.CASES["arf_slice"], np.float32)
    with pytest.raises(IndexError):
        compute_radiation_force(r["p"], r["c"], r["rho"], r["alpha"], 1e6, gate=[0, 999])
    with pytest.raises(ValueError):
        compute_radiation_force(r["p"], r["c"], r["rho"], r["alpha"], 1e6, gate=slice(5, 5))
    with pytest.raises(ValueError):
        compute_radiation_force(r["p"][..., 0], r["c"], r["rho"], r["alpha"], 1e6)
