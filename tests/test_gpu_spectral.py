"""The direct spectral Poisson solve against the reference's CG (FP64 oracle).

Both invert A = -div_c(grad_c .).  The spectral solve is exact; a CG run to a
tight tolerance must agree with it to that tolerance's truncation level, and
the projected field's divergence must vanish to FP64 round-off.
"""

from __future__ import annotations

import numpy as np
import pytest

import cases
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["proj_taper_s0", "proj_taper_s1", "proj_blob"])
def test_spectral_matches_tight_cg(cuda, name):
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O

    case = cases.CASES[name]
    f = cases.projection_inputs(case, np.float64)
    d = case["h"]
    ref = O.project_vector_field(*[a.copy() for a in f], d, d, d, 1e-13, 20000,
                                 dtype=np.float64)
    out = sw.project_vector_field(*f, d, d, d, 0.0, 0, method="spectral")
    for a, b in zip(out, ref):
        assert rel_l2(a, b) <= 1e-9
    m = O.shell_mask(out[0].shape, np.float64)
    div_in = O.divergence_center(*[a * m for a in f], d, d, d) * m
    div_out = O.divergence_center(*out, d, d, d) * m
    assert np.abs(div_out).max() <= 1e-11 * np.abs(div_in).max()


@pytest.mark.parametrize("shape", [(5, 7, 9), (17, 13, 11), (40, 9, 133), (3, 20, 6)])
def test_spectral_odd_grids(cuda, shape):
    import shearwave_b200 as sw
    from oracle import shearwave_oracle as O

    rng = np.random.default_rng(sum(shape))
    h = (0.5e-3, 0.7e-3, 0.4e-3)
    f = [rng.standard_normal(shape) for _ in range(3)]
    ref = O.project_vector_field(*[a.copy() for a in f], *h, 1e-13, 50000, dtype=np.float64)
    out = sw.project_vector_field(*f, *h, 0.0, 0, method="spectral")
    for a, b in zip(out, ref):
        assert rel_l2(a, b) <= 1e-8


def test_mixed_auto_uses_spectral_within_budget(cuda):
    """Mixed form with poisson_tol 1e-10 (spectral) vs the FP64 oracle (CG)."""
    import shearwave_b200 as sw
    from conftest import load_golden

    case = cases.CASES["fdtd_hetero"]
    gold = load_golden("fdtd_hetero")
    inp = cases.fdtd_inputs(case, np.float32)
    info = {}
    u, v = sw.shear_fdtd(inp["bx"], inp["by"], inp["bz"], inp["rho"], inp["mu"], case["dX"],
                         case["dY"], case["dZ"], case["dT"], case["n_steps"],
                         dict(inp["opts"], info=info))
    assert info["cg"][0]["method"] == "spectral"
    # the mixed-form budget; observed ~1e-6 (FP32 rounding of the fields)
    assert rel_l2(u, gold["f64_u"]) <= 1e-4
    assert rel_l2(v, gold["f64_v"]) <= 1e-4
