"""The custom ops on the GPU: torch.library.opcheck of their schemas (which
arguments they write) and of their fake implementations against the real
outputs, including the time-loop ops on a small solve's device state."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHECKS = ("test_schema", "test_faketensor")


def test_opcheck_operators(cuda):
    import torch

    ops = torch.ops.shearwave_b200
    h = [1e-3, 1.1e-3, 0.9e-3]
    for dt in (torch.float32, torch.float64):
        f = torch.randn(12, 10, 14, device=cuda, dtype=dt)
        g = torch.randn(12, 10, 14, device=cuda, dtype=dt)
        torch.library.opcheck(ops.laplacian, (f, h), test_utils=CHECKS)
        torch.library.opcheck(ops.divergence, (f, g, f, h), test_utils=CHECKS)
        torch.library.opcheck(ops.gradient, (f, h), test_utils=CHECKS)
        torch.library.opcheck(ops.strain, (f, g, f, h, True, True), test_utils=CHECKS)
        torch.library.opcheck(ops.strain, (f, g, f, h, True, False), test_utils=CHECKS)
        u = torch.randn(12, 10, 14, 3, device=cuda, dtype=dt)
        torch.library.opcheck(ops.strain_aos, (u, h, False), test_utils=CHECKS)
        e = torch.randn(7, 5, 6, device=cuda, dtype=dt)
        torch.library.opcheck(ops.strain_invariants, (e,), test_utils=CHECKS)


def test_opcheck_projection(cuda):
    import torch

    ops = torch.ops.shearwave_b200
    f = torch.randn(12, 10, 14, device=cuda, dtype=torch.float64)
    h = [1e-3, 1e-3, 1e-3]
    torch.library.opcheck(ops.project, (None, None, f, h, 1e-8, 400, "cg"), test_utils=CHECKS)
    torch.library.opcheck(ops.project, (f, None, f, h, 1e-8, 400, "spectral"),
                          test_utils=CHECKS)


def test_opcheck_time_loop(cuda):
    """fdtd_steps_ and fdtd_finish on the state of a small solve (both forms)."""
    import torch

    from shearwave_b200 import solver as S
    from shearwave_b200 import workloads as W

    for precision in ("mixed", "fp64"):
        p = W.problem_inclusions((14, 12, 18), 8, seed=5, tol=1e-9)
        sv = S._Solve(**{k: p[k] for k in ("bx", "by", "bz", "rho", "mu", "dX", "dY", "dZ",
                                           "dT", "n_steps")},
                      opts=dict(p["opts"], precision=precision))
        for k, comps in sv.separable_inputs():
            fs, _st = S._project_raw(comps, sv.spacing, sv.tol, sv.max_iters, sv.method)
            sv.store_pattern(k, fs)
        sv.build_terms()
        b = sv.run.bundle()
        torch.library.opcheck(torch.ops.shearwave_b200.fdtd_steps_, (*b, 0, 4),
                              test_utils=("test_schema",))
        torch.library.opcheck(torch.ops.shearwave_b200.fdtd_finish, (*b, 4, True),
                              test_utils=CHECKS)


def test_shear_fdtd_runs_through_the_ops(cuda, monkeypatch):
    """The drop-in's time loop reaches the library through torch.ops."""
    import shearwave_b200 as sw
    from shearwave_b200 import ops
    from shearwave_b200 import workloads as W

    seen = []
    real = ops.fdtd_steps_

    def spy(*a):
        seen.append((a[-2], a[-1]))
        return real(*a)

    monkeypatch.setattr(ops, "fdtd_steps_", spy)
    p = W.problem_inclusions((16, 14, 20), 12, seed=9, tol=1e-9)
    u, v = sw.shear_fdtd(p["bx"], p["by"], p["bz"], p["rho"], p["mu"], p["dX"], p["dY"],
                         p["dZ"], p["dT"], p["n_steps"], p["opts"])
    assert seen == [(0, 12)]
    assert np.all(np.isfinite(u)) and np.any(u != 0)
