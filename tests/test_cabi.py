"""The C-ABI library loads on a CPU-only host and exports every declared symbol.

No compute entry point is called here (there is no GPU); only the pure helpers
``sw_abi_version``, ``sw_pitch`` and ``sw_project_workspace_bytes``.
"""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT

import shearwave_b200._native as native

HEADER = ROOT / "include" / "shearwave_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sw_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = native.load()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), f"{name} declared in {HEADER.name} but not exported"


def test_binding_covers_the_header():
    assert set(native.exported_symbols()) <= set(declared_functions())
    assert set(declared_functions()) <= set(native.exported_symbols())


def test_pure_helpers():
    lib = native.load()
    assert lib.sw_abi_version() == 1
    assert lib.sw_pitch(64) == 64
    assert lib.sw_pitch(65) == 72
    assert lib.sw_pitch(1) == 8
    b = lib.sw_project_workspace_bytes(64, 64, 64)
    assert b >= 5 * 64**3 * 8
    assert lib.sw_project_workspace_bytes(0, 4, 4) == 0


def test_library_is_in_tree_and_built_for_sm100a():
    path = native.LIB_PATH
    assert path.is_file()
    assert path.parent.parent.name == "shearwave_b200"
    # the descriptor layout used by ctypes matches the C header's field order
    assert ctypes.sizeof(native.FdtdDesc) > 0


def test_spectral_basis_diagonalises_the_projection_operator():
    """Host-side basis of the direct Poisson solve: Q^T A_1 Q = diag(lam), Q orthonormal.

    A_1 is the reference's 1-D operator -div_c(grad_c .) with both
    differences zero on the shell (src/shearwave/solver.py:708-729,
    1024-1026), built here column by column.
    """
    import numpy as np

    lib = native.load()

    def a1(n, h):
        m = n - 2
        A = np.zeros((m, m))
        for col in range(m):
            x = np.zeros(n)
            x[col + 1] = 1.0
            g = np.zeros(n)
            g[1:-1] = (x[2:] - x[:-2]) / (2 * h)
            d = np.zeros(n)
            d[1:-1] = (g[2:] - g[:-2]) / (2 * h)
            A[:, col] = -d[1:-1]
        return A

    for n in (4, 5, 6, 7, 10, 11, 64, 65, 130):
        m = n - 2
        Q = np.zeros(m * m)
        lam = np.zeros(m)
        assert lib.sw_spectral_basis(n, 0.5e-3, Q.ctypes.data, lam.ctypes.data) == 0
        Q = Q.reshape(m, m)
        A = a1(n, 0.5e-3)
        assert np.abs(Q.T @ Q - np.eye(m)).max() < 1e-13
        assert np.abs(Q.T @ A @ Q - np.diag(lam)).max() / np.abs(A).max() < 1e-13


def test_tune_knobs_roundtrip():
    """Launch-shape knobs: defaults, set / get, range checks (host only)."""
    from shearwave_b200 import tune

    old = tune.get_knobs()
    assert set(old) == {"ctas_per_sm", "batch_tiles_per_cta", "xchunk", "tile_shape",
                        "steps_per_pass"}
    assert old["steps_per_pass"] == 0  # automatic unless a caller sets it
    try:
        with tune.knobs(ctas_per_sm=1, xchunk=32, steps_per_pass=2):
            assert tune.get_knobs()["ctas_per_sm"] == 1
            assert tune.get_knobs()["xchunk"] == 32
            assert tune.get_knobs()["steps_per_pass"] == 2
        assert tune.get_knobs() == old
        for bad in ({"ctas_per_sm": 3}, {"ctas_per_sm": 0}, {"batch_tiles_per_cta": 0},
                    {"xchunk": -1}, {"tile_shape": 3}, {"steps_per_pass": 3},
                    {"steps_per_pass": -1}, {"nope": 1}):
            with pytest.raises(ValueError):
                tune.set_knobs(**bad)
        assert tune.get_knobs() == old
    finally:
        tune.set_knobs(**old)


def test_tune_workload_key_and_shorten():
    import numpy as np

    from shearwave_b200 import tune

    bz = np.zeros((30, 40, 50), np.float32)
    p = {"bx": None, "by": None, "bz": bz, "rho": 1.0, "mu": 1.0, "dX": 1, "dY": 1, "dZ": 1,
         "dT": 1, "n_steps": 100, "opts": {"env_t": np.ones(100), "force_terms": [
             ((None, None, bz), np.ones(100))]}, "snapshot_stride": 10}
    assert tune.workload_key(p) == "mixed:single:32x48x48"
    assert tune.workload_key([p, p], "fp64") == "fp64:batch2:2^17"
    q = tune._shorten(p, 16)
    assert q["n_steps"] == 16 and len(q["opts"]["env_t"]) == 16
    assert len(q["opts"]["force_terms"][0][1]) == 16 and "snapshot_stride" not in q
    assert p["n_steps"] == 100 and len(p["opts"]["env_t"]) == 100
