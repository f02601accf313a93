"""The C-ABI library loads on a CPU-only host and exports every declared symbol.

No compute entry point is called here (there is no GPU); only the pure helpers
``sw_abi_version``, ``sw_pitch`` and ``sw_project_workspace_bytes``.
"""

from __future__ import annotations

import ctypes
import re

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
