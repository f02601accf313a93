"""sw_project_noalloc: the projection for callers that cannot allocate device memory.

Hosts that only lend the library their own input and output buffers — an
application whose device memory is reserved up front by its own pool, or a
binding that has no way to allocate a device workspace — call
sw_project_noalloc instead of sw_project.  It runs the same CG with its
scratch in an array compiled into the library.  This test calls both entry
points through the C ABI on the same inputs, twice in a row with different
fields (the shared scratch keeps the previous call's contents, so the second
call checks that nothing stale leaks through), and requires the results to
agree within the FP64 parity tolerance of the other tests (1e-10) with the
same CG iteration count.  It also checks that a grid too large for the
scratch is refused with a clear error instead of running.

Collected last (file name) so a run that stops at the first failure has run
every other test first; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    t = [np.sin(np.pi * np.linspace(0, 1, n)) for n in shape]
    taper = t[0][:, None, None] * t[1][None, :, None] * t[2][None, None, :]
    return [rng.standard_normal(shape) * taper for _ in range(3)]


def test_noalloc_matches_workspace_entry_point_twice(cuda):
    import torch

    import shearwave_b200._native as native

    lib = native.load()
    native.call("sw_set_device", 0)
    stream = torch.cuda.current_stream().cuda_stream
    shape = (40, 36, 50)
    nx, ny, nz = shape
    h = (0.5e-3, 0.45e-3, 0.55e-3)
    pz = lib.sw_pitch(nz)
    for seed in (11, 12):  # two calls in a row through the shared scratch
        f = [torch.from_numpy(a).to("cuda") for a in _fields(shape, seed)]
        args = (native.SW_F64, *(a.data_ptr() for a in f), ny * nz, nz, 1, nx, ny, nz, *h,
                1e-10, 2000)
        ws_bytes = int(lib.sw_project_workspace_bytes(nx, ny, nz))
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
        ref = torch.empty((3, nx * ny * pz), dtype=torch.float64, device="cuda")
        st_ref = native.CGStats()
        native.call("sw_project", *args, ref.data_ptr(), ws.data_ptr(), ws_bytes,
                    C.byref(st_ref), stream)
        got = torch.full((3, nx * ny * pz), float("nan"), dtype=torch.float64, device="cuda")
        st = native.CGStats()
        native.call("sw_project_noalloc", *args, got.data_ptr(), C.byref(st), stream)
        torch.cuda.synchronize()
        assert st.reason == st_ref.reason == native.SW_CG_CONVERGED
        assert st.iters == st_ref.iters > 0
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) <= TOL


def test_noalloc_refuses_grids_beyond_its_scratch(cuda):
    import torch

    import shearwave_b200._native as native

    lib = native.load()
    native.call("sw_set_device", 0)
    nx = ny = nz = 128  # needs ~80 MB of scratch, above the 32 MiB held
    assert lib.sw_project_workspace_bytes(nx, ny, nz) > lib.sw_project_noalloc_scratch_bytes()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    rc = lib.sw_project_noalloc(native.SW_F64, None, None, None, ny * nz, nz, 1, nx, ny, nz,
                                1e-3, 1e-3, 1e-3, 1e-10, 100, out.data_ptr(), None,
                                torch.cuda.current_stream().cuda_stream)
    assert rc == native.SW_ERANGE
    assert b"scratch" in lib.sw_last_error()
