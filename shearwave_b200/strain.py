"""Strain post-pass on the B200 CUDA library (drop-in for src/shearwave/strain.py).

``compute_strain_tensor`` and ``compute_strain_invariants`` keep the
reference's signatures, Voigt ordering ``[exx, eyy, ezz, gyz, gxz, gxy]``
(engineering shear), dtypes and error messages (strain.py:16-159).
``compute_strain_fields`` is the fused post-pass: one kernel reads the three
displacement components once and writes the Voigt tensor and all four
invariants.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native
from ._device import dtype_code, is_tensor, ptr, require_cuda, stream_handle, to_device

__all__ = ["compute_strain_fields", "compute_strain_invariants", "compute_strain_tensor"]


def _validate(ux, uy, uz, dX, dY, dZ):
    """Input checks of strain.py:138-159 (same messages)."""
    if ux.ndim != 3:
        raise ValueError(f"Displacement arrays must be 3-D, got ndim={ux.ndim}")
    if tuple(ux.shape) != tuple(uy.shape) or tuple(ux.shape) != tuple(uz.shape):
        raise ValueError(
            "All displacement components must share the same shape: "
            f"ux={tuple(ux.shape)}, uy={tuple(uy.shape)}, uz={tuple(uz.shape)}"
        )
    for name, val in (("dX", dX), ("dY", dY), ("dZ", dZ)):
        if val <= 0:
            raise ValueError(f"Grid spacing {name} must be positive, got {val}")


def _dtype(*arrs) -> torch.dtype:
    dts = [a.dtype if is_tensor(a) else np.asarray(a).dtype for a in arrs]
    return torch.float32 if all(d in (np.float32, torch.float32) for d in dts) else torch.float64


def compute_strain_tensor(ux, uy, uz, dX, dY, dZ):
    """Voigt strain tensor (nx, ny, nz, 6) in the input dtype (strain.py:16-70)."""
    _validate(ux, uy, uz, dX, dY, dZ)
    dev = require_cuda()
    dt = _dtype(ux, uy, uz)
    a, b, c = (to_device(v, dt, dev) for v in (ux, uy, uz))
    nx, ny, nz = a.shape
    eps = torch.empty((nx, ny, nz, 6), dtype=dt, device=dev)
    _native.call("sw_strain", dtype_code(dt), ptr(a), ptr(b), ptr(c), ny * nz, nz, 1, nx, ny, nz,
                 dX, dY, dZ, ptr(eps), None, None, None, None, stream_handle())
    return eps if is_tensor(ux) else eps.cpu().numpy()


def compute_strain_invariants(epsilon):
    """Volumetric, deviatoric, max-shear and von Mises strain (strain.py:73-135).

    Returns a dict of arrays of shape ``epsilon.shape[:-1]``; ``von_mises`` is
    float64 like the reference's (numpy promotes it through the float64
    ``sqrt(2/3)`` factor).
    """
    if epsilon.shape[-1] != 6:
        raise ValueError(
            f"Expected last dimension == 6 (Voigt notation), got {epsilon.shape[-1]}"
        )
    dev = require_cuda()
    dt = _dtype(epsilon)
    e = to_device(epsilon, dt, dev)
    lead = tuple(e.shape[:-1])
    n = int(np.prod(lead)) if lead else 1
    outs = {k: torch.empty(lead, dtype=dt, device=dev)
            for k in ("volumetric", "deviatoric", "max_shear")}
    outs["von_mises"] = torch.empty(lead, dtype=torch.float64, device=dev)
    _native.call("sw_strain_invariants", dtype_code(dt), ptr(e), n, ptr(outs["volumetric"]),
                 ptr(outs["deviatoric"]), ptr(outs["max_shear"]), ptr(outs["von_mises"]),
                 stream_handle())
    order = ("volumetric", "deviatoric", "max_shear", "von_mises")
    if is_tensor(epsilon):
        return {k: outs[k] for k in order}
    return {k: outs[k].cpu().numpy() for k in order}


def compute_strain_fields(u, dX, dY, dZ, *, return_tensor=True, return_device=False):
    """Fused strain post-pass of a solver displacement ``u`` (nx, ny, nz, 3).

    One kernel reads the three components once and writes the Voigt tensor
    (if ``return_tensor``) and the four invariants.  Returns
    ``(epsilon or None, invariants dict)``; identical values to
    ``compute_strain_tensor`` followed by ``compute_strain_invariants``.
    """
    if u.ndim != 4 or u.shape[-1] != 3:
        raise ValueError("u must have shape (nx, ny, nz, 3)")
    for name, val in (("dX", dX), ("dY", dY), ("dZ", dZ)):
        if val <= 0:
            raise ValueError(f"Grid spacing {name} must be positive, got {val}")
    dev = require_cuda()
    dt = _dtype(u)
    t = to_device(u, dt, dev)
    nx, ny, nz, _ = t.shape
    eps = torch.empty((nx, ny, nz, 6), dtype=dt, device=dev) if return_tensor else None
    inv = {k: torch.empty((nx, ny, nz), dtype=dt, device=dev)
           for k in ("volumetric", "deviatoric", "max_shear")}
    inv["von_mises"] = torch.empty((nx, ny, nz), dtype=torch.float64, device=dev)
    base = t.data_ptr()
    es = t.element_size()
    # AoS input: component c starts at element c, strides (ny*nz*3, nz*3, 3)
    _native.call("sw_strain", dtype_code(dt), base, base + es, base + 2 * es, ny * nz * 3, nz * 3,
                 3, nx, ny, nz, dX, dY, dZ, ptr(eps), ptr(inv["volumetric"]),
                 ptr(inv["deviatoric"]), ptr(inv["max_shear"]), ptr(inv["von_mises"]),
                 stream_handle())
    dev_out = return_device or is_tensor(u)
    conv = (lambda x: x) if dev_out else (lambda x: None if x is None else x.cpu().numpy())
    return conv(eps), {k: conv(v) for k, v in inv.items()}
