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

from . import ops
from ._device import is_tensor, require_cuda, to_device

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
    eps = ops.strain(a, b, c, [dX, dY, dZ], True, False)[0]
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
    e = to_device(epsilon, dt, dev).contiguous()
    order = ("volumetric", "deviatoric", "max_shear", "von_mises")
    outs = dict(zip(order, ops.strain_invariants(e)))
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
    t = to_device(u, dt, dev).contiguous()
    # one kernel reads the AoS components in place (strides 3 nz ny, 3 nz, 3)
    eps, *rest = ops.strain_aos(t, [dX, dY, dZ], bool(return_tensor))
    eps = eps if return_tensor else None
    inv = dict(zip(("volumetric", "deviatoric", "max_shear", "von_mises"), rest))
    dev_out = return_device or is_tensor(u)
    conv = (lambda x: x) if dev_out else (lambda x: None if x is None else x.cpu().numpy())
    return conv(eps), {k: conv(v) for k, v in inv.items()}
