"""Acoustic radiation force producers on the GPU (the step before shear_fdtd).

Drop-in replacements for ``compute_radiation_force`` and
``compute_radiation_force_velocity`` (src/shearwave/radiation_force.py:27-157):
same arguments, same auto-gate rule, same formula, the result in the
inputs' promoted dtype (float32 for float32 records and maps).  The records
are read straight from their (nx, ny, nz, nt) layout by the kernels of
``csrc/sw_arf.cu``; means are accumulated in FP64 (the reference accumulates
float32 records in float32, so float32 results agree to a few ulps, not
bit for bit).
"""

from __future__ import annotations

import numpy as np
import torch

from . import ops
from ._device import is_tensor, require_cuda, to_device

__all__ = ["compute_radiation_force", "compute_radiation_force_velocity", "auto_gate"]


def _dtype_of(a):
    if is_tensor(a):
        return a.dtype
    if isinstance(a, np.ndarray):
        return torch.float64 if a.dtype == np.float64 else torch.float32
    return None  # Python scalars take the arrays' dtype


def _result_dtype(*arrays):
    dts = [d for d in (_dtype_of(a) for a in arrays) if d is not None]
    return torch.float64 if torch.float64 in dts else torch.float32


def _record(a, dt, dev):
    t = to_device(a, dt, dev)
    if t.ndim != 4:
        raise ValueError("pressure and velocity records must have shape (nx, ny, nz, nt)")
    return t.contiguous()


def _map(v, shape, dev):
    """A material map as FP64 on the device, and its stride (0 for a scalar)."""
    if np.ndim(v) == 0 and not (is_tensor(v) and v.ndim > 0):
        return torch.full((1,), float(v), dtype=torch.float64, device=dev), 0
    t = to_device(v, torch.float64, dev).contiguous()
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"map shape {tuple(t.shape)} does not match the grid {tuple(shape)}")
    return t, 1


def auto_gate(p) -> np.ndarray:
    """The reference's auto gate (radiation_force.py:63-68): the time indices
    where the mean over cells of p^2 is at least 10 % of its peak; every
    index when none is (an all-NaN envelope).  The envelope is computed on
    the GPU in FP64."""
    dev = require_cuda()
    dt = _dtype_of(p) or torch.float32
    t = _record(p, dt, dev)
    nx, ny, nz, nt = t.shape
    e = ops.arf_envelope(t, nx * ny * nz, nt).cpu().numpy()
    mask = e >= 0.1 * e.max()
    return np.nonzero(mask)[0] if mask.any() else np.arange(nt)


def _gate_indices(gate, nt) -> np.ndarray:
    if isinstance(gate, slice):
        idx = np.arange(nt)[gate]
    else:
        g = np.asarray(gate.cpu() if is_tensor(gate) else gate)
        idx = np.nonzero(g)[0] if g.dtype == bool else g.astype(np.int64).ravel()
        idx = np.where(idx < 0, idx + nt, idx)
    if idx.size == 0:
        raise ValueError("gate selects no time index")
    if idx.min() < 0 or idx.max() >= nt:
        raise IndexError(f"gate index out of range for nt={nt}")
    return idx.astype(np.int32)


def _force(records, c_map, rho_map, alpha_coeff_map, f0, gate):
    dev = require_cuda()
    dt_in = _result_dtype(*records)
    dt_out = _result_dtype(*records, c_map, rho_map, alpha_coeff_map)
    recs = [_record(r, dt_in, dev) for r in records]
    nx, ny, nz, nt = recs[0].shape
    if any(tuple(r.shape) != (nx, ny, nz, nt) for r in recs):
        raise ValueError("pressure and velocity records must have the same shape")
    ncell = nx * ny * nz
    idx = auto_gate(recs[0]) if gate is None else _gate_indices(gate, nt)
    g = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).to(dev)
    maps = [_map(m, (nx, ny, nz), dev) for m in (c_map, rho_map, alpha_coeff_map)]
    strides = {s for _, s in maps}
    if len(strides) > 1:  # mix of scalars and fields: broadcast the scalars
        maps = [(m.expand(ncell).contiguous() if s == 0 else m, 1) for m, s in maps]
    stride = maps[0][1]
    # pressure alone, or pressure and 3 velocity components
    vel = recs[1:] if len(recs) == 4 else [None, None, None]
    outs = ops.arf_force(recs[0], *vel, [nx, ny, nz], nt, g, maps[0][0], maps[1][0], maps[2][0],
                         stride, float(f0), dt_out)
    if is_tensor(records[0]):
        return outs
    return [x.cpu().numpy() for x in outs]


def compute_radiation_force(pressure_4d, c_map, rho_map, alpha_coeff_map, f0, gate=None):
    """Body force b = 2 alpha_Np Isppa / c with Isppa = mean_gate(p^2) / (rho c)
    (radiation_force.py:27-85).  ``gate``: a slice, an index array, a boolean
    mask, or None for the auto gate.  Returns (nx, ny, nz)."""
    return _force([pressure_4d], c_map, rho_map, alpha_coeff_map, f0, gate)[0]


def compute_radiation_force_velocity(pressure_4d, velocity_u_4d, velocity_w_4d, velocity_v_4d,
                                     c_map, rho_map, alpha_coeff_map, f0, gate=None):
    """Vector body force from the time-averaged Poynting vector,
    b_i = 2 alpha_Np mean_gate(p v_i) / c (radiation_force.py:88-157); the
    gate comes from the pressure as in compute_radiation_force.  ``rho_map``
    is accepted for interface parity and unused, like the reference's.
    Returns (bx, by, bz)."""
    del rho_map  # interface parity with compute_radiation_force (unused)
    bx, by, bz = _force([pressure_4d, velocity_u_4d, velocity_w_4d, velocity_v_4d], c_map,
                        1.0, alpha_coeff_map, f0, gate)
    return bx, by, bz
