"""Drop-in ``shear_fdtd`` and projection / operator API on the B200 CUDA library.

Mirrors the public solver functions of pinton-lab/shearwave
(src/shearwave/solver.py): same argument order, array layout, opts keys,
error messages and returned ``(u, v)``.  All arithmetic runs in the sm_100a
kernels of ``libshearwave_b200.so``; this module validates arguments, moves
arrays to the device (torch owns the memory) and sequences the C-ABI calls.

Precision (``opts["precision"]``):

* ``"mixed"`` (default): FP32 fields in increment form (displacement and
  per-step increment stored, so the velocity never comes from a difference
  of two nearly equal displacements), FP64 projection; returns float32 like
  the reference.  ``opts["kahan"]=True`` adds a compensated displacement
  sum (12 more bytes read and written per cell-step) for very long runs:
  without it the measured error against the FP64 form is 2e-7 (u) and
  2.4e-6 (v) relative L2 after 4000 steps of the 256x256x384 layered case,
  growing about linearly with the step count.
* ``"fp64"``: the plain FP64 form, the reference's arithmetic in float64
  (matches an FP64 run of the reference to relative L2 <= 1e-10); returns
  float64.
"""

from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import torch

from . import _native, ops
from ._device import (
    dtype_code,
    is_tensor,
    np_dtype,
    ptr,
    require_cuda,
    stream_handle,
    to_device,
    to_host,
)

__all__ = [
    "divergence_center",
    "elastic_solve_static",
    "gradient_center",
    "hann1d",
    "laplacian_center",
    "project_body_force_to_shear",
    "project_vector_field",
    "shear_fdtd",
    "shear_fdtd_batch",
    "shear_fdtd_jax",
]

_PRECISION = {
    "mixed": _native.SW_MIXED_F32,
    "fp32": _native.SW_MIXED_F32,
    "float32": _native.SW_MIXED_F32,
    "fp64": _native.SW_PLAIN_F64,
    "plain": _native.SW_PLAIN_F64,
    "float64": _native.SW_PLAIN_F64,
}

# Force terms of one step the two-steps-per-pass kernel holds (its shared
# term buffer); a solve with more at any step runs one step per launch.
_TWO_STEP_TERM_CAP = 32


def _precision(opts: dict) -> int:
    p = opts.get("precision", "mixed")
    try:
        return _PRECISION[str(p).lower()]
    except KeyError:
        raise ValueError(f"precision must be one of {sorted(_PRECISION)}, got {p!r}") from None


def _field_dtype(prec: int) -> torch.dtype:
    return torch.float64 if prec == _native.SW_PLAIN_F64 else torch.float32


def _shape(a) -> tuple:
    return tuple(a.shape)


# ---------------------------------------------------------------------------
# FD operators (solver.py:686-729)
# ---------------------------------------------------------------------------
def _op_dtype(a) -> torch.dtype:
    dt = a.dtype if is_tensor(a) else np.asarray(a).dtype
    if dt in (torch.float32, np.float32):
        return torch.float32
    return torch.float64


def laplacian_center(field, dX, dY, dZ):
    """Compact 7-point Laplacian at cell centres, zero on the shell (solver.py:686-695)."""
    dev = require_cuda()
    f = to_device(field, _op_dtype(field), dev)
    out = ops.laplacian(f, [dX, dY, dZ])
    return out if is_tensor(field) else out.cpu().numpy()


def divergence_center(fx, fy, fz, dX, dY, dZ):
    """2h central divergence at cell centres, zero on the shell (solver.py:708-717)."""
    dev = require_cuda()
    dt = torch.promote_types(torch.promote_types(_op_dtype(fx), _op_dtype(fy)), _op_dtype(fz))
    a, b, c = (to_device(v, dt, dev) for v in (fx, fy, fz))
    out = ops.divergence(a, b, c, [dX, dY, dZ])
    return out if is_tensor(fx) else out.cpu().numpy()


def gradient_center(phi, dX, dY, dZ):
    """2h central gradient at cell centres, zero on the shell (solver.py:720-729)."""
    dev = require_cuda()
    p = to_device(phi, _op_dtype(phi), dev)
    g = ops.gradient(p, [dX, dY, dZ])
    return tuple(g) if is_tensor(phi) else tuple(t.cpu().numpy() for t in g)


# ---------------------------------------------------------------------------
# Projection (solver.py:644-683, 1010-1050)
# ---------------------------------------------------------------------------
_METHODS = ("cg", "spectral")


def _projection_method(choice: str, prec: int, tol: float) -> str:
    """Resolve opts["projection"].

    "auto": the plain FP64 form always runs the reference's CG (its 1e-10
    parity is with the CG's truncated iterate); the mixed form uses the exact
    spectral solve when poisson_tol <= 1e-8, where it differs from the
    reference's converged CG by less than the CG's own truncation (far inside
    the 1e-4 budget), and the CG otherwise.
    """
    if choice == "auto":
        if prec == _native.SW_PLAIN_F64:
            return "cg"
        return "spectral" if float(tol) <= 1e-8 else "cg"
    if choice not in _METHODS:
        raise ValueError(f"projection must be 'auto' or one of {_METHODS}")
    return choice


_CG_REASONS = _native.CG_REASONS


def _stats_dict(st: torch.Tensor, method: str = "cg") -> dict:
    """A host stats row [iters, reason, rel, max_div] as the info dict."""
    v = st.tolist()
    return {"iters": int(v[0]), "reason": _CG_REASONS.get(int(v[1]), str(int(v[1]))),
            "rel": float(v[2]), "max_div": float(v[3]), "method": method}


def _project_raw(comps, spacing, tol, max_iters, method: str = "cg"):
    """Project device components (CG or the direct spectral solve): returns
    the padded FP64 result (3, ncell) and the info dict."""
    out, st = ops.project(*comps, list(spacing), float(tol), int(max_iters), method)
    return out, _stats_dict(st, method)


def _unpad(fs: torch.Tensor, shape, dt: torch.dtype, dev) -> list[torch.Tensor]:
    nx, ny, nz = shape
    outs = []
    for c in range(3):
        o = torch.empty((nx, ny, nz), dtype=dt, device=dev)
        ops.convert_(o, fs[c], 1, [nx, ny, nz], [0, ny * nz, nz, 1], 1.0, None, [0, 0, 0])
        outs.append(o)
    return outs


def project_vector_field(fx, fy, fz, dX, dY, dZ, tol, max_iters, *, info=None, method="cg"):
    """Helmholtz-Hodge projection onto discretely divergence-free fields.

    solver.py:644-683.  The CG (solver.py:1010-1050) runs in FP64 on the GPU
    with the reference's stopping rule.  ``method="spectral"`` solves the
    Poisson problem directly instead (exact solution, ``tol`` and
    ``max_iters`` unused).  Returns three arrays in the input dtype (float32
    unless the inputs are float64).  ``info`` (dict) receives the CG
    iteration count and exit reason.
    """
    if method not in _METHODS:
        raise ValueError(f"method must be one of {_METHODS}")
    dev = require_cuda()
    dt = torch.promote_types(torch.promote_types(_op_dtype(fx), _op_dtype(fy)), _op_dtype(fz))
    comps = [to_device(v, dt, dev) for v in (fx, fy, fz)]
    shape = _shape(comps[0])
    if any(_shape(c) != shape for c in comps) or len(shape) != 3:
        raise ValueError("fx, fy, fz must be 3-D arrays of the same shape")
    fs, st = _project_raw(comps, (dX, dY, dZ), tol, max_iters, method)
    if info is not None:
        info.update(st)
    outs = _unpad(fs, shape, dt, dev)
    if is_tensor(fx):
        return tuple(outs)
    return tuple(o.cpu().numpy() for o in outs)


def elastic_solve_static(bz, dX, dY, dZ, mu, tol=1e-6, max_iters=1500, *, verbose=False,
                         info=None):
    """Solve ``mu * laplace(u) = -bz`` (zero shell) by CG on ``(-mu L7) u = bz``.

    solver.py:569-625, with the reference's loop (break on ``p.Ap <= 0``,
    stop at ``sqrt(r.r / rs0) < tol``) in FP64 on the GPU.  Returns u in the
    dtype of ``bz`` (float32 unless bz is float64).
    """
    dev = require_cuda()
    dt = _op_dtype(bz)
    b = to_device(bz, dt, dev)
    shape = _shape(b)
    if len(shape) != 3:
        raise ValueError("bz must be a 3-D array")
    nx, ny, nz = shape
    m, ms = _material(mu, shape, dt, dev)
    out, st = ops.static_solve(b, m, float(ms), [dX, dY, dZ], float(tol), int(max_iters))
    u = torch.empty(shape, dtype=dt, device=dev)
    ops.convert_(u, out[0], 1, [nx, ny, nz], [0, ny * nz, nz, 1], 1.0, None, [0, 0, 0])
    d = _stats_dict(st)
    d.pop("method")
    if verbose:
        print(f"CG (GPU): it={d['iters']}/{max_iters}, rel={d['rel']:.3e}, {d['reason']}")
    if info is not None:
        info.update(d)
    return u if is_tensor(bz) else u.cpu().numpy()


def project_body_force_to_shear(bz, dX, dY, dZ, tol=5e-5, max_iters=400):
    """Project a z-only body force (solver.py:628-641)."""
    z = np.zeros(_shape(bz), dtype=np.float32)
    b = bz if is_tensor(bz) else np.asarray(bz, dtype=np.float32)
    return project_vector_field(z, z, b, dX, dY, dZ, tol, max_iters)


# ---------------------------------------------------------------------------
# shear_fdtd (solver.py:27-243) and the shear_fdtd_jax extras (246-566)
# ---------------------------------------------------------------------------
def hann1d(n):
    """1-D Hann window of length n as float32 (solver.py:1053-1057); host helper
    used to taper synthetic sources."""
    if n <= 1:
        return np.ones((n,), dtype=np.float32)
    return np.hanning(n).astype(np.float32)


def _check_jax_kwargs(n_steps, trace_indices, return_traces, snapshot_stride):
    """Validation of solver.py:290-303 and 396-408."""
    if return_traces and trace_indices is None:
        raise ValueError("trace_indices must be provided when return_traces=True.")
    if snapshot_stride is not None:
        if not isinstance(snapshot_stride, (int, np.integer)) or int(snapshot_stride) <= 0:
            raise ValueError("snapshot_stride must be a positive integer.")
        snapshot_stride = int(snapshot_stride)
        if n_steps % snapshot_stride != 0:
            raise ValueError(
                f"n_steps ({n_steps}) must be a multiple of snapshot_stride ({snapshot_stride})."
            )
        if return_traces:
            raise ValueError("return_traces and snapshot_stride are not both supported in v1.")
    cells = None
    if trace_indices is not None:
        if not isinstance(trace_indices, (tuple, list)) or len(trace_indices) != 3:
            raise ValueError("trace_indices must be a 3-tuple: (ix, iy, iz).")
        ix, iy, iz = (np.asarray(t, dtype=np.int32) for t in trace_indices)
        if not (ix.shape == iy.shape == iz.shape):
            raise ValueError("trace index arrays must share the same shape.")
        if ix.ndim != 1:
            raise ValueError("trace index arrays must be 1D.")
        cells = np.stack([ix, iy, iz], axis=1)
    return snapshot_stride, cells


def _material(v, shape, dt, dev):
    """(device array or None, scalar) for a material input (solver.py:1072-1079)."""
    if np.isscalar(v):
        return None, float(v)
    if _shape(v) != shape:
        raise ValueError("Material field has incompatible shape.")
    return to_device(v, dt, dev), 0.0


class _Forces:
    """Force terms of one solve: projected patterns plus the per-step table."""

    def __init__(self):
        self.separable = []      # list of ((bx, by, bz) device 3-D or None, env np array)
        self.stream4d = None     # (bx, by, bz) device 4-D or 3-D or None, for per-step projection
        self.zero_steps = None   # bool per step (4-D mode): the force slice is identically zero


def _gather_forces(bx, by, bz, opts, shape, n_steps, dt, dev, np_dt) -> _Forces:
    fr = _Forces()
    env_t = opts.get("env_t")

    def dev3(b):
        if b is None:
            return None
        if len(_shape(b)) != 3 or _shape(b) != shape:
            raise ValueError("Body-force component has incompatible shape.")
        return to_device(b, dt, dev)

    if env_t is not None:
        env = np.asarray(env_t.cpu() if is_tensor(env_t) else env_t, dtype=np_dt).ravel()
        if env.shape[0] != n_steps:
            raise ValueError(f"env_t length ({env.shape[0]}) must equal n_steps ({n_steps}).")
        fr.separable.append(((dev3(bx), dev3(by), dev3(bz)), env))
    else:
        comps = []
        any4 = False
        for b in (bx, by, bz):
            if b is None:
                comps.append(None)
                continue
            s = _shape(b)
            if len(s) == 3 and s == shape:
                comps.append(b)
            elif len(s) == 4 and s == (*shape, n_steps):
                comps.append(b)
                any4 = True
            else:
                raise ValueError("Body-force component has incompatible shape.")
        if not any4:
            # 3-D forces without env_t: the reference repeats them over every step
            # and projects each identical slice; one projection with scale 1 is
            # the same result.
            fr.separable.append((tuple(dev3(b) for b in comps), np.ones(n_steps, dtype=np_dt)))
        else:
            zero = np.ones(n_steps, dtype=bool)
            dcomps = []
            for b in comps:
                if b is None:
                    dcomps.append(None)
                    continue
                if len(_shape(b)) == 4:
                    if is_tensor(b):
                        nz_t = (b.reshape(-1, n_steps) != 0).any(0).cpu().numpy()
                    else:
                        nz_t = np.any(np.asarray(b).reshape(-1, n_steps) != 0, axis=0)
                    zero &= ~nz_t
                else:
                    zero &= not bool(np.any(np.asarray(b.cpu() if is_tensor(b) else b) != 0))
                dcomps.append(to_device(b, dt, dev))
            fr.stream4d = dcomps
            fr.zero_steps = zero
    for term in opts.get("force_terms") or ():
        if isinstance(term, dict):
            tb = (term.get("bx"), term.get("by"), term.get("bz"))
            tenv = term["env"]
        else:
            (tb, tenv) = term
        env = np.asarray(tenv.cpu() if is_tensor(tenv) else tenv, dtype=np_dt).ravel()
        if env.shape[0] != n_steps:
            raise ValueError(f"env_t length ({env.shape[0]}) must equal n_steps ({n_steps}).")
        fr.separable.append((tuple(dev3(b) for b in tb), env))
    return fr


class _Run:
    """Device state of one shear_fdtd solve: the tensors the time-loop ops
    read and write (``bundle()``) and its scalar settings."""

    def __init__(self, shape, spacing, dT, n_steps, prec, kahan, dev):
        self.dev = dev
        self.shape = shape
        self.nx, self.ny, self.nz = shape
        self.pz = ops.pitch(self.nz)
        self.ncell = self.nx * self.ny * self.pz
        self.prec = prec
        self.dt = _field_dtype(prec)
        self.spacing = tuple(float(h) for h in spacing)
        self.dT = float(dT)
        self.n_steps = int(n_steps)
        self.kahan = 1 if kahan else 0
        self.vel_damp = 0.0
        self.kernel = 0          # 0 TMA-staged step kernels, 1 direct loads
        self.xchunk = 0
        self.steps_per_pass = 0
        self.has_eta = 0
        self.snap_stride = 0
        self.stall_test = 0      # testing switch of the step kernels (sw_fdtd_desc.stall_test)
        nbuf, ncomp = (3, 3) if prec == _native.SW_PLAIN_F64 else (3, 9)
        self.state = torch.empty((nbuf, ncomp, self.ncell), dtype=self.dt, device=dev)
        # material coefficients: one allocation, component 0 the mu term,
        # component 1 the eta term (used only with viscosity)
        self.coef = torch.zeros((2, self.ncell), dtype=self.dt, device=dev)
        self.inv_rho = None
        if prec == _native.SW_PLAIN_F64:
            self.inv_rho = torch.zeros(self.ncell, dtype=self.dt, device=dev)
        self.flags = torch.zeros(1, dtype=torch.int32, device=dev)
        # device step counter: lets the library replay the loop as CUDA graphs
        self.clock = torch.zeros(1, dtype=torch.int32, device=dev)
        # launch-wide tile queue of this solve's step launches
        self.queue = torch.zeros(2, dtype=torch.int32, device=dev)
        # force patterns and term table (set by set_patterns)
        self.patterns = torch.zeros((1, 3, 0), dtype=self.dt, device=dev)
        self.term_off = torch.zeros(self.n_steps + 1, dtype=torch.int32, device=dev)
        self.term_pat = torch.zeros(1, dtype=torch.int32, device=dev)
        self.term_scale = torch.zeros(1, dtype=torch.float64, device=dev)
        self.snaps = None
        self.trace_cells = None
        self.traces = None
        self.keep = []  # inputs the device work still reads

    def fparams(self) -> list[float]:
        return [*self.spacing, self.dT, float(self.vel_damp)]

    def iparams(self) -> list[int]:
        return [self.prec, self.nx, self.ny, self.nz, self.n_steps, self.kahan,
                self.snap_stride, self.xchunk, self.steps_per_pass, self.kernel, self.has_eta,
                self.stall_test]

    def bundle(self) -> tuple:
        """Arguments shared by the fdtd ops (shearwave_b200.ops)."""
        return (self.state, self.coef, self.inv_rho, self.patterns, self.term_off,
                self.term_pat, self.term_scale, self.snaps, self.trace_cells, self.traces,
                self.flags, self.clock, self.queue, self.fparams(), self.iparams())

    @property
    def desc(self) -> _native.FdtdDesc:
        """The C-ABI descriptor of this solve (built from the tensors)."""
        return ops.make_desc(*self.bundle())

    def materials(self, rho, mu, eta, in_dt):
        dev = self.dev
        r, rs = _material(rho, self.shape, in_dt, dev)
        m, ms = _material(mu, self.shape, in_dt, dev)
        eta_mode, e, es = 0, None, 0.0
        if eta is not None:
            eta_mode = 1
            e, es = _material(eta, self.shape, in_dt, dev)
            self.has_eta = 1
        ops.fdtd_materials_(*self.bundle(), r, float(rs), m, float(ms), eta_mode, e, float(es))
        self.rho_dev, self.rho_s = r, rs
        self.keep += [r, m, e]

    def set_patterns(self, pats: torch.Tensor, term_off, term_pat, term_scale):
        self.patterns = pats
        self.term_off = torch.as_tensor(np.asarray(term_off, np.int32), device=self.dev)
        if len(term_pat):
            self.term_pat = torch.as_tensor(np.asarray(term_pat, np.int32), device=self.dev)
            self.term_scale = torch.as_tensor(np.asarray(term_scale, np.float64),
                                              device=self.dev)

    def pattern_from_tensor(self, fs: torch.Tensor, dst: torch.Tensor, spacing_dt2: float):
        """Store a projected force (3 padded FP64 components) as a pattern of this form."""
        strides = [self.ncell, self.ny * self.pz, self.pz, 1]
        if self.prec == _native.SW_PLAIN_F64:
            ops.convert_(dst, fs, 3, list(self.shape), strides, 1.0, None, [0, 0, 0])
        else:
            # dT^2 f_S / rho in FP32
            r = self.rho_dev
            if r is None:
                ops.convert_(dst, fs, 3, list(self.shape), strides, spacing_dt2 / self.rho_s,
                             None, [0, 0, 0])
            else:
                ops.convert_(dst, fs, 3, list(self.shape), strides, spacing_dt2, r,
                             [self.ny * self.nz, self.nz, 1])


def validate_inputs(bx, by, bz, rho, mu, eta, opts, shape, n_steps) -> None:
    """Every shape / length check of solver.py:88-171, 1060-1079 on the host.

    Raises the reference's ValueError messages before any device work.
    """
    env_t = opts.get("env_t")
    for b in (bx, by, bz):
        if b is None:
            continue
        s = _shape(b)
        ok = s == shape if env_t is not None else (s == shape or s == (*shape, n_steps))
        if not ok:
            raise ValueError("Body-force component has incompatible shape.")
    if env_t is not None:
        n_env = int(np.asarray(env_t.cpu() if is_tensor(env_t) else env_t).size)
        if n_env != n_steps:
            raise ValueError(f"env_t length ({n_env}) must equal n_steps ({n_steps}).")
    for term in opts.get("force_terms") or ():
        tb, tenv = ((term.get("bx"), term.get("by"), term.get("bz")), term["env"]) \
            if isinstance(term, dict) else term
        for b in tb:
            if b is not None and _shape(b) != shape:
                raise ValueError("Body-force component has incompatible shape.")
        n_env = int(np.asarray(tenv.cpu() if is_tensor(tenv) else tenv).size)
        if n_env != n_steps:
            raise ValueError(f"env_t length ({n_env}) must equal n_steps ({n_steps}).")
    for m in (rho, mu) + (() if eta is None else (eta,)):
        if not np.isscalar(m) and _shape(m) != shape:
            raise ValueError("Material field has incompatible shape.")
    for key in ("initial_u", "initial_v"):
        a = opts.get(key)
        if a is not None and _shape(a) != (*shape, 3):
            raise ValueError(f"{key} must match shape (nx,ny,nz,3)")


def _prepare_opts(opts):
    opts = dict(opts or {})
    reproject_every = int(opts.get("reproject_every", 0) or 0)
    if reproject_every < 0:
        raise ValueError("reproject_every must be a non-negative integer.")
    return opts, reproject_every


class _Solve:
    """Device state and phases of one shear_fdtd problem.

    Construction validates the arguments (the reference's checks and
    messages), uploads inputs, computes the material coefficients, the
    initial state and allocates the outputs.  The force projection, the time
    loop and the outputs are separate phases so that a batch of solves can
    run each phase for all of them together.
    """

    def __init__(self, bx, by, bz, rho, mu, dX, dY, dZ, dT, n_steps, opts, *,
                 snapshot_stride=None, trace_indices=None, return_traces=False):
        ref = bx if bx is not None else (by if by is not None else bz)
        if ref is None:
            raise ValueError("At least one body-force component must be provided.")
        opts, self.reproject_every = _prepare_opts(opts)
        if snapshot_stride is None:
            snapshot_stride = opts.get("snapshot_stride")
        snapshot_stride, trace_cells = _check_jax_kwargs(n_steps, trace_indices, return_traces,
                                                         snapshot_stride)
        n_steps = int(n_steps)
        self.opts = opts
        self.n_steps = n_steps
        self.spacing = (dX, dY, dZ)
        self.dT = dT
        self.tol = opts.get("poisson_tol", 1e-5)
        self.max_iters = opts.get("poisson_max_iters", 200)
        self.verbose = opts.get("verbose", False)
        self.progress_every = opts.get("progress_every", max(1, n_steps // 10))
        self.info = opts.get("info")
        self.prec = _precision(opts)
        dt = self.dt = _field_dtype(self.prec)
        np_dt = np_dtype(dt)
        shape = self.shape = tuple(int(s) for s in _shape(ref)[:3])
        nx, ny, nz = shape
        if trace_cells is not None and trace_cells.size:
            if np.any(trace_cells < 0) or np.any(trace_cells >= np.asarray(shape)):
                raise ValueError("trace_indices outside the grid.")
        eta = opts.get("eta", 0.0)
        if np.isscalar(eta):
            eta = float(eta) if float(eta) != 0.0 else None
        validate_inputs(bx, by, bz, rho, mu, eta, opts, shape, n_steps)
        kern = opts.get("step_kernel", "tma")
        if kern not in ("tma", "direct"):
            raise ValueError("step_kernel must be 'tma' or 'direct'")
        self.method = _projection_method(opts.get("projection", "auto"), self.prec, self.tol)
        dev = self.dev = require_cuda()
        self.forces = _gather_forces(bx, by, bz, opts, shape, n_steps, dt, dev, np_dt)

        self.tev = None  # CUDA events: start, steps begin, steps end, done
        if self.info is not None:
            self.tev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            self.tev[0].record()
        run = self.run = _Run(shape, (dX, dY, dZ), dT, n_steps, self.prec,
                              opts.get("kahan", False), dev)
        run.vel_damp = float(opts.get("vel_damp", 0.0))
        run.kernel = 0 if kern == "tma" else 1
        run.xchunk = int(opts.get("xchunk", 0) or 0)
        spp = int(opts.get("steps_per_pass", 0) or 0)
        if spp not in (0, 1, 2):
            raise ValueError("steps_per_pass must be 1 or 2 (0 = automatic)")
        run.steps_per_pass = spp
        if not opts.get("cuda_graph", True):
            run.clock = None
        run.materials(rho, mu, eta, dt)
        iu = iv = None
        if opts.get("initial_u") is not None:
            iu = to_device(opts["initial_u"], dt, dev)
        if opts.get("initial_v") is not None:
            iv = to_device(opts["initial_v"], dt, dev)
        ops.fdtd_init_(*run.bundle(), iu, iv)

        self.n_sep = len(self.forces.separable)
        # 4-D forces: every step whose force slice is non-zero is projected up
        # front (one batched CG over the slices) and kept on the device as a
        # pattern of its own, so the time loop streams them from HBM with no
        # host work between steps -- unless the patterns would take more
        # than opts["force_stream_bytes"] (4 GiB), in which case each slice
        # is projected on the host's cue just before its step
        self.stream_steps = None
        n_pat = self.n_sep
        if self.forces.stream4d is not None:
            nzs = [it for it in range(n_steps) if not self.forces.zero_steps[it]]
            need = len(nzs) * 3 * run.ncell * run.state.element_size()
            if need <= int(opts.get("force_stream_bytes", 4 << 30)):
                self.stream_steps = nzs
                n_pat += len(nzs)
            else:
                n_pat += 1
        self.pats = torch.zeros((max(n_pat, 1), 3, run.ncell), dtype=dt, device=dev)
        self.cg_log = []

        self.snaps = None
        if snapshot_stride:
            self.snaps = torch.zeros((n_steps // snapshot_stride, nx, ny, nz, 3), dtype=dt,
                                     device=dev)
            run.snap_stride = snapshot_stride
            run.snaps = self.snaps
        self.traces = None
        if trace_cells is not None and return_traces:
            tc = torch.as_tensor(trace_cells.reshape(-1), dtype=torch.int32, device=dev)
            self.traces = torch.zeros((trace_cells.shape[0], n_steps), dtype=dt, device=dev)
            run.trace_cells = tc
            run.traces = self.traces

    # ---- phases ---------------------------------------------------------
    def needs_per_step_host(self, callback) -> bool:
        """Whether the time loop must return to the host between steps."""
        return (callback is not None or self._host_projects_4d()
                or bool(self.reproject_every) or bool(self.verbose)
                or self.run.traces is not None or self.run.kernel != 0)

    def _host_projects_4d(self) -> bool:
        return self.forces.stream4d is not None and self.stream_steps is None

    def separable_inputs(self):
        """(pattern index, device components) of every separable force term."""
        return [(k, comps) for k, (comps, _env) in enumerate(self.forces.separable)]

    def _slice(self, it):
        """The force components of step it in 4-D mode (solver.py:198-199)."""
        return [None if b is None else (b[..., it] if b.dim() == 4 else b).contiguous()
                for b in self.forces.stream4d]

    def stream_inputs(self):
        """(pattern index, device components) of every 4-D force slice that is
        projected up front (the non-zero steps, in step order)."""
        if self.stream_steps is None:
            return []
        return [(self.n_sep + j, self._slice(it)) for j, it in enumerate(self.stream_steps)]

    def projection_inputs(self):
        return self.separable_inputs() + self.stream_inputs()

    def store_pattern(self, k: int, fs_out: torch.Tensor):
        """Store a projected pattern (3 padded FP64 components) as term k."""
        self.run.pattern_from_tensor(fs_out, self.pats[k], self.dT * self.dT)

    def build_terms(self):
        f = self.forces
        if self.stream_steps is not None:
            self._stream_index = {it: j for j, it in enumerate(self.stream_steps)}
        term_off, term_pat, term_scale = [0], [], []
        for it in range(self.n_steps):
            for k, (_c, env) in enumerate(f.separable):
                s = float(env[it])
                if s != 0.0:
                    term_pat.append(k)
                    term_scale.append(s)
            if f.stream4d is not None and not f.zero_steps[it]:
                term_pat.append(self.n_sep + (self._stream_index[it] if self.stream_steps
                                              is not None else 0))
                term_scale.append(1.0)
            term_off.append(len(term_pat))
        self.term_off = term_off
        if max((b - a for a, b in zip(term_off, term_off[1:])), default=0) > _TWO_STEP_TERM_CAP:
            # the two-steps-per-pass kernel holds at most this many force terms
            # of one step; more run one step per launch
            self.run.steps_per_pass = 1
        self.run.set_patterns(self.pats, term_off, term_pat, term_scale)

    def mark_steps_begin(self):
        if self.tev is not None:
            self.tev[1].record()

    def finish(self, return_device: bool):
        """Outputs of a finished solve (finish_enqueue + finish_collect)."""
        return self.finish_collect(self.finish_enqueue(return_device))

    def finish_enqueue(self, return_device: bool, copy_stream=None):
        """Enqueue the output conversion (and, for host outputs, copies into
        pinned host buffers on ``copy_stream``, which waits for the
        conversion); nothing here waits for the GPU.  Returns the handle that
        finish_collect turns into the result once the copies are done."""
        run, dt, dev = self.run, self.dt, self.dev
        nx, ny, nz = self.shape
        if self.tev is not None:
            self.tev[2].record()
        u, v = ops.fdtd_finish(*run.bundle(), self.n_steps, True)
        outs = [u, v]
        if self.snaps is not None:
            outs.append(self.snaps)
        elif self.traces is not None:
            outs.append(self.traces)
        if self.tev is not None:
            self.tev[3].record()
        flag = torch.empty(1, dtype=torch.int32, pin_memory=True)
        if return_device:
            flag.copy_(run.flags, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record()
            return {"outs": outs, "flag": flag, "event": ev, "device": True}
        done = torch.cuda.Event()
        done.record()
        cs = copy_stream if copy_stream is not None else torch.cuda.current_stream()
        cs.wait_event(done)
        host = []
        with torch.cuda.stream(cs):
            for t in outs:
                h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                h.copy_(t, non_blocking=True)
                t.record_stream(cs)  # the device buffer lives until the copy ran
                host.append(h)
            flag.copy_(run.flags, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(cs)
        return {"outs": host, "flag": flag, "event": ev, "device": False}

    def finish_collect(self, handle):
        """Wait for a finish_enqueue handle and return the solve's result."""
        handle["event"].synchronize()
        nonfinite = bool(int(handle["flag"][0]) & _native.FLAG_NONFINITE)
        if self.info is not None:
            tev = self.tev
            tev[3].synchronize()
            self.info.update(
                cg=self.cg_log, nonfinite=nonfinite,
                precision="fp64" if self.prec == _native.SW_PLAIN_F64 else "mixed",
                t_setup_ms=tev[0].elapsed_time(tev[1]),
                t_steps_ms=tev[1].elapsed_time(tev[2]),
                t_finish_ms=tev[2].elapsed_time(tev[3]),
                n_push_steps=int(sum(1 for i in range(self.n_steps)
                                     if self.term_off[i + 1] > self.term_off[i])))
        flags = int(handle["flag"][0])
        if flags & _native.FLAG_TIMEOUT:
            raise RuntimeError(
                "shear_fdtd: a step kernel's bounded device wait ran out and its tiles of this "
                "solve were abandoned (SW_ETIMEOUT); the result is incomplete")
        if flags & _native.FLAG_REFUSED:
            raise RuntimeError(
                "shear_fdtd: a step launch refused to issue a TMA copy to a misaligned "
                "shared-memory destination (SW_ETIMEOUT); the result is incomplete")
        if nonfinite:
            warnings.warn("shear_fdtd: non-finite displacement encountered (unstable dT?)",
                          RuntimeWarning, stacklevel=3)
        if handle["device"]:
            return tuple(handle["outs"])
        return tuple(h.numpy() for h in handle["outs"])

    def run_loop(self, callback):
        """The time loop of solver.py:194-239 for this solve alone."""
        run, dt, dev = self.run, self.dt, self.dev
        nx, ny, nz = self.shape
        n_steps = self.n_steps
        dX, dY, dZ = self.spacing
        f = self.forces
        per_step = callback is not None or self._host_projects_4d()
        events = set()
        if self.reproject_every:
            events.update(range(self.reproject_every, n_steps + 1, self.reproject_every))
        if self.verbose:
            events.update(range(self.progress_every, n_steps + 1, self.progress_every))
        self.mark_steps_begin()
        it = 0
        while it < n_steps:
            if per_step:
                end = it + 1
            else:
                later = [e for e in events if e > it]
                end = min(later) if later else n_steps
            if self._host_projects_4d() and not f.zero_steps[it]:
                # per-step projection of b[..., it] (solver.py:198-199)
                fs, st = _project_raw(self._slice(it), (dX, dY, dZ), self.tol,
                                      self.max_iters, self.method)
                self.cg_log.append(st)
                self.store_pattern(self.n_sep, fs)
            ops.fdtd_steps_(*run.bundle(), it, end - it)
            if callback is not None:
                u_cb, _ = ops.fdtd_finish(*run.bundle(), end, False)
                callback(end - 1, u_cb.cpu().numpy())
            if self.verbose and end % self.progress_every == 0:
                print(f"FDTD it={end}/{n_steps}")
            if self.reproject_every and end % self.reproject_every == 0:
                st = ops.fdtd_reproject_(*run.bundle(), end, float(self.tol),
                                         int(self.max_iters))
                self.cg_log += [_stats_dict(st[0]), _stats_dict(st[1])]
            it = end


def shear_fdtd(
    bx,
    by,
    bz,
    rho,
    mu,
    dX,
    dY,
    dZ,
    dT,
    n_steps,
    opts=None,
    callback=None,
    *,
    trace_indices=None,
    return_traces=False,
    return_device=False,
    snapshot_stride=None,
):
    """3-D collocated cell-centred shear FDTD solver on a B200 (drop-in).

    Same contract as the reference ``shear_fdtd`` (solver.py:27-243): forces
    ``(nx,ny,nz)`` (with ``opts["env_t"]``) or ``(nx,ny,nz,n_steps)``,
    scalar or ``(nx,ny,nz)`` materials, the same opts keys (``vel_damp``,
    ``eta``, ``env_t``, ``poisson_tol``, ``poisson_max_iters``,
    ``reproject_every``, ``verbose``, ``progress_every``, ``initial_u``,
    ``initial_v``) and returns ``(u, v)`` of shape ``(nx, ny, nz, 3)``.

    Also accepts the ``shear_fdtd_jax`` keywords (solver.py:259-262):
    ``snapshot_stride`` (adds ``u`` snapshots after every k steps as a third
    return value), ``trace_indices`` / ``return_traces`` (z-displacement
    traces ``(n_traces, n_steps)``) and ``return_device`` (torch CUDA tensors
    instead of numpy arrays).

    Additional opts: ``precision`` ("mixed" default, or "fp64"), ``projection``
    ("auto" default: the reference's CG for fp64, and for mixed the exact
    direct spectral Poisson solve when ``poisson_tol <= 1e-8``; or "cg" /
    "spectral" explicitly), ``kahan`` (False: compensated displacement sum), ``step_kernel`` ("tma" default, or "direct"), ``xchunk`` (planes
    per tile along x, 0 = automatic), ``steps_per_pass`` (mixed form: 2
    fuses two time steps per pass over HBM, except with ``kahan``; 1 one
    step per launch; 0 (default) two), ``cuda_graph`` (True: long step runs replay one instantiated CUDA
    graph of 32 steps), ``force_terms`` (extra separable terms:
    list of ``((bx, by, bz), env)``), ``force_stream_bytes`` (4-D forces: the
    non-zero slices are projected up front and streamed from the device
    while their patterns fit in this many bytes, 4 GiB by default; above it
    each slice is projected just before its step), ``snapshot_stride`` (alias of the
    keyword), ``info`` (dict filled with CG statistics, phase times and a
    non-finite flag).

    ``callback(it, u)`` is called after every step with a host copy of the new
    displacement (the reference passes its live buffer; writing into the copy
    does not feed back into the solve).
    """
    sv = _Solve(bx, by, bz, rho, mu, dX, dY, dZ, dT, n_steps, opts,
                snapshot_stride=snapshot_stride, trace_indices=trace_indices,
                return_traces=return_traces)
    return _solve_alone(sv, callback, return_device)


def _solve_alone(sv: _Solve, callback, return_device):
    """Projection, time loop and outputs of one solve."""
    if sv.verbose and sv.n_sep:
        print("Pre-computing Helmholtz projection (separable force)...")
    _project_inputs([sv])
    sv.build_terms()
    sv.run_loop(callback)
    return sv.finish(return_device)


def shear_fdtd_batch(problems, *, precision=None, return_device=False, errors="raise"):
    """Run many independent ``shear_fdtd`` problems together on one GPU.

    ``problems`` is a sequence of dicts of ``shear_fdtd`` keyword arguments
    (``bx, by, bz, rho, mu, dX, dY, dZ, dT, n_steps, opts`` and optionally
    ``snapshot_stride``); grids, materials, pushes and ``n_steps`` may all
    differ.  The force projections of all problems run as one batched CG
    (every launch advances every unfinished solve) and the time loops as one
    launch per pair of steps (per step where a solve starts or ends, or with
    ``steps_per_pass=1`` or ``kahan``) over the tiles of every running solve.  ``precision``
    overrides ``opts["precision"]`` for all problems.

    Problems that need the host between steps (callback-free here, but 4-D
    forces, ``reproject_every``, ``verbose``, traces or the direct kernels)
    are run one after another through :func:`shear_fdtd` on the same GPU.
    Returns a list of ``shear_fdtd`` results in input order.

    A solve whose device work was abandoned (a step kernel's bounded wait
    ran out) fails alone: the other solves' results are unaffected.  With
    ``errors="raise"`` (default) the first such error is raised once every
    solve has been collected; with ``errors="return"`` the failed solve's
    slot holds the exception instead of a result.
    """
    if errors not in ("raise", "return"):
        raise ValueError("errors must be 'raise' or 'return'")
    solves, results = [], [None] * len(problems)
    for i, p in enumerate(problems):
        opts = dict(p.get("opts") or {})
        if precision is not None:
            opts["precision"] = precision
        kw = {k: p[k] for k in ("bx", "by", "bz", "rho", "mu", "dX", "dY", "dZ", "dT", "n_steps")}
        sv = _Solve(**kw, opts=opts, snapshot_stride=p.get("snapshot_stride"))
        if sv.needs_per_step_host(None):
            results[i] = _solve_alone(sv, None, return_device)
            continue
        solves.append((i, sv))
    if not solves:
        return results
    precs = {sv.prec for _, sv in solves}
    groups = [[(i, sv) for i, sv in solves if sv.prec == pr] for pr in sorted(precs)]
    copy_stream = None if return_device else torch.cuda.Stream(device=solves[0][1].dev)
    first_error = None
    for group in groups:
        handles = _run_batch_group([sv for _, sv in group], return_device, copy_stream)
        for (i, sv), h in zip(group, handles):
            try:
                results[i] = sv.finish_collect(h)
            except RuntimeError as e:
                results[i] = e
                first_error = first_error or e
    if first_error is not None and errors == "raise":
        raise first_error
    return results


def _run_batch_group(solves, return_device, copy_stream):
    """Batched projection + batched time loop for solves of one precision.

    The loop is enqueued in segments that end where a solve ends; each
    finished solve's output conversion and copy to pinned host memory
    (``copy_stream``) are enqueued right there, so they run while the
    longer solves are still stepping.  Returns one finish handle per solve.
    """
    # ---- batched projection of every pattern ----
    _project_inputs(solves)
    for sv in solves:
        sv.build_terms()
        sv.mark_steps_begin()
    # ---- batched time loop ----
    n = len(solves)
    handles = [None] * n
    it = 0
    for end in sorted({sv.n_steps for sv in solves}):
        if end > it:
            _batch_steps([sv.run for sv in solves], [], it, end - it)
            it = end
        for k, sv in enumerate(solves):
            if sv.n_steps == end:
                handles[k] = sv.finish_enqueue(return_device, copy_stream)
    return handles


def _project_inputs(solves, chunk=16):
    """Project every force pattern of the solves (separable terms and the
    non-zero 4-D slices) and store them: the spectral solves one by one, the
    CG solves as batched CGs of up to ``chunk`` fields (every CG launch
    advances all of them, each with its own stopping rule)."""
    jobs = []
    for sv in solves:
        for k, comps in sv.projection_inputs():
            if sv.method == "spectral":  # direct solves: one after another, each ~1 ms
                fs, st = _project_raw(comps, sv.spacing, sv.tol, sv.max_iters, "spectral")
                sv.cg_log.append(st)
                sv.store_pattern(k, fs)
            else:
                jobs.append((comps, sv, k))
    for dt in sorted({sv.dt for _, sv, _ in jobs}, key=str):
        same = [j for j in jobs if j[1].dt == dt]
        for a in range(0, len(same), chunk):
            part = same[a:a + chunk]
            outs, stats = ops.project_batch(
                [c[0] for c, _, _ in part], [c[1] for c, _, _ in part],
                [c[2] for c, _, _ in part], [h for _, sv, _ in part for h in sv.spacing],
                [float(sv.tol) for _, sv, _ in part], [int(sv.max_iters) for _, sv, _ in part])
            for (_, sv, k), fs, st in zip(part, outs, stats):
                sv.cg_log.append(_stats_dict(st))
                sv.store_pattern(k, fs)


def _batch_steps(runs, begins, it0, nsteps):
    """One fdtd_batch_steps_ call over the solves' device state (begins: an
    empty list starts every solve at step 0)."""
    b = [r.bundle() for r in runs]
    ops.fdtd_batch_steps_([x[0] for x in b], [x[1] for x in b], [x[2] for x in b],
                          [x[3] for x in b],
                          [x[4] for x in b], [x[5] for x in b], [x[6] for x in b],
                          [x[7] for x in b], [x[10] for x in b], [x[12] for x in b],
                          [f for x in b for f in x[13]], [i for x in b for i in x[14]],
                          list(begins), int(it0), int(nsteps))


def shear_fdtd_jax(bx, by, bz, rho, mu, dX, dY, dZ, dT, n_steps, opts=None, callback=None,
                   trace_indices=None, return_traces=False, return_device=False,
                   snapshot_stride=None):
    """``shear_fdtd_jax`` contract (solver.py:246-566) on the CUDA path.

    Same errors as the reference's JAX solver: no callback, no
    ``reproject_every``; device outputs are torch CUDA tensors.
    """
    ref = bx if bx is not None else (by if by is not None else bz)
    if ref is None:
        raise ValueError("At least one body-force component must be provided.")
    if callback is not None:
        raise ValueError("callback is not supported in shear_fdtd_jax.")
    _check_jax_kwargs(n_steps, trace_indices, return_traces, snapshot_stride)
    opts = dict(opts or {})
    if opts.get("reproject_every"):
        raise NotImplementedError(
            "reproject_every is only implemented in the NumPy solver (shear_fdtd)."
        )
    opts.pop("jit", None)
    return shear_fdtd(bx, by, bz, rho, mu, dX, dY, dZ, dT, n_steps, opts,
                      trace_indices=trace_indices, return_traces=return_traces,
                      return_device=return_device, snapshot_stride=snapshot_stride)
