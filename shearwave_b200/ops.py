"""The C ABI of libshearwave_b200.so as PyTorch operators (``torch.ops.shearwave_b200``).

Every entry point the host API computes with is registered here as a
``torch.library`` custom op: tensors own all device memory, the op reads
their device pointers, builds the C-ABI arguments and enqueues the CUDA
kernels on the current stream of the tensors' device.  The package's public
functions (``shear_fdtd``, ``project_vector_field``, the operators, strain
and radiation force) call these ops and nothing else, so torch sees every
call: each op declares which tensors it writes, has a fake (shape-only)
implementation for FakeTensor tracing and ``torch.compile``, and is
registered for CUDA only (a CPU tensor is refused by the dispatcher -- there
is no CPU path).

Conventions: an optional tensor argument of ``None`` is a NULL pointer;
``h`` is the grid spacing ``[dX, dY, dZ]``; padded fields hold components as
planes of ``nx * ny * pz`` elements with ``pz = sw_pitch(nz)``; ``stats``
tensors are host float64 ``[iters, reason, rel, max_div]`` per CG solve.
Ops that must read a device result (the CG loop, the projection) synchronise
their stream; every other op only enqueues work.

Reference functions behind the ops (pinton-lab/shearwave):
laplacian / divergence / gradient -- src/shearwave/solver.py:686-729;
project, project_batch -- solver.py:644-683, 1010-1050; static_solve --
solver.py:569-625; fdtd_* -- solver.py:27-243; strain_* --
src/shearwave/strain.py:16-135; arf_* -- src/shearwave/radiation_force.py:27-157.
"""

import ctypes as C
from typing import Optional, Sequence

import torch
from torch.library import custom_op

from . import _native

NS = "shearwave_b200"
Tensor = torch.Tensor

# iparams of the fdtd ops (one int list, so a schema stays short)
I_PREC, I_NX, I_NY, I_NZ, I_NSTEPS, I_KAHAN, I_SNAP, I_XCHUNK, I_SPP, I_KERNEL, I_ETA, \
    I_STALL = range(12)
# fparams of the fdtd ops
F_DX, F_DY, F_DZ, F_DT, F_DAMP = range(5)


def _stream(t: Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _p(t: Optional[Tensor]):
    return None if t is None else t.data_ptr()


def _code(dt: torch.dtype) -> int:
    if dt == torch.float32:
        return _native.SW_F32
    if dt == torch.float64:
        return _native.SW_F64
    raise TypeError(f"unsupported dtype {dt}")


def pitch(nz: int) -> int:
    """Padded z pitch of a padded field (sw_pitch): nz rounded up to 8."""
    return (int(nz) + 7) // 8 * 8


def _stats_tensor(st) -> Tensor:
    return torch.tensor([float(st.iters), float(st.reason), float(st.rel), float(st.max_div)],
                        dtype=torch.float64)


def _op(name, mutates=()):
    return custom_op(f"{NS}::{name}", mutates_args=tuple(mutates), device_types="cuda")


# ---------------------------------------------------------------------------
# collocated FD operators
# ---------------------------------------------------------------------------
@_op("laplacian")
def laplacian(f: Tensor, h: Sequence[float]) -> Tensor:
    """laplacian_center: interior 7-point Laplacian, zero shell."""
    out = torch.empty_like(f)
    nx, ny, nz = f.shape
    _native.call("sw_laplacian", _code(f.dtype), f.data_ptr(), out.data_ptr(), nx, ny, nz,
                 *h, _stream(f))
    return out


@laplacian.register_fake
def _(f, h):
    return torch.empty_like(f)


@_op("divergence")
def divergence(fx: Tensor, fy: Tensor, fz: Tensor, h: Sequence[float]) -> Tensor:
    """divergence_center: interior 2h central divergence, zero shell."""
    out = torch.empty_like(fx)
    nx, ny, nz = fx.shape
    _native.call("sw_divergence", _code(fx.dtype), fx.data_ptr(), fy.data_ptr(), fz.data_ptr(),
                 out.data_ptr(), nx, ny, nz, *h, _stream(fx))
    return out


@divergence.register_fake
def _(fx, fy, fz, h):
    return torch.empty_like(fx)


@_op("gradient")
def gradient(phi: Tensor, h: Sequence[float]) -> tuple[Tensor, Tensor, Tensor]:
    """gradient_center: interior 2h central gradient, zero shell."""
    g = [torch.empty_like(phi) for _ in range(3)]
    nx, ny, nz = phi.shape
    _native.call("sw_gradient", _code(phi.dtype), phi.data_ptr(), g[0].data_ptr(),
                 g[1].data_ptr(), g[2].data_ptr(), nx, ny, nz, *h, _stream(phi))
    return g[0], g[1], g[2]


@gradient.register_fake
def _(phi, h):
    return torch.empty_like(phi), torch.empty_like(phi), torch.empty_like(phi)


# ---------------------------------------------------------------------------
# projection, static solve, padded-field conversion
# ---------------------------------------------------------------------------
def _ref(*ts):
    for t in ts:
        if t is not None:
            return t
    raise ValueError("at least one component is required")


@_op("project")
def project(fx: Optional[Tensor], fy: Optional[Tensor], fz: Optional[Tensor],
            h: Sequence[float], tol: float, max_iters: int, method: str) -> tuple[Tensor, Tensor]:
    """Helmholtz-Hodge projection of dense (nx, ny, nz) components in FP64
    (``method`` "cg": the reference's CG and stopping rule; "spectral": the
    direct solve).  Returns the projected force as 3 padded FP64 components
    and the host stats.  Synchronises the stream."""
    ref = _ref(fx, fy, fz)
    lib = _native.load()
    nx, ny, nz = ref.shape
    code = _code(ref.dtype)
    st = _native.CGStats()
    out = torch.empty((3, nx * ny * pitch(nz)), dtype=torch.float64, device=ref.device)
    fs = (_p(fx), _p(fy), _p(fz))
    if method == "spectral":
        nb = int(lib.sw_project_spectral_workspace_bytes(nx, ny, nz))
        ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=ref.device)
        _native.call("sw_project_spectral", code, *fs, ny * nz, nz, 1, nx, ny, nz, *h,
                     out.data_ptr(), ws.data_ptr(), nb, C.byref(st), _stream(ref))
    elif method == "cg":
        nb = int(lib.sw_project_workspace_bytes(nx, ny, nz))
        ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=ref.device)
        _native.call("sw_project", code, *fs, ny * nz, nz, 1, nx, ny, nz, *h, float(tol),
                     int(max_iters), out.data_ptr(), ws.data_ptr(), nb, C.byref(st),
                     _stream(ref))
    else:
        raise ValueError(f"unknown projection method {method!r}")
    return out, _stats_tensor(st)


@project.register_fake
def _(fx, fy, fz, h, tol, max_iters, method):
    ref = _ref(fx, fy, fz)
    nx, ny, nz = ref.shape
    return (ref.new_empty((3, nx * ny * pitch(nz)), dtype=torch.float64),
            torch.empty(4, dtype=torch.float64))


@_op("project_batch")
def project_batch(fx: Sequence[Optional[Tensor]], fy: Sequence[Optional[Tensor]],
                  fz: Sequence[Optional[Tensor]], h: Sequence[float], tol: Sequence[float],
                  max_iters: Sequence[int]) -> tuple[list[Tensor], Tensor]:
    """Batched CG projection of n solves (same dtype): every CG launch advances
    every unfinished solve, each with its own stopping rule.  ``h`` holds 3
    spacings per solve.  Returns the padded FP64 outputs and (n, 4) stats."""
    lib = _native.load()
    n = len(fx)
    jobs = (_native.ProjectJob * n)()
    outs, keep = [], []
    for k in range(n):
        ref = _ref(fx[k], fy[k], fz[k])
        nx, ny, nz = ref.shape
        nb = int(lib.sw_project_workspace_bytes(nx, ny, nz))
        ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=ref.device)
        out = torch.empty((3, nx * ny * pitch(nz)), dtype=torch.float64, device=ref.device)
        j = jobs[k]
        j.in_dtype = _code(ref.dtype)
        j.fx, j.fy, j.fz = _p(fx[k]), _p(fy[k]), _p(fz[k])
        j.sx, j.sy, j.sz = ny * nz, nz, 1
        j.nx, j.ny, j.nz = nx, ny, nz
        j.dX, j.dY, j.dZ = h[3 * k], h[3 * k + 1], h[3 * k + 2]
        j.tol = float(tol[k])
        j.max_iters = int(max_iters[k])
        j.out = out.data_ptr()
        j.workspace = ws.data_ptr()
        j.workspace_bytes = nb
        outs.append(out)
        keep.append(ws)
    stats = (_native.CGStats * n)()
    if n:
        dev = outs[0].device
        tb = int(lib.sw_project_batch_table_bytes(n))
        table = torch.empty(tb, dtype=torch.uint8, device=dev)
        _native.call("sw_project_batch", jobs, n, table.data_ptr(), tb, stats, _stream(outs[0]))
    st = torch.stack([_stats_tensor(s) for s in stats]) if n else torch.empty((0, 4),
                                                                                dtype=torch.float64)
    return outs, st


@project_batch.register_fake
def _(fx, fy, fz, h, tol, max_iters):
    outs = []
    for k in range(len(fx)):
        ref = _ref(fx[k], fy[k], fz[k])
        nx, ny, nz = ref.shape
        outs.append(ref.new_empty((3, nx * ny * pitch(nz)), dtype=torch.float64))
    return outs, torch.empty((len(fx), 4), dtype=torch.float64)


@_op("convert_", mutates=("dst",))
def convert_(dst: Tensor, src: Tensor, ncomp: int, shape: Sequence[int],
             dst_strides: Sequence[int], scale: float, rho: Optional[Tensor],
             rho_strides: Sequence[int]) -> None:
    """dst = src * scale / rho (rho None: src * scale) from ``ncomp`` padded
    FP64 components into ``dst`` (element (x, y, z) of component c at
    c*cs + x*sx + y*sy + z*sz, ``dst_strides`` = [cs, sx, sy, sz])."""
    nx, ny, nz = shape
    rc = _code(rho.dtype) if rho is not None else _native.SW_F32
    _native.call("sw_convert", int(ncomp), src.data_ptr(), nx, ny, nz, _code(dst.dtype),
                 dst.data_ptr(), *dst_strides, float(scale), rc, _p(rho), *rho_strides,
                 _stream(dst))


@convert_.register_fake
def _(dst, src, ncomp, shape, dst_strides, scale, rho, rho_strides):
    return None


@_op("static_solve")
def static_solve(b: Tensor, mu: Optional[Tensor], mu_s: float, h: Sequence[float], tol: float,
                 max_iters: int) -> tuple[Tensor, Tensor]:
    """CG on (-mu L7) u = b (elastic_solve_static): u as one padded FP64 field
    and the host stats.  Synchronises the stream."""
    lib = _native.load()
    nx, ny, nz = b.shape
    nb = int(lib.sw_project_workspace_bytes(nx, ny, nz))
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=b.device)
    out = torch.empty((1, nx * ny * pitch(nz)), dtype=torch.float64, device=b.device)
    st = _native.CGStats()
    _native.call("sw_static_solve", _code(b.dtype), b.data_ptr(), _p(mu), float(mu_s), ny * nz,
                 nz, 1, nx, ny, nz, *h, float(tol), int(max_iters), out.data_ptr(),
                 ws.data_ptr(), nb, C.byref(st), _stream(b))
    return out, _stats_tensor(st)


@static_solve.register_fake
def _(b, mu, mu_s, h, tol, max_iters):
    nx, ny, nz = b.shape
    return (b.new_empty((1, nx * ny * pitch(nz)), dtype=torch.float64),
            torch.empty(4, dtype=torch.float64))


# ---------------------------------------------------------------------------
# strain post-pass
# ---------------------------------------------------------------------------
def _strain_outs(like: Tensor, shape, want_tensor: bool, want_invariants: bool = True):
    nx, ny, nz = shape
    eps = like.new_empty((nx, ny, nz, 6) if want_tensor else (0,))
    lead = (nx, ny, nz) if want_invariants else (0,)
    inv = [like.new_empty(lead) for _ in range(3)]
    vm = like.new_empty(lead, dtype=torch.float64)
    return eps, inv[0], inv[1], inv[2], vm


@_op("strain")
def strain(ux: Tensor, uy: Tensor, uz: Tensor, h: Sequence[float], want_tensor: bool,
           want_invariants: bool) -> tuple[Tensor, Tensor, Tensor, Tensor, Tensor]:
    """Voigt strain of dense components and / or its invariants in one pass:
    (eps, volumetric, deviatoric, max_shear, von_mises); an output that was
    not asked for is an empty tensor."""
    nx, ny, nz = ux.shape
    eps, vol, dev, ms, vm = _strain_outs(ux, (nx, ny, nz), want_tensor, want_invariants)
    inv = (vol, dev, ms, vm) if want_invariants else (None,) * 4
    _native.call("sw_strain", _code(ux.dtype), ux.data_ptr(), uy.data_ptr(), uz.data_ptr(),
                 ny * nz, nz, 1, nx, ny, nz, *h, eps.data_ptr() if want_tensor else None,
                 *(_p(t) for t in inv), _stream(ux))
    return eps, vol, dev, ms, vm


@strain.register_fake
def _(ux, uy, uz, h, want_tensor, want_invariants):
    return _strain_outs(ux, ux.shape, want_tensor, want_invariants)


@_op("strain_aos")
def strain_aos(u: Tensor, h: Sequence[float],
               want_tensor: bool) -> tuple[Tensor, Tensor, Tensor, Tensor, Tensor]:
    """The fused strain post-pass of a solver displacement u (nx, ny, nz, 3):
    (eps or an empty tensor, volumetric, deviatoric, max_shear, von_mises)."""
    nx, ny, nz, _ = u.shape
    eps, vol, dev, ms, vm = _strain_outs(u, (nx, ny, nz), want_tensor)
    base, es = u.data_ptr(), u.element_size()
    _native.call("sw_strain", _code(u.dtype), base, base + es, base + 2 * es, ny * nz * 3,
                 nz * 3, 3, nx, ny, nz, *h, eps.data_ptr() if want_tensor else None,
                 vol.data_ptr(), dev.data_ptr(), ms.data_ptr(), vm.data_ptr(), _stream(u))
    return eps, vol, dev, ms, vm


@strain_aos.register_fake
def _(u, h, want_tensor):
    return _strain_outs(u, u.shape[:3], want_tensor)


@_op("strain_invariants")
def strain_invariants(eps: Tensor) -> tuple[Tensor, Tensor, Tensor, Tensor]:
    """Invariants of Voigt 6-vectors (..., 6): volumetric, deviatoric,
    max_shear (eps dtype) and von_mises (float64)."""
    lead = tuple(eps.shape[:-1])
    n = 1
    for s in lead:
        n *= int(s)
    outs = [eps.new_empty(lead) for _ in range(3)] + [eps.new_empty(lead, dtype=torch.float64)]
    _native.call("sw_strain_invariants", _code(eps.dtype), eps.data_ptr(), n,
                 *(o.data_ptr() for o in outs), _stream(eps))
    return outs[0], outs[1], outs[2], outs[3]


@strain_invariants.register_fake
def _(eps):
    lead = tuple(eps.shape[:-1])
    return (eps.new_empty(lead), eps.new_empty(lead), eps.new_empty(lead),
            eps.new_empty(lead, dtype=torch.float64))


# ---------------------------------------------------------------------------
# radiation force
# ---------------------------------------------------------------------------
@_op("arf_envelope")
def arf_envelope(p: Tensor, ncell: int, nt: int) -> Tensor:
    """Auto-gate envelope: mean over cells of p^2 per time sample (FP64)."""
    nb = max(1, int(_native.load().sw_arf_workspace_bytes(ncell, nt)))
    ws = torch.empty(nb, dtype=torch.uint8, device=p.device)
    env = torch.empty(nt, dtype=torch.float64, device=p.device)
    _native.call("sw_arf_envelope", _code(p.dtype), p.data_ptr(), ncell, nt, env.data_ptr(),
                 ws.data_ptr(), nb, _stream(p))
    return env


@arf_envelope.register_fake
def _(p, ncell, nt):
    return p.new_empty((nt,), dtype=torch.float64)


@_op("arf_force")
def arf_force(p: Tensor, vx: Optional[Tensor], vy: Optional[Tensor], vz: Optional[Tensor],
              shape: Sequence[int], nt: int, gate: Tensor, c_map: Tensor, rho_map: Tensor,
              alpha_map: Tensor, map_stride: int, f0: float,
              out_dtype: torch.dtype) -> list[Tensor]:
    """Radiation force over the gated samples: one field (pressure form) or
    three (velocity form, when vx, vy, vz are given)."""
    nf = 3 if vx is not None else 1
    nx, ny, nz = shape
    outs = [p.new_empty((nx, ny, nz), dtype=out_dtype) for _ in range(nf)]
    o = [x.data_ptr() for x in outs] + [None] * (3 - nf)
    _native.call("sw_arf_force", _code(p.dtype), nf, p.data_ptr(), _p(vx), _p(vy), _p(vz),
                 nx * ny * nz, nt, gate.data_ptr(), int(gate.numel()), c_map.data_ptr(),
                 rho_map.data_ptr(), alpha_map.data_ptr(), map_stride, float(f0),
                 _code(out_dtype), *o, _stream(p))
    return outs


@arf_force.register_fake
def _(p, vx, vy, vz, shape, nt, gate, c_map, rho_map, alpha_map, map_stride, f0, out_dtype):
    nf = 3 if vx is not None else 1
    return [p.new_empty(tuple(shape), dtype=out_dtype) for _ in range(nf)]


# ---------------------------------------------------------------------------
# time loop
# ---------------------------------------------------------------------------
# A solve's device state is a bundle of tensors (see solver._Run.bundle):
#   state (3, ncomp, ncell), coef (2, ncell), inv_rho (ncell) or None,
#   patterns (K, 3, ncell), term_off / term_pat (int32) / term_scale (f64),
#   snaps / trace_cells / traces or None, flags (int32, 1), clock (int32, 1)
#   or None, queue (int32, 2) or None,
# plus fparams [dX, dY, dZ, dT, vel_damp] and iparams (I_* above).  The op
# builds the sw_fdtd_desc from them on every call.
def make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
              trace_cells, traces, flags, clock, queue, fparams, iparams) -> _native.FdtdDesc:
    d = _native.FdtdDesc()
    d.precision = int(iparams[I_PREC])
    d.nx, d.ny, d.nz = (int(iparams[k]) for k in (I_NX, I_NY, I_NZ))
    d.pz = pitch(d.nz)
    d.n_steps = int(iparams[I_NSTEPS])
    d.dX, d.dY, d.dZ, d.dT, d.vel_damp = (float(fparams[k]) for k in range(5))
    for i in range(3):
        d.state[i] = state[i].data_ptr()
    d.coef_m = coef[0].data_ptr()
    d.coef_e = coef[1].data_ptr() if iparams[I_ETA] else None
    d.inv_rho = _p(inv_rho)
    # an empty placeholder (before the projection) is no pattern at all
    d.patterns = patterns.data_ptr() if patterns.numel() else None
    d.n_patterns = int(patterns.shape[0]) if patterns.numel() else 0
    d.term_off = _p(term_off)
    d.term_pat = _p(term_pat)
    d.term_scale = _p(term_scale)
    d.kahan = int(iparams[I_KAHAN])
    d.snap_stride = int(iparams[I_SNAP]) if snaps is not None else 0
    d.snaps = _p(snaps)
    d.n_traces = int(trace_cells.numel() // 3) if (trace_cells is not None and
                                                  traces is not None) else 0
    d.trace_cells = _p(trace_cells) if d.n_traces else None
    d.traces = _p(traces) if d.n_traces else None
    d.flags = _p(flags)
    d.xchunk = int(iparams[I_XCHUNK])
    d.steps_per_pass = int(iparams[I_SPP])
    d.kernel = int(iparams[I_KERNEL])
    d.clock = _p(clock)
    d.queue = _p(queue)
    d.stall_test = int(iparams[I_STALL])
    return d


_BUNDLE = ("state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor, "
           "term_off: Tensor, term_pat: Tensor, term_scale: Tensor, snaps: Optional[Tensor], "
           "trace_cells: Optional[Tensor], traces: Optional[Tensor], flags: Tensor, "
           "clock: Optional[Tensor], queue: Optional[Tensor], fparams: Sequence[float], "
           "iparams: Sequence[int]")


@_op("fdtd_materials_", mutates=("coef", "inv_rho"))
def fdtd_materials_(state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor,
                    term_off: Tensor, term_pat: Tensor, term_scale: Tensor,
                    snaps: Optional[Tensor], trace_cells: Optional[Tensor],
                    traces: Optional[Tensor], flags: Tensor, clock: Optional[Tensor],
                    queue: Optional[Tensor], fparams: Sequence[float], iparams: Sequence[int],
                    rho: Optional[Tensor], rho_s: float, mu: Optional[Tensor], mu_s: float,
                    eta_mode: int, eta: Optional[Tensor], eta_s: float) -> None:
    """Material coefficients of the solve from rho, mu, eta (dense or scalar)."""
    d = make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
                  trace_cells, traces, flags, clock, queue, fparams, iparams)
    ref = next((t for t in (rho, mu, eta) if t is not None), coef)
    in_code = _code(ref.dtype) if ref is not coef else _code(coef.dtype)
    _native.call("sw_fdtd_materials", C.byref(d), in_code, _p(rho), float(rho_s), _p(mu),
                 float(mu_s), int(eta_mode), _p(eta), float(eta_s), _stream(coef))


@_op("fdtd_init_", mutates=("state",))
def fdtd_init_(state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor,
               term_off: Tensor, term_pat: Tensor, term_scale: Tensor, snaps: Optional[Tensor],
               trace_cells: Optional[Tensor], traces: Optional[Tensor], flags: Tensor,
               clock: Optional[Tensor], queue: Optional[Tensor], fparams: Sequence[float],
               iparams: Sequence[int], init_u: Optional[Tensor],
               init_v: Optional[Tensor]) -> None:
    """Initial state from initial_u / initial_v (solver.py:157-171)."""
    d = make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
                  trace_cells, traces, flags, clock, queue, fparams, iparams)
    _native.call("sw_fdtd_init", C.byref(d), _p(init_u), _p(init_v), _stream(state))


@_op("fdtd_steps_", mutates=("state", "snaps", "traces", "flags", "clock", "queue"))
def fdtd_steps_(state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor,
                term_off: Tensor, term_pat: Tensor, term_scale: Tensor,
                snaps: Optional[Tensor], trace_cells: Optional[Tensor],
                traces: Optional[Tensor], flags: Tensor, clock: Optional[Tensor],
                queue: Optional[Tensor], fparams: Sequence[float], iparams: Sequence[int],
                it0: int, nsteps: int) -> None:
    """Advance steps it0 .. it0+nsteps-1 of the solve (solver.py:194-234)."""
    d = make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
                  trace_cells, traces, flags, clock, queue, fparams, iparams)
    _native.call("sw_fdtd_steps", C.byref(d), int(it0), int(nsteps), _stream(state))


@_op("fdtd_finish", mutates=("flags",))
def fdtd_finish(state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor,
                term_off: Tensor, term_pat: Tensor, term_scale: Tensor,
                snaps: Optional[Tensor], trace_cells: Optional[Tensor],
                traces: Optional[Tensor], flags: Tensor, clock: Optional[Tensor],
                queue: Optional[Tensor], fparams: Sequence[float], iparams: Sequence[int],
                steps_done: int, want_v: bool) -> tuple[Tensor, Tensor]:
    """u and (if ``want_v``) v = (u_curr - u_prev) / dT after ``steps_done``
    steps as dense (nx, ny, nz, 3) arrays (solver.py:241-243); v is an empty
    tensor otherwise.  Sets the non-finite bit of ``flags`` when a value of
    u or v is not finite."""
    d = make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
                  trace_cells, traces, flags, clock, queue, fparams, iparams)
    shp = (d.nx, d.ny, d.nz, 3)
    u = state.new_empty(shp)
    v = state.new_empty(shp if want_v else (0,))
    _native.call("sw_fdtd_finish", C.byref(d), int(steps_done), u.data_ptr(),
                 v.data_ptr() if want_v else None, _stream(state))
    return u, v


@fdtd_finish.register_fake
def _(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps, trace_cells,
      traces, flags, clock, queue, fparams, iparams, steps_done, want_v):
    shp = (int(iparams[I_NX]), int(iparams[I_NY]), int(iparams[I_NZ]), 3)
    return state.new_empty(shp), state.new_empty(shp if want_v else (0,))


@_op("fdtd_reproject_", mutates=("state",))
def fdtd_reproject_(state: Tensor, coef: Tensor, inv_rho: Optional[Tensor], patterns: Tensor,
                    term_off: Tensor, term_pat: Tensor, term_scale: Tensor,
                    snaps: Optional[Tensor], trace_cells: Optional[Tensor],
                    traces: Optional[Tensor], flags: Tensor, clock: Optional[Tensor],
                    queue: Optional[Tensor], fparams: Sequence[float], iparams: Sequence[int],
                    steps_done: int, tol: float, max_iters: int) -> Tensor:
    """reproject_every (solver.py:236-239): project u_curr and u_prev in place.
    Returns the (2, 4) host stats.  Synchronises the stream."""
    d = make_desc(state, coef, inv_rho, patterns, term_off, term_pat, term_scale, snaps,
                  trace_cells, traces, flags, clock, queue, fparams, iparams)
    lib = _native.load()
    nb = int(lib.sw_project_workspace_bytes(d.nx, d.ny, d.nz))
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=state.device)
    tmp = torch.empty((3, d.nx * d.ny * d.pz), dtype=torch.float64, device=state.device)
    st = (_native.CGStats * 2)()
    _native.call("sw_fdtd_reproject", C.byref(d), int(steps_done), float(tol), int(max_iters),
                 tmp.data_ptr(), ws.data_ptr(), nb, st, _stream(state))
    return torch.stack([_stats_tensor(st[0]), _stats_tensor(st[1])])


@fdtd_reproject_.register_fake
def _(*args):
    return torch.empty((2, 4), dtype=torch.float64)


@_op("fdtd_batch_steps_", mutates=("state", "flags", "queue"))
def fdtd_batch_steps_(state: Sequence[Tensor], coef: Sequence[Tensor],
                      inv_rho: Sequence[Optional[Tensor]],
                      patterns: Sequence[Tensor], term_off: Sequence[Tensor],
                      term_pat: Sequence[Tensor], term_scale: Sequence[Tensor],
                      snaps: Sequence[Optional[Tensor]], flags: Sequence[Tensor],
                      queue: Sequence[Optional[Tensor]], fparams: Sequence[float],
                      iparams: Sequence[int], begins: Sequence[int], it0: int,
                      nsteps: int) -> None:
    """Advance a batch of independent solves together (sw_fdtd_batch_steps):
    solve i runs its local step it - begins[i] at global step it while that
    lies in [0, n_steps).  ``fparams`` / ``iparams`` hold 5 / 12 values per
    solve; an empty ``begins`` starts every solve at step 0.  One launch per
    step or pair of steps covers every running solve."""
    n = len(state)
    descs = (_native.FdtdDesc * n)()
    nf, ni = len(fparams) // n, len(iparams) // n
    for k in range(n):
        descs[k] = make_desc(state[k], coef[k], inv_rho[k], patterns[k], term_off[k], term_pat[k],
                             term_scale[k], snaps[k], None, None, flags[k], None, queue[k],
                             fparams[nf * k: nf * (k + 1)], iparams[ni * k: ni * (k + 1)])
    beg = (C.c_int32 * n)(*[int(b) for b in begins]) if len(begins) else None
    lib = _native.load()
    tb = int(lib.sw_fdtd_batch_table_bytes(n))
    table = torch.empty(tb + 64, dtype=torch.uint8, device=state[0].device)
    base = (table.data_ptr() + 63) // 64 * 64
    # (the table's memory goes back to torch's cache for this stream; a later
    # allocation that reuses it is ordered after these launches)
    _native.call("sw_fdtd_batch_steps", descs, beg, n, int(it0), int(nsteps), base, tb,
                 _stream(state[0]))


for _mut in (fdtd_materials_, fdtd_init_, fdtd_steps_, fdtd_batch_steps_):
    _mut.register_fake(lambda *args, **kwargs: None)
