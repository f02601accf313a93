"""CPU oracle for the shear_fdtd hot path.  TEST INFRASTRUCTURE ONLY.

This module restates, in plain NumPy, the algorithm of pinton-lab/shearwave's
NumPy backend for the path that the CUDA library accelerates:

* the collocated FD operators       (src/shearwave/solver.py:686-729)
* the FP64 conjugate-gradient solve (src/shearwave/solver.py:1010-1050)
* the Helmholtz-Hodge projection    (src/shearwave/solver.py:644-683)
* the explicit time loop            (src/shearwave/solver.py:27-243)
* the static elastic CG solve       (src/shearwave/solver.py:569-625)
* the strain post-pass              (src/shearwave/strain.py:16-159)
* the radiation-force producers     (src/shearwave/radiation_force.py:27-157)

It is the CHECKER, never the product: only the test suite, the smoke check and
the CPU-baseline leg of the benchmark may import it.  The product path lives in
``shearwave_b200`` and runs CUDA kernels only.

Precision
---------
Every function takes ``dtype``.  ``np.float32`` reproduces the reference as it
ships (fields cast to float32, CG in float64).  ``np.float64`` is the FP64
oracle: the same arithmetic with every float32 cast widened to float64, which
is what the reference computes when its module-level ``np.float32`` is swapped
for ``np.float64``.  The elementwise operations are issued in the same order
and with the same operands as the reference, so a float32 run here matches the
shipped reference bit for bit and a float64 run matches the widened reference
bit for bit (pinned by tests/test_oracle_golden.py against fixtures that
tests/golden/make_golden.py produced by running the reference itself).
"""

from __future__ import annotations

import numpy as np

__all__ = [
    "compute_radiation_force",
    "compute_radiation_force_velocity",
    "compute_strain_invariants",
    "compute_strain_tensor",
    "divergence_center",
    "elastic_solve_static",
    "gradient_center",
    "laplacian_center",
    "poisson_cg",
    "project_vector_field",
    "shear_fdtd",
    "shell_mask",
]

_AXES = (0, 1, 2)


def _nbr(a: np.ndarray, axis: int, off: int) -> np.ndarray:
    """Interior-shaped view of ``a`` shifted by ``off`` cells along ``axis``."""
    sl = []
    for d in _AXES:
        n = a.shape[d]
        o = off if d == axis else 0
        sl.append(slice(1 + o, n - 1 + o))
    return a[tuple(sl)]


_INNER = (slice(1, -1),) * 3


def shell_mask(shape, dtype=np.float32) -> np.ndarray:
    """1 on interior cells, 0 on the one-voxel zero-Dirichlet shell.

    solver.py:152-153 / 664-665.
    """
    m = np.zeros(tuple(shape)[:3], dtype=dtype)
    m[_INNER] = 1.0
    return m


# ---------------------------------------------------------------------------
# FD operators (solver.py:686-729)
# ---------------------------------------------------------------------------
def laplacian_center(f: np.ndarray, dX: float, dY: float, dZ: float) -> np.ndarray:
    """Compact 7-point Laplacian on interior cells, zero on the shell.

    Per axis ``((f[i+1] - 2 f[i]) + f[i-1]) / h**2``; axes summed x, y, z in
    order (solver.py:686-695).
    """
    out = np.zeros_like(f, dtype=f.dtype)
    c = f[_INNER]
    acc = None
    for ax, h in zip(_AXES, (dX, dY, dZ)):
        term = (_nbr(f, ax, 1) - 2.0 * c + _nbr(f, ax, -1)) / (h**2)
        acc = term if acc is None else acc + term
    out[_INNER] = acc
    return out


def divergence_center(fx, fy, fz, dX, dY, dZ) -> np.ndarray:
    """2h central divergence on interior cells, zero on the shell (solver.py:708-717)."""
    dtype = np.result_type(fx.dtype, fy.dtype, fz.dtype)
    out = np.zeros_like(fx, dtype=dtype)
    acc = None
    for ax, comp, h in zip(_AXES, (fx, fy, fz), (dX, dY, dZ)):
        term = (_nbr(comp, ax, 1) - _nbr(comp, ax, -1)) / (2.0 * h)
        acc = term if acc is None else acc + term
    out[_INNER] = acc
    return out


def gradient_center(phi, dX, dY, dZ):
    """2h central gradient on interior cells, zero on the shell (solver.py:720-729)."""
    outs = []
    for ax, h in zip(_AXES, (dX, dY, dZ)):
        g = np.zeros_like(phi, dtype=phi.dtype)
        g[_INNER] = (_nbr(phi, ax, 1) - _nbr(phi, ax, -1)) / (2.0 * h)
        outs.append(g)
    return tuple(outs)


# ---------------------------------------------------------------------------
# Poisson CG and projection (solver.py:1010-1050, 644-683)
# ---------------------------------------------------------------------------
class CGStats:
    """Iteration count and exit reason of one oracle CG solve."""

    __slots__ = ("iters", "reason", "rel")

    def __init__(self):
        self.iters = 0
        self.reason = "max_iters"
        self.rel = float("nan")

    def __repr__(self):
        return f"CGStats(iters={self.iters}, reason={self.reason!r}, rel={self.rel:.3e})"


def poisson_cg(rhs, dX, dY, dZ, mask_center, tol=1e-4, max_iters=200, stats=None):
    """CG on ``A x = rhs`` with ``A = -div_c(grad_c(.))`` in float64.

    Stopping rule of solver.py:1033-1048: break when ``p.Ap`` is non-finite
    or <= 0 (x untouched that iteration), when ``r.r`` is non-finite (after x
    was updated), or when ``sqrt(rs_new / rs0) < tol`` with
    ``rs0 = max(r0.r0, eps64)``.  ``stats`` (a :class:`CGStats`) receives the
    number of completed x updates and the exit reason.  Returns x cast to
    ``rhs.dtype``.
    """
    eps = np.finfo(np.float64).eps
    b = rhs.astype(np.float64, copy=False)
    m = mask_center.astype(np.float64, copy=False)
    x = np.zeros_like(b)

    def apply_a(v):
        g = gradient_center(v, dX, dY, dZ)
        return -divergence_center(g[0], g[1], g[2], dX, dY, dZ)

    r = (b - apply_a(x)) * m
    p = r.copy()
    rr = np.sum(r * r)
    rr0 = max(rr, eps)
    st = stats if stats is not None else CGStats()
    st.iters, st.reason = 0, "max_iters"
    for _ in range(max_iters):
        ap = apply_a(p) * m
        pap = np.sum(p * ap)
        if not np.isfinite(pap) or pap <= 0.0:
            st.reason = "breakdown"
            break
        alpha = rr / pap
        x = (x + alpha * p) * m
        r = (r - alpha * ap) * m
        st.iters += 1
        rr_new = np.sum(r * r)
        if not np.isfinite(rr_new):
            st.reason = "nonfinite"
            break
        st.rel = float(np.sqrt(rr_new / rr0))
        if np.sqrt(rr_new / rr0) < tol:
            st.reason = "converged"
            break
        beta = rr_new / max(rr, eps)
        p = (r + beta * p) * m
        rr = rr_new
    return x.astype(rhs.dtype, copy=False)


def project_vector_field(fx, fy, fz, dX, dY, dZ, tol, max_iters, dtype=np.float32, stats=None):
    """Helmholtz-Hodge projection onto discretely divergence-free fields.

    solver.py:644-683: mask first, take div_c, early exit when
    ``max|div| < 1e-12`` (returns the masked input), else solve
    ``A phi = -div`` by :func:`poisson_cg` and return ``(f - grad_c phi) * mask``.
    """
    m = shell_mask(fx.shape, dtype)
    fx = fx.astype(dtype, copy=False) * m
    fy = fy.astype(dtype, copy=False) * m
    fz = fz.astype(dtype, copy=False) * m
    div = divergence_center(fx, fy, fz, dX, dY, dZ)
    div *= m
    if np.max(np.abs(div)) < 1e-12:
        if stats is not None:
            stats.iters, stats.reason = 0, "early_exit"
        fx *= m
        fy *= m
        fz *= m
        return fx, fy, fz
    phi = poisson_cg(-div, dX, dY, dZ, m, tol=tol, max_iters=max_iters, stats=stats)
    g = gradient_center(phi, dX, dY, dZ)
    return (fx - g[0]) * m, (fy - g[1]) * m, (fz - g[2]) * m


# ---------------------------------------------------------------------------
# Time loop (solver.py:27-243, 1060-1079)
# ---------------------------------------------------------------------------
def _material(v, shape, dtype):
    """Scalar -> full field, array -> cast + shape check (solver.py:1072-1079)."""
    if np.isscalar(v):
        return np.full(shape, float(v), dtype=dtype)
    a = np.asarray(v, dtype=dtype)
    if a.shape != shape:
        raise ValueError("Material field has incompatible shape.")
    return a


def _body4d(v, shape, n_steps, dtype):
    """3-D -> repeated 4-D force, None -> zeros (solver.py:1060-1069)."""
    if v is None:
        return np.zeros((*shape, n_steps), dtype=dtype)
    a = np.asarray(v, dtype=dtype)
    if a.ndim == 3:
        a = np.repeat(a[..., np.newaxis], n_steps, axis=3)
    if a.ndim != 4 or a.shape != (*shape, n_steps):
        raise ValueError("Body-force component has incompatible shape.")
    return a


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
    dtype=np.float32,
    snapshot_stride=None,
    force_terms=None,
    cg_stats=None,
):
    """Oracle time loop of solver.py:27-243.

    ``dtype`` selects float32 (reference as shipped) or float64 (FP64 oracle).
    ``snapshot_stride=k`` additionally returns ``u`` after every k steps, which
    is what solver.py:469-507 returns and what the reference tests collect
    through the callback (tests/test_snapshot_stride.py:55-70).
    ``force_terms`` (list of ``((bx, by, bz), env)``) adds further separable
    force terms; by linearity of the projection and of the scheme this equals
    the sum of one reference run per term.
    ``cg_stats`` (list) receives one :class:`CGStats` per projection.
    """
    ref = bx if bx is not None else (by if by is not None else bz)
    if ref is None:
        raise ValueError("At least one body-force component must be provided.")
    opts = opts or {}
    vel_damp = opts.get("vel_damp", 0.0)
    tol = opts.get("poisson_tol", 1e-5)
    max_iters = opts.get("poisson_max_iters", 200)
    reproject_every = int(opts.get("reproject_every", 0) or 0)
    if reproject_every < 0:
        raise ValueError("reproject_every must be a non-negative integer.")
    nx, ny, nz = ref.shape[:3]
    shape = (nx, ny, nz)

    def project(fx, fy, fz):
        st = CGStats()
        out = project_vector_field(
            fx.astype(dtype, copy=True),
            fy.astype(dtype, copy=True),
            fz.astype(dtype, copy=True),
            dX, dY, dZ, tol, max_iters, dtype=dtype, stats=st,
        )
        if cg_stats is not None:
            cg_stats.append(st)
        return out

    env_t = opts.get("env_t")
    terms = []  # (projected pattern triple, envelope) for separable mode
    if env_t is not None:
        env_t = np.asarray(env_t, dtype=dtype).ravel()
        if env_t.shape[0] != n_steps:
            raise ValueError(
                f"env_t length ({env_t.shape[0]}) must equal n_steps ({n_steps})."
            )
        zero = np.zeros(shape, dtype=dtype)
        pat = tuple(zero if b is None else np.asarray(b, dtype=dtype) for b in (bx, by, bz))
        separable = True
    else:
        b4 = tuple(_body4d(b, shape, n_steps, dtype) for b in (bx, by, bz))
        separable = False

    rho_f = _material(rho, shape, dtype)
    mu_f = _material(mu, shape, dtype)
    m_over = mu_f / rho_f
    inv_rho = 1.0 / rho_f
    eta = opts.get("eta", 0.0)
    if np.isscalar(eta):
        eta = _material(float(eta), shape, dtype) if float(eta) != 0.0 else None
    elif eta is not None:
        eta = _material(eta, shape, dtype)
    e_over = None if eta is None else eta / rho_f

    u_prev = np.zeros((*shape, 3), dtype=dtype)
    u_curr = np.zeros_like(u_prev)
    u_next = np.zeros_like(u_prev)
    mask = shell_mask(shape, dtype)
    mask4 = mask[..., None]
    dt2 = dT * dT

    init_u = opts.get("initial_u")
    init_v = opts.get("initial_v")
    if init_u is not None:
        init_u = np.asarray(init_u, dtype=dtype)
        if init_u.shape != u_curr.shape:
            raise ValueError("initial_u must match shape (nx,ny,nz,3)")
        u_curr = init_u * mask4
    if init_v is not None:
        init_v = np.asarray(init_v, dtype=dtype)
        if init_v.shape != u_curr.shape:
            raise ValueError("initial_v must match shape (nx,ny,nz,3)")
        u_prev = u_curr - dT * init_v
        u_prev *= mask4

    if separable:
        terms.append((project(*pat), env_t))
    for (tb, tenv) in force_terms or ():
        tenv = np.asarray(tenv, dtype=dtype).ravel()
        tp = tuple(np.zeros(shape, dtype) if b is None else np.asarray(b, dtype) for b in tb)
        terms.append((project(*tp), tenv))

    snaps = [] if snapshot_stride else None
    for it in range(n_steps):
        if separable or terms:
            f = None
            for (pf, env) in terms:
                s = env[it]
                contrib = [pf[c] * s for c in range(3)]
                f = contrib if f is None else [f[c] + contrib[c] for c in range(3)]
            if not separable:
                extra = project(b4[0][..., it], b4[1][..., it], b4[2][..., it])
                f = [extra[c] + f[c] for c in range(3)]
        else:
            f = list(project(b4[0][..., it], b4[1][..., it], b4[2][..., it]))

        acc = [m_over * laplacian_center(u_curr[..., c], dX, dY, dZ) + f[c] * inv_rho
               for c in range(3)]
        if e_over is not None:
            vel = (u_curr - u_prev) / dT
            vel *= mask4
            for c in range(3):
                acc[c] += e_over * laplacian_center(vel[..., c], dX, dY, dZ)
        for c in range(3):
            u_next[..., c] = 2.0 * u_curr[..., c] - u_prev[..., c] + dt2 * acc[c]
        if vel_damp > 0.0:
            u_next = u_curr + (1.0 - vel_damp) * (u_next - u_curr)
        u_next *= mask4
        if callback is not None:
            callback(it, u_next)
        if snaps is not None and (it + 1) % snapshot_stride == 0:
            snaps.append(u_next.copy())
        u_prev, u_curr = u_curr, u_next.copy()
        if reproject_every and (it + 1) % reproject_every == 0:
            for arr in (u_curr, u_prev):
                q = project(arr[..., 0], arr[..., 1], arr[..., 2])
                arr[..., 0], arr[..., 1], arr[..., 2] = q
    u = u_curr.copy()
    v = (u_curr - u_prev) / dT
    if snaps is not None:
        return u, v, (np.stack(snaps) if snaps else np.zeros((0, *u.shape), dtype))
    return u, v


# ---------------------------------------------------------------------------
# Static elastic solve (solver.py:569-625)
# ---------------------------------------------------------------------------
def elastic_solve_static(bz, dX, dY, dZ, mu, tol=1e-6, max_iters=1500, dtype=np.float32,
                         stats=None):
    """CG on ``(-mu L7) u = bz`` in ``dtype`` (solver.py:569-625).

    The residual floor is ``finfo(dtype).eps``: the reference writes
    ``np.finfo(np.float32).eps``, which the FP64 widening turns into the
    float64 epsilon.
    """
    shape = bz.shape
    mu_f = _material(mu, shape, dtype)
    b = bz.astype(dtype)
    u = np.zeros_like(b, dtype=dtype)
    m = shell_mask(shape, dtype)
    eps32 = np.finfo(dtype).eps

    def apply_a(v):
        return -mu_f * laplacian_center(v, dX, dY, dZ)

    r = b - apply_a(u)
    r *= m
    p = r.copy()
    rr = np.sum(r * r)
    rr0 = max(rr, eps32)
    st = stats if stats is not None else CGStats()
    st.iters, st.reason = 0, "max_iters"
    for _ in range(max_iters):
        ap = apply_a(p)
        pap = np.sum(p * ap)
        if pap <= 0.0:
            st.reason = "breakdown"
            break
        alpha = rr / pap
        u = (u + alpha * p) * m
        r = (r - alpha * ap) * m
        st.iters += 1
        rr_new = np.sum(r * r)
        rel = np.sqrt(rr_new / rr0)
        st.rel = float(rel)
        if rel < tol:
            st.reason = "converged"
            break
        beta = rr_new / max(rr, eps32)
        p = (r + beta * p) * m
        rr = rr_new
    return u


# ---------------------------------------------------------------------------
# Strain post-pass (strain.py:16-159)
# ---------------------------------------------------------------------------
def compute_strain_tensor(ux, uy, uz, dX, dY, dZ) -> np.ndarray:
    """Voigt strain ``[exx, eyy, ezz, gyz, gxz, gxy]`` with engineering shear.

    strain.py:16-70, input checks strain.py:138-159.
    """
    if ux.ndim != 3:
        raise ValueError(f"Displacement arrays must be 3-D, got ndim={ux.ndim}")
    if ux.shape != uy.shape or ux.shape != uz.shape:
        raise ValueError(
            "All displacement components must share the same shape: "
            f"ux={ux.shape}, uy={uy.shape}, uz={uz.shape}"
        )
    for name, h in (("dX", dX), ("dY", dY), ("dZ", dZ)):
        if h <= 0:
            raise ValueError(f"Grid spacing {name} must be positive, got {h}")
    dtype = np.result_type(ux.dtype, uy.dtype, uz.dtype)
    eps = np.zeros((*ux.shape, 6), dtype=dtype)
    gx = gradient_center(ux, dX, dY, dZ)
    gy = gradient_center(uy, dX, dY, dZ)
    gz = gradient_center(uz, dX, dY, dZ)
    eps[..., 0] = gx[0]
    eps[..., 1] = gy[1]
    eps[..., 2] = gz[2]
    eps[..., 3] = gy[2] + gz[1]
    eps[..., 4] = gx[2] + gz[0]
    eps[..., 5] = gx[1] + gy[0]
    return eps


def compute_strain_invariants(eps: np.ndarray) -> dict:
    """Volumetric, deviatoric norm, max shear and von Mises (strain.py:73-135)."""
    if eps.shape[-1] != 6:
        raise ValueError(
            f"Expected last dimension == 6 (Voigt notation), got {eps.shape[-1]}"
        )
    exx, eyy, ezz, gyz, gxz, gxy = (eps[..., k] for k in range(6))
    vol = (exx + eyy + ezz) / 3.0
    dxx, dyy, dzz = exx - vol, eyy - vol, ezz - vol
    shear2 = 0.5 * (gyz**2 + gxz**2 + gxy**2)
    dev = np.sqrt(dxx**2 + dyy**2 + dzz**2 + shear2)
    j2 = 0.5 * (dxx**2 + dyy**2 + dzz**2 + 0.5 * (gyz**2 + gxz**2 + gxy**2))
    return {
        "volumetric": vol,
        "deviatoric": dev,
        "max_shear": np.sqrt(np.maximum(j2, 0.0)),
        "von_mises": np.sqrt(2.0 / 3.0) * dev,
    }


# ---------------------------------------------------------------------------
# acoustic radiation force (src/shearwave/radiation_force.py)
# ---------------------------------------------------------------------------
def _arf_gate(p):
    """Auto gate (radiation_force.py:63-68): t where mean_cells p^2 >= 0.1 max."""
    env = (p**2).mean(axis=(0, 1, 2))
    keep = env >= 0.1 * env.max()
    return slice(None) if not keep.any() else np.nonzero(keep)[0]


def _alpha_np(alpha_coeff_map, f0):
    """dB/cm/MHz -> Np/m (radiation_force.py:78-80)."""
    return (alpha_coeff_map * (f0 / 1e6)) / 8.685889638 * 100.0


def compute_radiation_force(pressure_4d, c_map, rho_map, alpha_coeff_map, f0, gate=None):
    """b = 2 alpha_Np Isppa / c, Isppa = mean_gate(p^2) / (rho c)
    (radiation_force.py:27-85)."""
    if gate is None:
        gate = _arf_gate(pressure_4d)
    isppa = np.mean(pressure_4d[:, :, :, gate] ** 2, axis=3) / (rho_map * c_map)
    return 2.0 * _alpha_np(alpha_coeff_map, f0) * isppa / c_map


def compute_radiation_force_velocity(pressure_4d, velocity_u_4d, velocity_w_4d, velocity_v_4d,
                                     c_map, rho_map, alpha_coeff_map, f0, gate=None):
    """b_i = (2 alpha_Np / c) mean_gate(p v_i) (radiation_force.py:88-157)."""
    if gate is None:
        gate = _arf_gate(pressure_4d)
    pg = pressure_4d[:, :, :, gate]
    flux = [np.mean(pg * v[:, :, :, gate], axis=3)
            for v in (velocity_u_4d, velocity_w_4d, velocity_v_4d)]
    coeff = 2.0 * _alpha_np(alpha_coeff_map, f0) / c_map
    return coeff * flux[0], coeff * flux[1], coeff * flux[2]
