// The shear_fdtd time loop: materials, initial state, the fused step kernels,
// the outputs and the in-loop re-projection.
//
// Reference: shear_fdtd (src/shearwave/solver.py:27-243).  Per interior cell
// and component the reference computes
//     a     = (mu/rho) L7(u_c) + f/rho + (eta/rho) L7((u_c - u_p)/dT)
//     u_n   = 2 u_c - u_p + dT^2 a
//     u_n   = u_c + (1 - vel_damp)(u_n - u_c)        (vel_damp > 0)
// with L7 the compact 7-point Laplacian and everything zero on the shell.
// The three components are independent; one kernel updates all three so the
// material coefficients are read once.
//
// Two forms:
//  * plain FP64 (SW_PLAIN_F64): state u_prev / u_curr / u_next in three
//    rotating FP64 buffers, the reference's arithmetic in FP64.
//  * mixed FP32 (SW_MIXED_F32): state (u, d = u_c - u_p, c) in FP32, three
//    rotating buffers (the state after t steps in buffer t mod 3, so a kernel
//    that fuses two steps never writes the buffer it reads), with
//    d_n = (1 - vd) (d + m' L7(u) + e' L7(d) + sum_j s_j P_j),
//    m' = dT^2 mu/rho, e' = dT eta/rho, P_j = dT^2 f_S/rho, and the
//    displacement accumulated as u_n = u + d_n with Kahan compensation c.
//    Storing the increment instead of u_prev removes the cancellation in
//    u_c - u_p, and the compensated sum keeps u's rounding from building up
//    over thousands of steps.
#include <math.h>

#include <algorithm>

#include "sw_common.cuh"
#include "sw_project.cuh"
#include "sw_step.cuh"
#include "sw_step_tma.cuh"

namespace sw {

// ---------------------------------------------------------------------------
// descriptor translation
// ---------------------------------------------------------------------------
int make_step_args(const sw_fdtd_desc* d, StepArgs* a) {
  if (d == nullptr) {
    set_error("null descriptor");
    return SW_EINVAL;
  }
  if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0 || d->pz != pad_pitch(d->nz)) {
    set_error("descriptor: bad grid (%d, %d, %d) pitch %d (expected %d)", d->nx, d->ny, d->nz,
              d->pz, pad_pitch(d->nz));
    return SW_EINVAL;
  }
  if (d->precision != SW_PLAIN_F64 && d->precision != SW_MIXED_F32) {
    set_error("descriptor: unknown precision %d", d->precision);
    return SW_EINVAL;
  }
  if (!(d->dX > 0 && d->dY > 0 && d->dZ > 0 && d->dT > 0)) {
    set_error("descriptor: spacings and dT must be positive");
    return SW_EINVAL;
  }
  *a = StepArgs{};
  a->g = make_geom(d->nx, d->ny, d->nz, d->pz);
  int xc = d->xchunk > 0 ? d->xchunk : choose_xchunk(a->g, 8 * 148);
  a->ts = make_tiles(a->g, xc);
  a->precision = d->precision;
  for (int i = 0; i < 3; ++i) a->state[i] = d->state[i];
  a->coef_m = d->coef_m;
  a->coef_e = d->coef_e;
  a->inv_rho = d->inv_rho;
  a->patterns = d->patterns;
  a->term_off = d->term_off;
  a->term_pat = d->term_pat;
  a->term_scale = d->term_scale;
  a->ihx2 = 1.0 / (d->dX * d->dX);
  a->ihy2 = 1.0 / (d->dY * d->dY);
  a->ihz2 = 1.0 / (d->dZ * d->dZ);
  a->dT = d->dT;
  a->inv_dt = 1.0 / d->dT;
  a->dt2 = d->dT * d->dT;
  a->use_damp = d->vel_damp > 0.0 ? 1 : 0;
  a->damp = 1.0 - d->vel_damp;
  a->kahan = d->kahan;
  a->n_steps = d->n_steps;
  a->snap_stride = d->snap_stride;
  a->snaps = d->snaps;
  a->n_traces = d->n_traces;
  a->trace_cells = d->trace_cells;
  a->traces = d->traces;
  a->flags = d->flags;
  a->kernel = d->kernel;
  a->xchunk = d->xchunk;
  a->steps_per_pass = d->steps_per_pass;
  a->clock = d->clock;
  a->queue = d->queue;
  a->stall_test = d->stall_test;
  const int nbuf = 3;
  for (int i = 0; i < nbuf; ++i)
    if (a->state[i] == nullptr) {
      set_error("descriptor: state[%d] is null", i);
      return SW_EINVAL;
    }
  if (a->coef_m == nullptr || (d->precision == SW_PLAIN_F64 && a->inv_rho == nullptr)) {
    set_error("descriptor: material coefficients missing");
    return SW_EINVAL;
  }
  if (d->n_patterns > 0 && (a->patterns == nullptr || a->term_off == nullptr ||
                            a->term_pat == nullptr || a->term_scale == nullptr)) {
    set_error("descriptor: force terms missing");
    return SW_EINVAL;
  }
  return SW_OK;
}

// ---------------------------------------------------------------------------
// materials
// ---------------------------------------------------------------------------
template <typename Tin>
__global__ void materials_kernel(StepArgs a, const Tin* __restrict__ rho, double rho_s,
                                 const Tin* __restrict__ mu, double mu_s, int eta_mode,
                                 const Tin* __restrict__ eta, double eta_s) {
  const Geom g = a.g;
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(q % g.nz);
    const long long xy = q / g.nz;
    const long long i = xy * g.pz + z;  // x*ny*pz + y*pz + z
    const double r = rho ? (double)rho[q] : rho_s;
    const double m = mu ? (double)mu[q] : mu_s;
    const double e = eta_mode ? (eta ? (double)eta[q] : eta_s) : 0.0;
    if (a.precision == SW_PLAIN_F64) {
      ((double*)a.coef_m)[i] = m / r;
      ((double*)a.inv_rho)[i] = 1.0 / r;
      if (eta_mode) ((double*)a.coef_e)[i] = e / r;
    } else {
      ((float*)a.coef_m)[i] = (float)(a.dt2 * (m / r));
      if (eta_mode) ((float*)a.coef_e)[i] = (float)(a.dT * (e / r));
    }
  }
}

// ---------------------------------------------------------------------------
// initial state (solver.py:147-171)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void init_kernel(StepArgs a, const T* __restrict__ iu, const T* __restrict__ iv) {
  const Geom g = a.g;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.ncell;
       i += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(i % g.pz);
    const long long xy = i / g.pz;
    const int y = (int)(xy % g.ny);
    const int x = (int)(xy / g.ny);
    const bool in = interior(g, x, y, z);
    const long long q = ((long long)x * g.ny + y) * g.nz + z;  // dense cell index
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double u0 = (in && iu) ? (double)iu[3 * q + c] : 0.0;
      const double v0 = (in && iv) ? (double)iv[3 * q + c] : 0.0;
      if (a.precision == SW_PLAIN_F64) {
        double* b0 = (double*)a.state[0];
        double* b1 = (double*)a.state[1];
        double* b2 = (double*)a.state[2];
        // u_prev = (u_curr - dT v) * mask; zero when initial_v is absent
        b0[c * g.ncell + i] = (in && iv) ? u0 - a.dT * v0 : 0.0;
        b1[c * g.ncell + i] = u0;
        b2[c * g.ncell + i] = 0.0;
      } else {
        float* s0 = (float*)a.state[0];
        // d = u_curr - u_prev: dT v with initial_v, u_curr without it
        const double d0 = iv ? a.dT * v0 : u0;
        s0[c * g.ncell + i] = (float)u0;
        s0[(3 + c) * g.ncell + i] = in ? (float)d0 : 0.0f;
        s0[(6 + c) * g.ncell + i] = 0.0f;
        for (int b = 1; b < 3; ++b) {
          float* sb = (float*)a.state[b];
          sb[c * g.ncell + i] = 0.0f;
          sb[(3 + c) * g.ncell + i] = 0.0f;
          sb[(6 + c) * g.ncell + i] = 0.0f;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// step kernels
// ---------------------------------------------------------------------------
__device__ inline long long snap_index(const Geom& g, int slot, int x, int y, int z, int c) {
  return ((((long long)slot * g.nx + x) * g.ny + y) * g.nz + z) * 3 + c;
}

// Plain FP64 step.  Mirrors solver.py:195-226 in operation order (products
// by reciprocals instead of divisions).
__global__ void __launch_bounds__(TILE_THREADS) step_f64(const __grid_constant__ StepArgs a,
                                                         int it) {
  const Geom& g = a.g;
  const double* __restrict__ up = (const double*)a.state[it % 3];
  const double* __restrict__ uc = (const double*)a.state[(it + 1) % 3];
  double* __restrict__ un = (double*)a.state[(it + 2) % 3];
  const double* __restrict__ mr = (const double*)a.coef_m;
  const double* __restrict__ er = (const double*)a.coef_e;
  const double* __restrict__ ir = (const double*)a.inv_rho;
  const double* __restrict__ pat = (const double*)a.patterns;
  const int j0 = a.term_off ? a.term_off[it] : 0;
  const int j1 = a.term_off ? a.term_off[it + 1] : 0;
  const bool snap = a.snap_stride > 0 && a.snaps != nullptr && ((it + 1) % a.snap_stride) == 0;
  const int slot = snap ? (it + 1) / a.snap_stride - 1 : 0;
  const long long sx = g.sxy, sy = g.pz;
  for (int t = blockIdx.x; t < a.ts.count; t += gridDim.x) {
    const TileCoord tc = tile_coord(g, a.ts, t);
    const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
    if (z < 1 || z > g.nz - 2 || y < 1 || y > g.ny - 2) continue;
    for (int x = tc.x0; x < tc.x1; ++x) {
      const long long i = (long long)x * sx + (long long)y * sy + z;
      const double m = mr[i];
      const double e = er ? er[i] : 0.0;
      const double rinv = ir[i];
      bool bad = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long b = c * g.ncell + i;
        const double ucc = uc[b];
        const double lap_u = ((uc[b + sx] - 2.0 * ucc) + uc[b - sx]) * a.ihx2 +
                             ((uc[b + sy] - 2.0 * ucc) + uc[b - sy]) * a.ihy2 +
                             ((uc[b + 1] - 2.0 * ucc) + uc[b - 1]) * a.ihz2;
        double f = 0.0;
        for (int j = j0; j < j1; ++j) {
          const double fj = pat[((long long)a.term_pat[j] * 3 + c) * g.ncell + i] * a.term_scale[j];
          f = (j == j0) ? fj : f + fj;
        }
        double acc = m * lap_u + f * rinv;
        const double upc = up[b];
        if (er) {
          const double vc = (ucc - upc) * a.inv_dt;
          const double lap_v =
              (((uc[b + sx] - up[b + sx]) * a.inv_dt - 2.0 * vc) + (uc[b - sx] - up[b - sx]) * a.inv_dt) *
                  a.ihx2 +
              (((uc[b + sy] - up[b + sy]) * a.inv_dt - 2.0 * vc) + (uc[b - sy] - up[b - sy]) * a.inv_dt) *
                  a.ihy2 +
              (((uc[b + 1] - up[b + 1]) * a.inv_dt - 2.0 * vc) + (uc[b - 1] - up[b - 1]) * a.inv_dt) *
                  a.ihz2;
          acc += e * lap_v;
        }
        double unew = (2.0 * ucc - upc) + a.dt2 * acc;
        if (a.use_damp) unew = ucc + a.damp * (unew - ucc);
        un[b] = unew;
        bad |= !isfinite(unew);
        if (snap) ((double*)a.snaps)[snap_index(g, slot, x, y, z, c)] = unew;
      }
      if (bad && a.flags) atomicOr(a.flags, 1);
    }
  }
}

// Mixed FP32 step in increment form with Kahan-compensated displacement.
__global__ void __launch_bounds__(TILE_THREADS) step_f32(const __grid_constant__ StepArgs a,
                                                         int it) {
  const Geom& g = a.g;
  const float* __restrict__ S = (const float*)a.state[it % 3];
  float* __restrict__ D = (float*)a.state[(it + 1) % 3];
  const float* __restrict__ mr = (const float*)a.coef_m;
  const float* __restrict__ er = (const float*)a.coef_e;
  const float* __restrict__ pat = (const float*)a.patterns;
  const int j0 = a.term_off ? a.term_off[it] : 0;
  const int j1 = a.term_off ? a.term_off[it + 1] : 0;
  const bool snap = a.snap_stride > 0 && a.snaps != nullptr && ((it + 1) % a.snap_stride) == 0;
  const int slot = snap ? (it + 1) / a.snap_stride - 1 : 0;
  const float hx = (float)a.ihx2, hy = (float)a.ihy2, hz = (float)a.ihz2;
  const float hc = lap7_centre_coef(hx, hy, hz);
  const float damp = (float)a.damp;
  const long long sx = g.sxy, sy = g.pz, nc = g.ncell;
  for (int t = blockIdx.x; t < a.ts.count; t += gridDim.x) {
    const TileCoord tc = tile_coord(g, a.ts, t);
    const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
    if (z < 1 || z > g.nz - 2 || y < 1 || y > g.ny - 2) continue;
    for (int x = tc.x0; x < tc.x1; ++x) {
      const long long i = (long long)x * sx + (long long)y * sy + z;
      const float m = mr[i];
      const float e = er ? er[i] : 0.0f;
      bool bad = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float* U = S + c * nc;
        const float* Dd = S + (3 + c) * nc;
        const float u0 = U[i], d0 = Dd[i];
        // the pair kernels' sequence (sw_step.cuh), one explicitly rounded
        // operation at a time
        const float lu = lap7f(__fadd_rn(U[i + sx], U[i - sx]), __fadd_rn(U[i + sy], U[i - sy]),
                               __fadd_rn(U[i + 1], U[i - 1]), u0, hx, hy, hz, hc);
        float inc = __fmaf_rn(m, lu, d0);
        if (er) {
          const float ld =
              lap7f(__fadd_rn(Dd[i + sx], Dd[i - sx]), __fadd_rn(Dd[i + sy], Dd[i - sy]),
                    __fadd_rn(Dd[i + 1], Dd[i - 1]), d0, hx, hy, hz, hc);
          inc = __fmaf_rn(e, ld, inc);
        }
        for (int j = j0; j < j1; ++j)
          inc = __fmaf_rn(pat[((long long)a.term_pat[j] * 3 + c) * nc + i],
                          (float)a.term_scale[j], inc);
        if (a.use_damp) inc = __fmul_rn(inc, damp);
        float unew, cnew;
        if (a.kahan) {
          const float cc = S[(6 + c) * nc + i];
          const float yk = __fsub_rn(inc, cc);
          unew = __fadd_rn(u0, yk);
          cnew = __fsub_rn(__fsub_rn(unew, u0), yk);
        } else {
          unew = __fadd_rn(u0, inc);
          cnew = 0.0f;
        }
        D[c * nc + i] = unew;
        D[(3 + c) * nc + i] = inc;
        D[(6 + c) * nc + i] = cnew;
        bad |= !isfinite(unew);
        if (snap) ((float*)a.snaps)[snap_index(g, slot, x, y, z, c)] = unew;
      }
      if (bad && a.flags) atomicOr(a.flags, 1);
    }
  }
}

// u_z at the trace cells after step `it` (shear_fdtd_jax trace semantics,
// solver.py:444-447: u_next[ix, iy, iz, 2]).
__global__ void trace_kernel(const __grid_constant__ StepArgs a, int it) {
  const Geom& g = a.g;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.n_traces;
       k += gridDim.x * blockDim.x) {
    const int x = a.trace_cells[3 * k], y = a.trace_cells[3 * k + 1], z = a.trace_cells[3 * k + 2];
    const long long i = (long long)x * g.sxy + (long long)y * g.pz + z + 2 * g.ncell;
    if (a.precision == SW_PLAIN_F64) {
      const double* un = (const double*)a.state[(it + 2) % 3];
      ((double*)a.traces)[(long long)k * a.n_steps + it] = un[i];
    } else {
      const float* D = (const float*)a.state[(it + 1) % 3];
      ((float*)a.traces)[(long long)k * a.n_steps + it] = D[i];
    }
  }
}

// ---------------------------------------------------------------------------
// outputs (solver.py:241-243)
// ---------------------------------------------------------------------------
// Also raises bit 0 of the solve's flag word when the final state holds a
// non-finite value: a NaN or an infinity, once in u or d, stays there, so
// the end state tells whether any step produced one (the mixed step kernels
// leave this check to here).
__global__ void finish_kernel(StepArgs a, int done, void* uo, void* vo) {
  const Geom g = a.g;
  const long long n = (long long)g.nx * g.ny * g.nz;
  bool bad = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(q % g.nz);
    const long long i = (q / g.nz) * g.pz + z;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (a.precision == SW_PLAIN_F64) {
        const double* up = (const double*)a.state[done % 3];
        const double* uc = (const double*)a.state[(done + 1) % 3];
        const double cu = uc[c * g.ncell + i];
        const double cv = (cu - up[c * g.ncell + i]) / a.dT;
        if (uo) ((double*)uo)[3 * q + c] = cu;
        if (vo) ((double*)vo)[3 * q + c] = cv;
        bad |= !isfinite(cu) || !isfinite(cv);
      } else {
        const float* S = (const float*)a.state[done % 3];
        const float cu = S[c * g.ncell + i], cd = S[(3 + c) * g.ncell + i];
        if (uo) ((float*)uo)[3 * q + c] = cu;
        if (vo) ((float*)vo)[3 * q + c] = cd / (float)a.dT;
        bad |= !isfinite(cu) || !isfinite(cd);
      }
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0 && a.flags) atomicOr(a.flags, 1);
}

// dst = src * scale / rho  (see sw_convert)
template <typename Tout, typename Trho>
__global__ void convert_kernel(int ncomp, const double* __restrict__ src, Geom g, Tout* dst,
                               long long cs, long long sx, long long sy, long long sz,
                               double scale, const Trho* __restrict__ rho, long long rx,
                               long long ry, long long rz) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(q % g.nz);
    const long long xy = q / g.nz;
    const int y = (int)(xy % g.ny);
    const int x = (int)(xy / g.ny);
    const long long i = xy * g.pz + z;
    double f = scale;
    if (rho) f = scale / (double)rho[x * rx + y * ry + z * rz];
    for (int c = 0; c < ncomp; ++c)
      dst[c * cs + x * sx + y * sy + z * sz] = (Tout)(src[c * g.ncell + i] * f);
  }
}

// padded FP64 field -> state buffer components (re-projection write-back)
__global__ void write_back_kernel(const double* __restrict__ src, Geom g, void* dst, int f32,
                                  long long comp0) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3 * g.ncell;
       i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / g.ncell, r = i % g.ncell;
    if (f32) ((float*)dst)[(comp0 + c) * g.ncell + r] = (float)src[i];
    else ((double*)dst)[(comp0 + c) * g.ncell + r] = src[i];
  }
}

__global__ void zero_comp_kernel(float* dst, Geom g, long long comp0, int ncomp) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ncomp * g.ncell;
       i += (long long)gridDim.x * blockDim.x)
    dst[comp0 * g.ncell + i] = 0.0f;
}

int launch_steps(const StepArgs& a, int it0, int nsteps, cudaStream_t s) {
  if (a.ts.count == 0) return SW_OK;
  if (a.kernel == 0 && a.n_traces == 0) return launch_steps_tma(a, a.xchunk, it0, nsteps, s);
  if (a.kernel == 0) {  // TMA steps one at a time, with the trace gather after each
    for (int it = it0; it < it0 + nsteps; ++it) {
      int rc = launch_steps_tma(a, a.xchunk, it, 1, s);
      if (rc != SW_OK) return rc;
      trace_kernel<<<(a.n_traces + 127) / 128, 128, 0, s>>>(a, it);
      count_launches(1);
    }
    SW_CHECK_LAUNCH("trace");
    return SW_OK;
  }
  const int grid = std::min(a.ts.count, 148 * 16);
  for (int it = it0; it < it0 + nsteps; ++it) {
    if (a.precision == SW_PLAIN_F64)
      step_f64<<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(a, it);
    else
      step_f32<<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(a, it);
    if (a.n_traces > 0) trace_kernel<<<(a.n_traces + 127) / 128, 128, 0, s>>>(a, it);
  }
  count_launches((unsigned long long)nsteps * (a.n_traces > 0 ? 2 : 1));
  SW_CHECK_LAUNCH("step");
  return SW_OK;
}

}  // namespace sw

using namespace sw;

extern "C" int sw_fdtd_materials(const sw_fdtd_desc* d, int in_dtype, const void* rho,
                                 double rho_s, const void* mu, double mu_s, int eta_mode,
                                 const void* eta, double eta_s, void* stream) {
  StepArgs a;
  int rc = make_step_args(d, &a);
  if (rc != SW_OK) return rc;
  if (eta_mode && a.coef_e == nullptr) {
    set_error("sw_fdtd_materials: eta requested but coef_e is null");
    return SW_EINVAL;
  }
  const long long n = (long long)a.g.nx * a.g.ny * a.g.nz;
  const int grid = grid_blocks(n, 256, 148 * 32);
  cudaStream_t s = (cudaStream_t)stream;
  if (in_dtype == SW_F32)
    materials_kernel<float><<<grid, 256, 0, s>>>(a, (const float*)rho, rho_s, (const float*)mu,
                                                 mu_s, eta_mode, (const float*)eta, eta_s);
  else if (in_dtype == SW_F64)
    materials_kernel<double><<<grid, 256, 0, s>>>(a, (const double*)rho, rho_s,
                                                  (const double*)mu, mu_s, eta_mode,
                                                  (const double*)eta, eta_s);
  else {
    set_error("sw_fdtd_materials: unknown dtype %d", in_dtype);
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("materials");
  return SW_OK;
}

extern "C" int sw_fdtd_init(const sw_fdtd_desc* d, const void* init_u, const void* init_v,
                            void* stream) {
  StepArgs a;
  int rc = make_step_args(d, &a);
  if (rc != SW_OK) return rc;
  const int grid = grid_blocks(a.g.ncell, 256, 148 * 32);
  cudaStream_t s = (cudaStream_t)stream;
  if (a.precision == SW_PLAIN_F64)
    init_kernel<double><<<grid, 256, 0, s>>>(a, (const double*)init_u, (const double*)init_v);
  else
    init_kernel<float><<<grid, 256, 0, s>>>(a, (const float*)init_u, (const float*)init_v);
  count_launches(1);
  SW_CHECK_LAUNCH("init");
  return SW_OK;
}

extern "C" int sw_fdtd_steps(const sw_fdtd_desc* d, int32_t it0, int32_t nsteps, void* stream) {
  StepArgs a;
  int rc = make_step_args(d, &a);
  if (rc != SW_OK) return rc;
  if (it0 < 0 || nsteps < 0 || it0 + nsteps > a.n_steps) {
    set_error("sw_fdtd_steps: steps [%d, %d) outside [0, %d)", it0, it0 + nsteps, a.n_steps);
    return SW_EINVAL;
  }
  return launch_steps(a, it0, nsteps, (cudaStream_t)stream);
}

extern "C" int sw_fdtd_finish(const sw_fdtd_desc* d, int32_t steps_done, void* u_out,
                              void* v_out, void* stream) {
  StepArgs a;
  int rc = make_step_args(d, &a);
  if (rc != SW_OK) return rc;
  const long long n = (long long)a.g.nx * a.g.ny * a.g.nz;
  finish_kernel<<<grid_blocks(n, 256, 148 * 32), 256, 0, (cudaStream_t)stream>>>(a, steps_done,
                                                                                  u_out, v_out);
  count_launches(1);
  SW_CHECK_LAUNCH("finish");
  return SW_OK;
}

extern "C" int sw_fdtd_status(const sw_fdtd_desc* d, int32_t* host_flags, void* stream) {
  if (d == nullptr) {
    set_error("sw_fdtd_status: null descriptor");
    return SW_EINVAL;
  }
  int32_t f = 0;
  if (d->flags != nullptr) {
    cudaError_t e = cudaMemcpyAsync(&f, d->flags, sizeof f, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e, "sw_fdtd_status");
  } else {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_status(e, "sw_fdtd_status");
  }
  if (host_flags != nullptr) *host_flags = f;
  if (f & kFlagTimeout) {
    set_error("a step kernel's bounded wait ran out: tiles of this solve were abandoned");
    return SW_ETIMEOUT;
  }
  if (f & kFlagRefused) {
    set_error("a step launch refused to issue a TMA to a misaligned shared-memory destination");
    return SW_ETIMEOUT;
  }
  if (f & kFlagNonFinite) {
    set_error("non-finite displacement in the state");
    return SW_ENONFINITE;
  }
  return SW_OK;
}

extern "C" int sw_fdtd_reproject(const sw_fdtd_desc* d, int32_t steps_done, double tol,
                                 int max_iters, double* tmp, void* workspace,
                                 size_t workspace_bytes, sw_cg_stats* stats, void* stream) {
  StepArgs a;
  int rc = make_step_args(d, &a);
  if (rc != SW_OK) return rc;
  if (tmp == nullptr) {
    set_error("sw_fdtd_reproject: null tmp");
    return SW_EINVAL;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const Geom& g = a.g;
  InStride st{g.sxy, g.pz, 1};
  const int grid = grid_blocks(3 * g.ncell, 256, 148 * 32);
  if (a.precision == SW_PLAIN_F64) {
    // u_curr then u_prev (solver.py:237-239)
    double* bufs[2] = {(double*)a.state[(steps_done + 1) % 3], (double*)a.state[steps_done % 3]};
    for (int k = 0; k < 2; ++k) {
      double* b = bufs[k];
      rc = project_field(SW_F64, b, b + g.ncell, b + 2 * g.ncell, st, g, d->dX, d->dY, d->dZ, tol,
                         max_iters, tmp, workspace, workspace_bytes, stats ? stats + k : nullptr,
                         s);
      if (rc != SW_OK) return rc;
      write_back_kernel<<<grid, 256, 0, s>>>(tmp, g, b, 0, 0);
      count_launches(1);
      SW_CHECK_LAUNCH("reproject write-back");
    }
  } else {
    // project u and the increment d (= P(u_curr) - P(u_prev) by linearity)
    float* S = (float*)a.state[steps_done % 3];
    for (int k = 0; k < 2; ++k) {
      float* b = S + (long long)(3 * k) * g.ncell;
      rc = project_field(SW_F32, b, b + g.ncell, b + 2 * g.ncell, st, g, d->dX, d->dY, d->dZ, tol,
                         max_iters, tmp, workspace, workspace_bytes, stats ? stats + k : nullptr,
                         s);
      if (rc != SW_OK) return rc;
      write_back_kernel<<<grid, 256, 0, s>>>(tmp, g, S, 1, 3 * k);
      count_launches(1);
      SW_CHECK_LAUNCH("reproject write-back");
    }
    zero_comp_kernel<<<grid, 256, 0, s>>>(S, g, 6, 3);
    count_launches(1);
    SW_CHECK_LAUNCH("reproject reset");
  }
  return SW_OK;
}

extern "C" int sw_convert(int ncomp, const double* src, int nx, int ny, int nz, int out_dtype,
                          void* dst, int64_t dst_cs, int64_t dst_sx, int64_t dst_sy,
                          int64_t dst_sz, double scale, int rho_dtype, const void* rho,
                          int64_t rho_sx, int64_t rho_sy, int64_t rho_sz, void* stream) {
  if (src == nullptr || dst == nullptr || nx <= 0 || ny <= 0 || nz <= 0 || ncomp <= 0) {
    set_error("sw_convert: bad arguments");
    return SW_EINVAL;
  }
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  const long long n = (long long)nx * ny * nz;
  const int grid = grid_blocks(n, 256, 148 * 32);
  cudaStream_t s = (cudaStream_t)stream;
#define SW_CONV(TO, TR)                                                                     \
  convert_kernel<TO, TR><<<grid, 256, 0, s>>>(ncomp, src, g, (TO*)dst, dst_cs, dst_sx, dst_sy, \
                                              dst_sz, scale, (const TR*)rho, rho_sx, rho_sy,  \
                                              rho_sz)
  if (out_dtype == SW_F32 && rho_dtype == SW_F32) SW_CONV(float, float);
  else if (out_dtype == SW_F32 && rho_dtype == SW_F64) SW_CONV(float, double);
  else if (out_dtype == SW_F64 && rho_dtype == SW_F32) SW_CONV(double, float);
  else if (out_dtype == SW_F64 && rho_dtype == SW_F64) SW_CONV(double, double);
  else {
    set_error("sw_convert: unknown dtype");
    return SW_EINVAL;
  }
#undef SW_CONV
  count_launches(1);
  SW_CHECK_LAUNCH("convert");
  return SW_OK;
}
