// Acoustic radiation force from recorded pressure (and particle velocity):
// the producers that feed shear_fdtd's body force.
//
// Reference: compute_radiation_force and compute_radiation_force_velocity
// (src/shearwave/radiation_force.py:27-85, 88-157).  Inputs are the
// reference's (nx, ny, nz, nt) arrays, time fastest, so a cell's series is
// one contiguous row of nt values:
//
//  * arf_env_partial / arf_env_final: the auto-gate envelope
//    env[t] = mean over cells of p[cell, t]^2 (radiation_force.py:63-68),
//    a column reduction of the (cells x nt) matrix.  Each block reduces a
//    contiguous band of rows with threads across columns (coalesced), into
//    FP64 partials that a second kernel sums in block order: deterministic.
//  * arf_force: per cell, a group of lanes reads the gated entries of its
//    row, reduces sum p*q in FP64 (q = p, or a velocity component), and the
//    group leader applies the reference's formula:
//      alpha_Np = alpha_coeff * f0_MHz / 8.685889638 * 100
//      scalar:  b = 2 alpha_Np (mean p^2 / (rho c)) / c
//      vector:  b_i = (2 alpha_Np / c) mean(p v_i)
// Both passes are HBM-bound reads of the pressure (and velocity) records.
#include <algorithm>

#include "sw_common.cuh"

namespace sw {
namespace {

constexpr int kEnvThreads = 256, kEnvCols = 4;  // columns per thread per chunk

template <typename T>
__global__ void __launch_bounds__(kEnvThreads)
    arf_env_partial(const T* __restrict__ p, long long ncell, int nt, long long rows_per_block,
                    double* __restrict__ partials) {
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  const long long r1 = r0 + rows_per_block < ncell ? r0 + rows_per_block : ncell;
  for (int cb = 0; cb < nt; cb += kEnvThreads * kEnvCols) {
    double acc[kEnvCols];
#pragma unroll
    for (int k = 0; k < kEnvCols; ++k) acc[k] = 0.0;
#pragma unroll 4
    for (long long r = r0; r < r1; ++r) {
      const T* row = p + r * nt;
#pragma unroll
      for (int k = 0; k < kEnvCols; ++k) {
        const int col = cb + threadIdx.x + k * kEnvThreads;
        if (col < nt) {
          const double v = (double)row[col];
          acc[k] += v * v;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kEnvCols; ++k) {
      const int col = cb + threadIdx.x + k * kEnvThreads;
      if (col < nt) partials[(long long)blockIdx.x * nt + col] = acc[k];
    }
  }
}

__global__ void arf_env_final(const double* __restrict__ partials, int nblk, int nt,
                              long long ncell, double* __restrict__ env) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += partials[(long long)b * nt + t];
    env[t] = s / (double)ncell;
  }
}

// Sum over the G lanes of a group (G a power of two <= 32, groups aligned).
template <int G>
__device__ inline double group_sum(double v) {
#pragma unroll
  for (int off = G / 2; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

struct ArfMaps {
  const double *c, *rho, *alpha;  // per cell, or one value when stride is 0
  long long stride;
};

template <typename T, typename To, int NF, int G>
__global__ void __launch_bounds__(256)
    arf_force(const T* __restrict__ p, const T* __restrict__ q0, const T* __restrict__ q1,
              const T* __restrict__ q2, long long ncell, int nt, const int* __restrict__ gate,
              int ngate, ArfMaps m, double f0_mhz, To* __restrict__ o0, To* __restrict__ o1,
              To* __restrict__ o2) {
  const int lane = threadIdx.x & 31, sub = lane & (G - 1);
  const long long group = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const long long ngroups = ((long long)gridDim.x * blockDim.x) / G;
  // every lane of a warp runs the same number of iterations (the shuffles
  // need the whole warp): loop to the warp's last group, skip cells >= ncell
  const long long warp_first = group - lane / G;
  for (long long base = warp_first; base < ncell; base += ngroups) {
    const long long cell = base + lane / G;
    const bool live = cell < ncell;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (live) {
      const long long row = cell * nt;
      for (int j = sub; j < ngate; j += G) {
        const int g = __ldg(gate + j);
        if ((unsigned)g >= (unsigned)nt) continue;  // the host validates; never read outside
        const long long k = row + g;
        const double pv = (double)p[k];
        if (NF == 1) {
          s0 += pv * pv;
        } else {
          s0 += pv * (double)q0[k];
          s1 += pv * (double)q1[k];
          s2 += pv * (double)q2[k];
        }
      }
    }
    s0 = group_sum<G>(s0);
    if (NF == 3) {
      s1 = group_sum<G>(s1);
      s2 = group_sum<G>(s2);
    }
    if (live && sub == 0) {
      const long long mi = cell * m.stride;
      const double c = m.c[mi], rho = m.rho[mi], alpha = m.alpha[mi];
      const double alpha_np = alpha * f0_mhz / 8.685889638 * 100.0;
      const double inv_n = 1.0 / (double)ngate;
      if (NF == 1) {
        const double isppa = (s0 * inv_n) / (rho * c);
        o0[cell] = (To)(2.0 * alpha_np * isppa / c);
      } else {
        const double coeff = 2.0 * alpha_np / c;
        o0[cell] = (To)(coeff * (s0 * inv_n));
        o1[cell] = (To)(coeff * (s1 * inv_n));
        o2[cell] = (To)(coeff * (s2 * inv_n));
      }
    }
  }
}

long long env_blocks(long long ncell) {
  const long long want = 8LL * kNumSMs;
  return ncell < want ? (ncell > 0 ? ncell : 1) : want;
}

template <typename T, typename To, int NF>
int launch_force(const void* p, const void* const* q, long long ncell, int nt, const int* gate,
                 int ngate, ArfMaps m, double f0_mhz, void* const* out, cudaStream_t s) {
  const long long warps = std::min<long long>((ncell + 3) / 4, 32LL * kNumSMs * 8);
  const int blocks = (int)std::max<long long>(1, (warps * 32 + 255) / 256);
  const T* pp = (const T*)p;
  const T* qa = NF == 3 ? (const T*)q[0] : nullptr;
  const T* qb = NF == 3 ? (const T*)q[1] : nullptr;
  const T* qc = NF == 3 ? (const T*)q[2] : nullptr;
  To* oa = (To*)out[0];
  To* ob = NF == 3 ? (To*)out[1] : nullptr;
  To* oc = NF == 3 ? (To*)out[2] : nullptr;
  // lanes per cell: enough to keep a row's gated entries in few passes
  if (ngate <= 8)
    arf_force<T, To, NF, 4><<<blocks, 256, 0, s>>>(pp, qa, qb, qc, ncell, nt, gate, ngate, m,
                                                    f0_mhz, oa, ob, oc);
  else if (ngate <= 32)
    arf_force<T, To, NF, 8><<<blocks, 256, 0, s>>>(pp, qa, qb, qc, ncell, nt, gate, ngate, m,
                                                    f0_mhz, oa, ob, oc);
  else if (ngate <= 128)
    arf_force<T, To, NF, 16><<<blocks, 256, 0, s>>>(pp, qa, qb, qc, ncell, nt, gate, ngate, m,
                                                     f0_mhz, oa, ob, oc);
  else
    arf_force<T, To, NF, 32><<<blocks, 256, 0, s>>>(pp, qa, qb, qc, ncell, nt, gate, ngate, m,
                                                     f0_mhz, oa, ob, oc);
  count_launches(1);
  SW_CHECK_LAUNCH("radiation force");
  return SW_OK;
}

}  // namespace
}  // namespace sw

using namespace sw;

extern "C" size_t sw_arf_workspace_bytes(int64_t ncell, int32_t nt) {
  if (ncell <= 0 || nt <= 0) return 0;
  return (size_t)env_blocks(ncell) * (size_t)nt * sizeof(double);
}

extern "C" int sw_arf_envelope(int dtype, const void* p, int64_t ncell, int32_t nt, double* env,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (p == nullptr || env == nullptr || ncell <= 0 || nt <= 0 ||
      (dtype != SW_F32 && dtype != SW_F64)) {
    set_error("sw_arf_envelope: bad arguments");
    return SW_EINVAL;
  }
  if (workspace == nullptr || workspace_bytes < sw_arf_workspace_bytes(ncell, nt)) {
    set_error("sw_arf_envelope: workspace must be >= %zu bytes", sw_arf_workspace_bytes(ncell, nt));
    return SW_EWORKSPACE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long long nblk = env_blocks(ncell);
  const long long rows = (ncell + nblk - 1) / nblk;
  double* part = (double*)workspace;
  if (dtype == SW_F32)
    arf_env_partial<float><<<(int)nblk, kEnvThreads, 0, s>>>((const float*)p, ncell, nt, rows, part);
  else
    arf_env_partial<double><<<(int)nblk, kEnvThreads, 0, s>>>((const double*)p, ncell, nt, rows,
                                                              part);
  arf_env_final<<<(nt + 255) / 256, 256, 0, s>>>(part, (int)nblk, nt, ncell, env);
  count_launches(2);
  SW_CHECK_LAUNCH("radiation-force envelope");
  return SW_OK;
}

extern "C" int sw_arf_force(int dtype, int n_fields, const void* p, const void* vx,
                            const void* vy, const void* vz, int64_t ncell, int32_t nt,
                            const int32_t* gate, int32_t n_gate, const double* c_map,
                            const double* rho_map, const double* alpha_map, int64_t map_stride,
                            double f0, int out_dtype, void* out0, void* out1, void* out2,
                            void* stream) {
  const bool ok_types = (dtype == SW_F32 || dtype == SW_F64) &&
                        (out_dtype == SW_F32 || out_dtype == SW_F64);
  if (!ok_types || p == nullptr || ncell <= 0 || nt <= 0 || gate == nullptr || n_gate <= 0 ||
      c_map == nullptr || rho_map == nullptr || alpha_map == nullptr ||
      (map_stride != 0 && map_stride != 1) || out0 == nullptr ||
      (n_fields != 1 && n_fields != 3) ||
      (n_fields == 3 && (vx == nullptr || vy == nullptr || vz == nullptr || out1 == nullptr ||
                         out2 == nullptr))) {
    set_error("sw_arf_force: bad arguments");
    return SW_EINVAL;
  }
  ArfMaps m{c_map, rho_map, alpha_map, map_stride};
  const void* q[3] = {vx, vy, vz};
  void* out[3] = {out0, out1, out2};
  const double f0_mhz = f0 / 1e6;
  cudaStream_t s = (cudaStream_t)stream;
  const bool f32 = dtype == SW_F32, o32 = out_dtype == SW_F32;
  if (n_fields == 1) {
    if (f32 && o32) return launch_force<float, float, 1>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
    if (f32) return launch_force<float, double, 1>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
    if (o32) return launch_force<double, float, 1>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
    return launch_force<double, double, 1>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
  }
  if (f32 && o32) return launch_force<float, float, 3>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
  if (f32) return launch_force<float, double, 3>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
  if (o32) return launch_force<double, float, 3>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
  return launch_force<double, double, 3>(p, q, ncell, nt, gate, n_gate, m, f0_mhz, out, s);
}
