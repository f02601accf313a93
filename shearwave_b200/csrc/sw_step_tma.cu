// TMA-staged fused step kernels (the production time-loop kernels).
//
// Same arithmetic as the reference update (src/shearwave/solver.py:195-226)
// and as the direct-load kernels in sw_step.cu, reorganised for B200:
//
//  * A CTA owns a TZ x TY tile of the (z, y) plane and marches along x over a
//    chunk of planes.  For every plane it needs the halo'd fields (u and d in
//    the mixed form, u_prev and u_curr in the plain form) at x-1, x, x+1.
//  * One elected thread streams planes into a 4-stage shared-memory ring with
//    4-D TMA tile loads (all halo'd components of a plane in one box, or two
//    boxes for the two FP64 buffers), completion on one mbarrier per stage.
//    Two planes are always in flight ahead of the plane being computed.
//  * The box starts 4 (FP32) / 2 (FP64) cells before the tile in z so the
//    innermost coordinate stays 16-byte aligned; y starts one row before.
//    Out-of-range rows/columns are zero-filled by TMA.
//  * Point-wise inputs (Kahan compensation, material coefficients, forces)
//    are read straight from global memory, coalesced along z; outputs are
//    written with coalesced stores.
// Every mbarrier wait is bounded; a timeout sets bit 1 of the solve's flag
// word and the CTA drains its outstanding copies (bounded) and returns.
#include <math.h>

#include <algorithm>

#include "sw_common.cuh"
#include "sw_step.cuh"
#include "sw_step_tma.cuh"
#include "sw_tma.cuh"

namespace sw {

// ---------------------------------------------------------------------------
// driver entry point for tensor-map encoding
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (fn == nullptr) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

int encode_tmap_4d(CUtensorMap* map, CUtensorMapDataType dt, void* base, const uint64_t dims[4],
                   const uint64_t strides_bytes[3], const uint32_t box[4]) {
  EncodeTiledFn fn = encode_fn();
  if (fn == nullptr) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return SW_ECUDA;
  }
  cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
  cuuint64_t s[3] = {strides_bytes[0], strides_bytes[1], strides_bytes[2]};
  cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
  cuuint32_t e[4] = {1, 1, 1, 1};
  CUresult r = fn(map, dt, 4, base, d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with CUresult %d", (int)r);
    return SW_ECUDA;
  }
  return SW_OK;
}

// ---------------------------------------------------------------------------
// shared pipeline helpers
// ---------------------------------------------------------------------------
struct Ring {
  uint64_t* bars;   // NST mbarriers
  uint32_t phases;  // parity bit per stage (uniform across the block)
};

// Wait for the next completion of `stage`; false when the bounded wait ran out.
__device__ inline bool ring_wait(Ring& r, int stage) {
  const uint32_t par = (r.phases >> stage) & 1u;
  const bool ok = mbar_wait_bounded(&r.bars[stage], par);
  r.phases ^= (1u << stage);
  return ok;
}

// ---------------------------------------------------------------------------
// mixed FP32 step, one tile
// ---------------------------------------------------------------------------
__device__ inline void tile_f32(const TmaF32& in, int local, int lit, float* sm, Ring& ring,
                                int* abort_flag) {
  constexpr int W = TmaF32::W, H = TmaF32::H, NST = TmaF32::NST, PL = TmaF32::STAGE;
  constexpr uint32_t BYTES = TmaF32::PLANE * sizeof(float);
  static_assert((PL * sizeof(float)) % 128 == 0, "TMA destinations must be 128-byte aligned");
  const Geom& g = in.g;
  const TileCoord tc = tile_coord_t(g, in.ts, local, TmaF32::TZ, TmaF32::TY);
  const CUtensorMap* tm = &in.tm[lit & 1];
  const float* __restrict__ S = in.state[lit & 1];
  float* __restrict__ D = in.state[(lit + 1) & 1];
  const int pfirst = tc.x0 - 1, plast = tc.x1;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int k = 0; k < NST && pfirst + k <= plast; ++k) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&ring.bars[k], BYTES);
      tma_load_4d(sm + k * PL, tm, &ring.bars[k], tc.z0 - 4, tc.y0 - 1, pfirst + k, 0);
    }
  }
  const int ly = tid >> 5, lane = tid & 31;
  const int y = tc.y0 + ly;
  const bool yin = (y >= 1 && y <= g.ny - 2);
  const int zc[2] = {tc.z0 + lane, tc.z0 + lane + 32};
  const bool act[2] = {yin && zc[0] >= 1 && zc[0] <= g.nz - 2,
                       yin && zc[1] >= 1 && zc[1] <= g.nz - 2};
  const int j0 = in.term_off ? in.term_off[lit] : 0;
  const int j1 = in.term_off ? in.term_off[lit + 1] : 0;
  const bool snap = in.snap_stride > 0 && in.snaps != nullptr && ((lit + 1) % in.snap_stride) == 0;
  const int slot = snap ? (lit + 1) / in.snap_stride - 1 : 0;
  const long long nc = g.ncell;
  for (int x = tc.x0; x < tc.x1; ++x) {
    bool ok = true;
    if (x == tc.x0) {
      ok &= ring_wait(ring, 0);
      ok &= ring_wait(ring, 1 % NST);
    }
    const int rel = x - pfirst;  // plane x-1 has rel-1
    const int sp = (rel - 1) % NST, sc = rel % NST, sn = (rel + 1) % NST;
    ok &= ring_wait(ring, sn);
    if (__syncthreads_or(!ok)) {  // block-uniform decision
      if (tid == 0) *abort_flag = 1;
      __syncthreads();
      return;
    }
    const float* Pp = sm + sp * PL;
    const float* Pc = sm + sc * PL;
    const float* Pn = sm + sn * PL;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (!act[k]) continue;
      const int z = zc[k];
      const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
      const float m = in.m[i];
      const float e = in.e ? in.e[i] : 0.0f;
      const int row = ly + 1, col = lane + 32 * k + 4;
      bool bad = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int o = (c * H + row) * W + col;
        const int od = o + 3 * H * W;
        const float u0 = Pc[o], d0 = Pc[od];
        const float lu = ((Pn[o] + Pp[o]) - 2.0f * u0) * in.hx +
                         ((Pc[o + W] + Pc[o - W]) - 2.0f * u0) * in.hy +
                         ((Pc[o + 1] + Pc[o - 1]) - 2.0f * u0) * in.hz;
        float inc = d0 + m * lu;
        if (in.e) {
          const float ld = ((Pn[od] + Pp[od]) - 2.0f * d0) * in.hx +
                           ((Pc[od + W] + Pc[od - W]) - 2.0f * d0) * in.hy +
                           ((Pc[od + 1] + Pc[od - 1]) - 2.0f * d0) * in.hz;
          inc += e * ld;
        }
        for (int j = j0; j < j1; ++j)
          inc += in.pat[((long long)in.term_pat[j] * 3 + c) * nc + i] * (float)in.term_scale[j];
        if (in.use_damp) inc *= in.damp;
        float unew, cnew;
        if (in.kahan) {
          const float cc = S[(6 + c) * nc + i];
          const float yk = inc - cc;
          unew = u0 + yk;
          cnew = (unew - u0) - yk;
        } else {
          unew = u0 + inc;
          cnew = 0.0f;
        }
        D[c * nc + i] = unew;
        D[(3 + c) * nc + i] = inc;
        D[(6 + c) * nc + i] = cnew;
        bad |= !isfinite(unew);
        if (snap)
          in.snaps[((((long long)slot * g.nx + x) * g.ny + y) * g.nz + z) * 3 + c] = unew;
      }
      if (bad && in.flags) atomicOr(in.flags, 1);
    }
    __syncthreads();  // every thread is done with plane x-1's stage
    if (tid == 0) {
      const int p = x - 1 + NST;
      if (p <= plast) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&ring.bars[sp], BYTES);
        tma_load_4d(sm + sp * PL, tm, &ring.bars[sp], tc.z0 - 4, tc.y0 - 1, p, 0);
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// plain FP64 step, one tile
// ---------------------------------------------------------------------------
__device__ inline void tile_f64(const TmaF64& in, int local, int lit, double* sm, Ring& ring,
                                int* abort_flag) {
  constexpr int W = TmaF64::W, H = TmaF64::H, NST = TmaF64::NST, PL = TmaF64::STAGE;
  constexpr int HALF = TmaF64::HALF;
  constexpr uint32_t BYTES = TmaF64::PLANE * sizeof(double);
  static_assert((HALF * sizeof(double)) % 128 == 0, "TMA destinations must be 128-byte aligned");
  const Geom& g = in.g;
  const TileCoord tc = tile_coord_t(g, in.ts, local, TmaF64::TZ, TmaF64::TY);
  const CUtensorMap* tmp = &in.tm[lit % 3];
  const CUtensorMap* tmc = &in.tm[(lit + 1) % 3];
  double* __restrict__ un = in.state[(lit + 2) % 3];
  const int pfirst = tc.x0 - 1, plast = tc.x1;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int k = 0; k < NST && pfirst + k <= plast; ++k) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&ring.bars[k], BYTES);
      tma_load_4d(sm + k * PL, tmp, &ring.bars[k], tc.z0 - 2, tc.y0 - 1, pfirst + k, 0);
      tma_load_4d(sm + k * PL + HALF, tmc, &ring.bars[k], tc.z0 - 2, tc.y0 - 1, pfirst + k, 0);
    }
  }
  const int ly = tid >> 5, lane = tid & 31;
  const int y = tc.y0 + ly, z = tc.z0 + lane;
  const bool act = (y >= 1 && y <= g.ny - 2 && z >= 1 && z <= g.nz - 2);
  const int j0 = in.term_off ? in.term_off[lit] : 0;
  const int j1 = in.term_off ? in.term_off[lit + 1] : 0;
  const bool snap = in.snap_stride > 0 && in.snaps != nullptr && ((lit + 1) % in.snap_stride) == 0;
  const int slot = snap ? (lit + 1) / in.snap_stride - 1 : 0;
  const long long nc = g.ncell;
  const double ihx2 = in.ihx2, ihy2 = in.ihy2, ihz2 = in.ihz2, inv_dt = in.inv_dt;
  for (int x = tc.x0; x < tc.x1; ++x) {
    bool ok = true;
    if (x == tc.x0) {
      ok &= ring_wait(ring, 0);
      ok &= ring_wait(ring, 1 % NST);
    }
    const int rel = x - pfirst;
    const int sp = (rel - 1) % NST, sc = rel % NST, sn = (rel + 1) % NST;
    ok &= ring_wait(ring, sn);
    if (__syncthreads_or(!ok)) {  // block-uniform decision
      if (tid == 0) *abort_flag = 1;
      __syncthreads();
      return;
    }
    if (act) {
      const double* Pp = sm + sp * PL;
      const double* Pc = sm + sc * PL;
      const double* Pn = sm + sn * PL;
      const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
      const double m = in.m[i];
      const double e = in.e ? in.e[i] : 0.0;
      const double rinv = (j1 > j0) ? in.ir[i] : 0.0;
      const int row = ly + 1, col = lane + 2;
      bool bad = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int op = (c * H + row) * W + col;  // u_prev component c
        const int oc = op + HALF;                // u_curr component c
        const double ucc = Pc[oc];
        const double lap_u = ((Pn[oc] - 2.0 * ucc) + Pp[oc]) * ihx2 +
                             ((Pc[oc + W] - 2.0 * ucc) + Pc[oc - W]) * ihy2 +
                             ((Pc[oc + 1] - 2.0 * ucc) + Pc[oc - 1]) * ihz2;
        double f = 0.0;
        for (int j = j0; j < j1; ++j) {
          const double fj = in.pat[((long long)in.term_pat[j] * 3 + c) * nc + i] * in.term_scale[j];
          f = (j == j0) ? fj : f + fj;
        }
        double acc = m * lap_u + f * rinv;
        const double upc = Pc[op];
        if (in.e) {
          const double vc = (ucc - upc) * inv_dt;
          const double lap_v =
              (((Pn[oc] - Pn[op]) * inv_dt - 2.0 * vc) + (Pp[oc] - Pp[op]) * inv_dt) * ihx2 +
              (((Pc[oc + W] - Pc[op + W]) * inv_dt - 2.0 * vc) + (Pc[oc - W] - Pc[op - W]) * inv_dt) *
                  ihy2 +
              (((Pc[oc + 1] - Pc[op + 1]) * inv_dt - 2.0 * vc) + (Pc[oc - 1] - Pc[op - 1]) * inv_dt) *
                  ihz2;
          acc += e * lap_v;
        }
        double unew = (2.0 * ucc - upc) + in.dt2 * acc;
        if (in.use_damp) unew = ucc + in.damp * (unew - ucc);
        un[c * nc + i] = unew;
        bad |= !isfinite(unew);
        if (snap)
          in.snaps[((((long long)slot * g.nx + x) * g.ny + y) * g.nz + z) * 3 + c] = unew;
      }
      if (bad && in.flags) atomicOr(in.flags, 1);
    }
    __syncthreads();
    if (tid == 0) {
      const int p = x - 1 + NST;
      if (p <= plast) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&ring.bars[sp], BYTES);
        tma_load_4d(sm + sp * PL, tmp, &ring.bars[sp], tc.z0 - 2, tc.y0 - 1, p, 0);
        tma_load_4d(sm + sp * PL + HALF, tmc, &ring.bars[sp], tc.z0 - 2, tc.y0 - 1, p, 0);
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <typename Inst>
__device__ inline int find_tma_inst(const Inst* __restrict__ tab, int ninst, int t) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (tab[mid].tile_base <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Drain: wait (bounded) until every stage with an outstanding load has
// completed, so no copy is still writing this CTA's shared memory.
template <int NST>
__device__ inline void ring_drain(Ring& ring, int outstanding_mask) {
  if (threadIdx.x != 0) return;
  for (int s = 0; s < NST; ++s)
    if (outstanding_mask & (1 << s)) mbar_wait_bounded(&ring.bars[s], (ring.phases >> s) & 1u);
}

template <bool BATCH>
__global__ void __launch_bounds__(256, 3)
    step_f32_tma(const __grid_constant__ TmaF32 one, const TmaF32* __restrict__ tab, int ninst,
                 int ntiles, int it) {
  extern __shared__ unsigned char smem_raw[];
  // 128-byte aligned header (mbarriers, abort flag) followed by the stages
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  int& abort_flag = *reinterpret_cast<int*>(base + 64);
  float* sm = reinterpret_cast<float*>(base + 128);
  if ((smem_addr(sm) & 127u) != 0u) {  // never issue a TMA to a misaligned destination
    int* fl = BATCH ? (ninst > 0 ? tab[0].flags : nullptr) : one.flags;
    if (threadIdx.x == 0 && fl) atomicOr(fl, 4);
    return;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < TmaF32::NST; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    abort_flag = 0;
  }
  __syncthreads();
  Ring ring{bars, 0u};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TmaF32* in;
    int local;
    if (BATCH) {
      const int ii = find_tma_inst(tab, ninst, t);
      in = &tab[ii];
      local = t - in->tile_base;
    } else {
      in = &one;
      local = t;
    }
    const int lit = it - in->it_begin;
    if (lit < 0 || lit >= in->n_steps) continue;
    tile_f32(*in, local, lit, sm, ring, &abort_flag);
    if (abort_flag) {
      if (threadIdx.x == 0 && in->flags) atomicOr(in->flags, 2);
      ring_drain<TmaF32::NST>(ring, (1 << TmaF32::NST) - 1);
      return;
    }
  }
}

template <bool BATCH>
__global__ void __launch_bounds__(256, 3)
    step_f64_tma(const __grid_constant__ TmaF64 one, const TmaF64* __restrict__ tab, int ninst,
                 int ntiles, int it) {
  extern __shared__ unsigned char smem_raw[];
  // 128-byte aligned header (mbarriers, abort flag) followed by the stages
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base);
  int& abort_flag = *reinterpret_cast<int*>(base + 64);
  double* sm = reinterpret_cast<double*>(base + 128);
  if ((smem_addr(sm) & 127u) != 0u) {  // never issue a TMA to a misaligned destination
    int* fl = BATCH ? (ninst > 0 ? tab[0].flags : nullptr) : one.flags;
    if (threadIdx.x == 0 && fl) atomicOr(fl, 4);
    return;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < TmaF64::NST; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    abort_flag = 0;
  }
  __syncthreads();
  Ring ring{bars, 0u};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const TmaF64* in;
    int local;
    if (BATCH) {
      const int ii = find_tma_inst(tab, ninst, t);
      in = &tab[ii];
      local = t - in->tile_base;
    } else {
      in = &one;
      local = t;
    }
    const int lit = it - in->it_begin;
    if (lit < 0 || lit >= in->n_steps) continue;
    tile_f64(*in, local, lit, sm, ring, &abort_flag);
    if (abort_flag) {
      if (threadIdx.x == 0 && in->flags) atomicOr(in->flags, 2);
      ring_drain<TmaF64::NST>(ring, (1 << TmaF64::NST) - 1);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// dynamic shared memory: alignment slack + header + stages
size_t tma_smem_bytes(int precision) {
  return precision == SW_PLAIN_F64 ? 256 + (size_t)TmaF64::NST * TmaF64::STAGE * sizeof(double)
                                   : 256 + (size_t)TmaF32::NST * TmaF32::STAGE * sizeof(float);
}

static int set_smem_attr(int precision) {
  static bool done[2] = {false, false};
  const int k = precision == SW_PLAIN_F64 ? 1 : 0;
  if (done[k]) return SW_OK;
  const int bytes = (int)tma_smem_bytes(precision);
  cudaError_t e;
  if (k) {
    e = cudaFuncSetAttribute(step_f64_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(step_f64_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               bytes);
  } else {
    e = cudaFuncSetAttribute(step_f32_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(step_f32_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               bytes);
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(step smem)");
  done[k] = true;
  return SW_OK;
}

int tma_xchunk(const Geom& g, int tz, int ty, long long want_tiles) {
  long long ntz = (g.nz + tz - 1) / tz, nty = (g.ny + ty - 1) / ty;
  long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0) return 1;
  long long cols = ntz * nty;
  long long nchunks = std::max(1LL, (want_tiles + cols - 1) / cols);
  long long xc = std::max(8LL, (nxi + nchunks - 1) / nchunks);
  return (int)std::min(xc, nxi);
}

int make_tma_f32(const StepArgs& a, int xchunk, TmaF32* t) {
  *t = TmaF32{};
  t->g = a.g;
  const int xc = xchunk > 0 ? xchunk : tma_xchunk(a.g, TmaF32::TZ, TmaF32::TY, 3 * 148);
  t->ts = make_tiles_t(a.g, xc, TmaF32::TZ, TmaF32::TY);
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 9};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 4, (uint64_t)a.g.sxy * 4,
                               (uint64_t)a.g.ncell * 4};
  const uint32_t box[4] = {TmaF32::W, TmaF32::H, 1, 6};
  for (int b = 0; b < 2; ++b) {
    t->state[b] = (float*)a.state[b];
    int rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                            box);
    if (rc != SW_OK) return rc;
  }
  t->m = (const float*)a.coef_m;
  t->e = (const float*)a.coef_e;
  t->pat = (const float*)a.patterns;
  t->term_off = a.term_off;
  t->term_pat = a.term_pat;
  t->term_scale = a.term_scale;
  t->hx = (float)a.ihx2;
  t->hy = (float)a.ihy2;
  t->hz = (float)a.ihz2;
  t->damp = (float)a.damp;
  t->use_damp = a.use_damp;
  t->kahan = a.kahan;
  t->n_steps = a.n_steps;
  t->snap_stride = a.snap_stride;
  t->snaps = (float*)a.snaps;
  t->flags = a.flags;
  t->it_begin = 0;
  t->tile_base = 0;
  return SW_OK;
}

int make_tma_f64(const StepArgs& a, int xchunk, TmaF64* t) {
  *t = TmaF64{};
  t->g = a.g;
  const int xc = xchunk > 0 ? xchunk : tma_xchunk(a.g, TmaF64::TZ, TmaF64::TY, 3 * 148);
  t->ts = make_tiles_t(a.g, xc, TmaF64::TZ, TmaF64::TY);
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 3};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 8, (uint64_t)a.g.sxy * 8,
                               (uint64_t)a.g.ncell * 8};
  const uint32_t box[4] = {TmaF64::W, TmaF64::H, 1, 3};
  for (int b = 0; b < 3; ++b) {
    t->state[b] = (double*)a.state[b];
    int rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, a.state[b], dims, strides,
                            box);
    if (rc != SW_OK) return rc;
  }
  t->m = (const double*)a.coef_m;
  t->e = (const double*)a.coef_e;
  t->ir = (const double*)a.inv_rho;
  t->pat = (const double*)a.patterns;
  t->term_off = a.term_off;
  t->term_pat = a.term_pat;
  t->term_scale = a.term_scale;
  t->ihx2 = a.ihx2;
  t->ihy2 = a.ihy2;
  t->ihz2 = a.ihz2;
  t->inv_dt = a.inv_dt;
  t->dt2 = a.dt2;
  t->damp = a.damp;
  t->use_damp = a.use_damp;
  t->n_steps = a.n_steps;
  t->snap_stride = a.snap_stride;
  t->snaps = (double*)a.snaps;
  t->flags = a.flags;
  t->it_begin = 0;
  t->tile_base = 0;
  return SW_OK;
}

int launch_steps_tma(const StepArgs& a, int xchunk, int it0, int nsteps, cudaStream_t s) {
  int rc = set_smem_attr(a.precision);
  if (rc != SW_OK) return rc;
  const size_t smem = tma_smem_bytes(a.precision);
  if (a.precision == SW_PLAIN_F64) {
    TmaF64 t;
    rc = make_tma_f64(a, xchunk, &t);
    if (rc != SW_OK) return rc;
    if (t.ts.count == 0) return SW_OK;
    const int grid = std::min(t.ts.count, 148 * 3);
    for (int it = it0; it < it0 + nsteps; ++it)
      step_f64_tma<false><<<grid, 256, smem, s>>>(t, nullptr, 1, t.ts.count, it);
  } else {
    TmaF32 t;
    rc = make_tma_f32(a, xchunk, &t);
    if (rc != SW_OK) return rc;
    if (t.ts.count == 0) return SW_OK;
    const int grid = std::min(t.ts.count, 148 * 3);
    for (int it = it0; it < it0 + nsteps; ++it)
      step_f32_tma<false><<<grid, 256, smem, s>>>(t, nullptr, 1, t.ts.count, it);
  }
  count_launches((unsigned long long)nsteps);
  SW_CHECK_LAUNCH("step (tma)");
  return SW_OK;
}

int launch_steps_tma_batch(int precision, const void* d_tab, int ninst, int ntiles, int it,
                           cudaStream_t s) {
  int rc = set_smem_attr(precision);
  if (rc != SW_OK) return rc;
  if (ntiles == 0) return SW_OK;
  const size_t smem = tma_smem_bytes(precision);
  const int grid = std::min(ntiles, 148 * 3);
  if (precision == SW_PLAIN_F64) {
    TmaF64 dummy{};
    step_f64_tma<true><<<grid, 256, smem, s>>>(dummy, (const TmaF64*)d_tab, ninst, ntiles, it);
  } else {
    TmaF32 dummy{};
    step_f32_tma<true><<<grid, 256, smem, s>>>(dummy, (const TmaF32*)d_tab, ninst, ntiles, it);
  }
  count_launches(1);
  SW_CHECK_LAUNCH("step (tma, batch)");
  return SW_OK;
}

}  // namespace sw
