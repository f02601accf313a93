// TMA-staged fused step kernels (the production time-loop kernels).
//
// Same arithmetic as the reference update (src/shearwave/solver.py:195-226)
// and as the direct-load kernels in sw_step.cu, reorganised for B200:
//
//  * A CTA owns a TZ x TY tile of the (z, y) plane and marches along x over a
//    chunk of planes.  For every plane it needs the halo'd fields (u and d in
//    the mixed form, u_prev and u_curr in the plain form) at x-1, x, x+1.
//  * One elected thread streams planes into a shared-memory ring with 4-D
//    TMA tile loads (all halo'd components of a plane in one box, or two
//    boxes for the two FP64 buffers), completion on one mbarrier per stage.
//    The x neighbours at x-1 come from registers (each thread keeps the centre
//    values of the plane it computed last), so a stage is freed as soon as
//    its plane is computed: the ring holds planes x and x+1 while the next
//    planes are in flight.
//  * The box starts 4 (FP32) / 2 (FP64) cells before the tile in z so the
//    innermost coordinate stays 16-byte aligned; y starts one row before.
//    Out-of-range rows/columns are zero-filled by TMA.
//  * Point-wise inputs (material coefficients, Kahan compensation) come by
//    TMA too: in the mixed kernel into the stage of their plane, in the FP64
//    kernel into a second ring.  Force patterns (push steps only) are read
//    straight from global memory, coalesced along z; outputs are written
//    with coalesced stores.
// Every mbarrier wait is bounded; a timeout sets bit 1 of the solve's flag
// word and the CTA drains its outstanding copies (bounded) and returns.
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <vector>

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
// pipeline helpers
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// mixed FP32 step: warp-specialised TMA pipeline
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 lds2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ float2 ldg2(const float* p) {
  return __ldg(reinterpret_cast<const float2*>(p));
}
__device__ __forceinline__ void stg2(float* p, float a, float b) {
  *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

// One plane of the mixed step for one thread's cell pair (z, z+1) of row y:
// 8-byte shared-memory loads and global stores serve both cells.  `o` is the
// pair's u component-0 index in the halo box, `ob` its index in the point
// boxes, `Di` its cell in the output buffer.  The arithmetic per cell is the
// same expression as in the direct kernel (sw_step.cu), so the results agree
// bit for bit.  Cells outside the interior (z = 0, z >= nz-1) get 0, which is
// what the shell and padding hold in every state buffer.  Non-finite values
// are detected once, in the finish kernel.  The switches are template
// arguments, fixed per tile: viscosity, compensated sum, damping, and whether
// this step adds force terms.
template <bool VISC, bool KAHAN, bool DAMP, bool PUSH, int HW>
__device__ __forceinline__ void f32_pair_plane(
    const float* __restrict__ Pc, const float* __restrict__ Pn, const float* __restrict__ Bc,
    const float* __restrict__ Bm, int o, int ob, int W, float2 (&pu)[3], float2 (&pd)[3],
    bool act_a, bool act_b, const Lap7Pair& lk, float damp,
    const TmaF32* __restrict__ in, int j0, int j1, unsigned nc, long long i,
    float* __restrict__ Di, float2 (&un)[3]) {
  // HW: halo-box cells per component; a point box holds PT cells per component
  constexpr int PT = TmaF32::PT;
  const float2 M = lds2(Bm + ob);
  const float2 E = VISC ? lds2(Bm + PT + ob) : make_float2(0.f, 0.f);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int oc = o + c * HW, od = oc + 3 * HW;
    const float2 C = lds2(Pc + oc), L = lds2(Pc + oc - 2), R = lds2(Pc + oc + 2);
    const float2 N = lds2(Pc + oc + W), S = lds2(Pc + oc - W), X = lds2(Pn + oc);
    const float2 lu = lap7_pair(C, L, R, X, pu[c], N, S, lk);
    const float2 Cd = lds2(Pc + od);
    float2 inc = ffma2(M, lu, Cd);
    if (VISC) {
      const float2 Ld = lds2(Pc + od - 2), Rd = lds2(Pc + od + 2);
      const float2 Nd = lds2(Pc + od + W), Sd = lds2(Pc + od - W), Xd = lds2(Pn + od);
      inc = ffma2(E, lap7_pair(Cd, Ld, Rd, Xd, pd[c], Nd, Sd, lk), inc);
      pd[c] = Cd;
    }
    pu[c] = C;
    if (PUSH) {
      for (int j = j0; j < j1; ++j) {
        const float2 P = ldg2(in->pat + ((long long)in->term_pat[j] * 3 + c) * nc + i);
        inc = ffma2(P, splat2((float)in->term_scale[j]), inc);
      }
    }
    if (DAMP) inc = fmul2(inc, splat2(damp));
    float2 un2;
    if (KAHAN) {
      const float2 K = lds2(Bc + c * PT + ob);
      const float2 yk = fsub2(inc, K);
      un2 = fadd2(C, yk);
      const float2 cn = fsub2(fsub2(un2, C), yk);
      stg2(Di + (size_t)(6 + c) * nc, act_a ? cn.x : 0.f, act_b ? cn.y : 0.f);
    } else {
      un2 = fadd2(C, inc);  // the compensation planes are neither read nor written
    }
    const float ua = act_a ? un2.x : 0.f, ub = act_b ? un2.y : 0.f;
    stg2(Di + (size_t)c * nc, ua, ub);
    stg2(Di + (size_t)(3 + c) * nc, act_a ? inc.x : 0.f, act_b ? inc.y : 0.f);
    un[c] = make_float2(ua, ub);
  }
}

// Rings of the mixed step kernel.  Ring A has NA stages of one plane's halo'd
// u and d; ring B has NB stages of one plane's point-wise inputs (the
// compensation planes when the ring has room for them (KR), then the
// material coefficients).  Without the compensation planes ring A gets a
// fifth stage (three planes in flight instead of two).  One ring with both
// in each stage was measured slower (more DRAM traffic, 15 % longer steps).
template <bool KR>
struct F32Ring {
  static_assert(TmaF32::MIN_CTAS == 2, "rings sized for two resident CTAs per SM");
  static constexpr int NA = KR ? 4 : 5, NB = 3;
  static constexpr int STAGE = round128(TmaF32::A_BYTES_MAX);                 // ring A stage
  static constexpr int C_OFF = 0;                                             // in a B stage
  static constexpr int M_OFF = C_OFF + (KR ? round128(TmaF32::C_BYTES) : 0);  // coefficients
  static constexpr int B_STAGE = M_OFF + round128(TmaF32::M_BYTES);
  static constexpr size_t SMEM = 128 + kRingOffset + (size_t)NA * STAGE + (size_t)NB * B_STAGE;
};
static_assert(F32Ring<false>::SMEM <= F32Ring<true>::SMEM, "the compact ring must not be larger");
static_assert(2 * (F32Ring<true>::SMEM + 1024) <= 233472, "two CTAs must fit one SM");

// Consumer side of the rings: where they live and the next stage of each.
template <bool KR>
struct F32Consumer {
  float* ring;  // ring A, then ring B
  WsHeader* hd;
  volatile int* abort_flag;
  RingPos<F32Ring<KR>::NA> a;  // next plane
  RingPos<F32Ring<KR>::NB> b;  // next point-wise plane
  __device__ const float* stage_a(int s) const { return ring + s * (F32Ring<KR>::STAGE / 4); }
  __device__ const float* stage_b(int s) const {
    return ring + F32Ring<KR>::NA * (F32Ring<KR>::STAGE / 4) + s * (F32Ring<KR>::B_STAGE / 4);
  }
};

// One tile of the consumer warps: plane x0-1 (centres only), then planes
// x0..x1-1, each waited for, computed and released; the closing halo plane
// x1 is released last.  On entry q.a is the stage of plane x0-1, whose full
// barrier the caller has waited on.  Returns false when a wait gave up.
template <int TZW, bool KR, bool VISC, bool KAHAN, bool DAMP, bool PUSH>
__device__ __forceinline__ bool f32_tile(const TmaF32* __restrict__ in, int local, int lit,
                                         F32Consumer<KR>& q, int warp, int lane) {
  constexpr int TYH = TmaF32::TZ * TmaF32::TY / TZW;
  constexpr int CF = F32Ring<KR>::C_OFF / 4, MF = F32Ring<KR>::M_OFF / 4;
  constexpr int HWB = TmaF32::box_cells(TZW);  // halo-box cells per component
  constexpr int Wb = TZW + 8;                  // halo box row length
  const Geom& g = in->g;
  const TileCoord tc = tile_coord_t(g, in->ts, local, TZW, TYH);
  float* __restrict__ D = in->state[(lit + 1) % 3];
  // this thread's cells: the pair z, z+1 of tile row `row`; a warp covers
  // one row of 32 pairs (64 x 8 tiles) or two rows of 16 (32 x 16 tiles)
  const int row = TZW == 64 ? warp : 2 * warp + (lane >> 4);
  const int lz = TZW == 64 ? 2 * lane : 2 * (lane & 15);
  const int y = tc.y0 + row;
  const bool yin = (y >= 1 && y <= g.ny - 2);
  const int z = tc.z0 + lz;
  const bool inrow = yin && z < g.pz;  // pz is even: the whole pair is in the row
  const bool act_a = yin && z >= 1 && z <= g.nz - 2;
  const bool act_b = yin && z + 1 >= 1 && z + 1 <= g.nz - 2;
  const int j0 = PUSH ? in->term_off[lit] : 0;
  const int j1 = PUSH ? in->term_off[lit + 1] : 0;
  const bool snap =
      in->snap_stride > 0 && in->snaps != nullptr && ((lit + 1) % in->snap_stride) == 0;
  const int slot = snap ? (lit + 1) / in->snap_stride - 1 : 0;
  const unsigned nc = (unsigned)g.ncell;  // the host keeps ncell below 2^32
  const float damp = in->damp;
  const Lap7Pair lk =
      lap7_pair_coefs(in->hx, in->hy, in->hz, lap7_centre_coef(in->hx, in->hy, in->hz));
  const int o = (row + 1) * Wb + lz + 4, ob = row * TZW + lz;
  // Plane x-1 enters only through its centre values (x neighbours of the
  // Laplacians), which each thread keeps in registers from the plane it
  // computed last; so a plane's stage is released as soon as the plane is
  // computed, and the ring holds planes x and x+1 with the rest in flight.
  float2 pu[3], pd[3];  // u and d of plane x-1 at this thread's cells
  {
    const float* P0 = q.stage_a(q.a.s);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      pu[c] = lds2(P0 + o + c * HWB);
      pd[c] = VISC ? lds2(P0 + o + (3 + c) * HWB) : make_float2(0.f, 0.f);
    }
  }
  __syncwarp();
  if (lane == 0) mbar_arrive(&q.hd->emptyA[q.a.s]);
  q.a.next();
  int s_cur = q.a.s;
  if (!ws_wait(&q.hd->fullA[s_cur], q.a.ph, q.abort_flag)) return false;
  q.a.next();
  long long i = (long long)tc.x0 * g.sxy + (long long)y * g.pz + z;
  for (int x = tc.x0; x < tc.x1; ++x, i += g.sxy) {
    const int s_next = q.a.s, sb = q.b.s;
    if (!ws_wait(&q.hd->fullA[s_next], q.a.ph, q.abort_flag)) return false;
    q.a.next();
    if (!ws_wait(&q.hd->fullB[sb], q.b.ph, q.abort_flag)) return false;
    q.b.next();
    if (inrow) {
      const float* Bs = q.stage_b(sb);
      float2 un[3];
      f32_pair_plane<VISC, KAHAN, DAMP, PUSH, HWB>(q.stage_a(s_cur), q.stage_a(s_next), Bs + CF,
                                                   Bs + MF, o, ob, Wb, pu, pd, act_a, act_b, lk,
                                                   damp, in, j0, j1, nc, i, D + i, un);
      if (snap) {
        float* sp = in->snaps + ((((long long)slot * g.nx + x) * g.ny + y) * g.nz + z) * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (act_a) sp[c] = un[c].x;
          if (act_b) sp[3 + c] = un[c].y;
        }
      }
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&q.hd->emptyA[s_cur]);  // plane x is done
      mbar_arrive(&q.hd->emptyB[sb]);
    }
    s_cur = s_next;
  }
  __syncwarp();
  if (lane == 0) mbar_arrive(&q.hd->emptyA[s_cur]);  // the closing halo plane x1
  return true;
}

// The tile's switches, resolved once per tile into a specialised plane loop
// (runtime branches in the plane loop cost about 15 % of its instructions).
template <int TZW, bool KR, bool VISC, bool DAMP, bool PUSH>
__device__ __forceinline__ bool f32_tile_k(bool kahan, const TmaF32* __restrict__ in, int local,
                                           int lit, F32Consumer<KR>& q, int warp, int lane) {
  if constexpr (KR) {
    if (kahan) return f32_tile<TZW, KR, VISC, true, DAMP, PUSH>(in, local, lit, q, warp, lane);
  }
  return f32_tile<TZW, KR, VISC, false, DAMP, PUSH>(in, local, lit, q, warp, lane);
}

template <int TZW, bool KR, bool VISC, bool DAMP>
__device__ __forceinline__ bool f32_tile_p(bool push, bool kahan, const TmaF32* __restrict__ in,
                                           int local, int lit, F32Consumer<KR>& q, int warp,
                                           int lane) {
  if (push) return f32_tile_k<TZW, KR, VISC, DAMP, true>(kahan, in, local, lit, q, warp, lane);
  return f32_tile_k<TZW, KR, VISC, DAMP, false>(kahan, in, local, lit, q, warp, lane);
}

template <int TZW, bool KR>
__device__ __forceinline__ bool f32_tile_any(const TmaF32* __restrict__ in, int local, int lit,
                                             F32Consumer<KR>& q, int warp, int lane) {
  const bool visc = in->ncoef > 1, damp = in->use_damp != 0, kahan = KR && in->kahan != 0;
  const bool push = in->term_off != nullptr && in->term_off[lit + 1] > in->term_off[lit];
  if (visc) {
    if (damp) return f32_tile_p<TZW, KR, true, true>(push, kahan, in, local, lit, q, warp, lane);
    return f32_tile_p<TZW, KR, true, false>(push, kahan, in, local, lit, q, warp, lane);
  }
  if (damp) return f32_tile_p<TZW, KR, false, true>(push, kahan, in, local, lit, q, warp, lane);
  return f32_tile_p<TZW, KR, false, false>(push, kahan, in, local, lit, q, warp, lane);
}

template <bool BATCH, int TZW, bool KR>
__global__ void __launch_bounds__(TmaF32::THREADS, TmaF32::MIN_CTAS)
    step_f32_tma(const __grid_constant__ TmaF32 one, const TmaF32* __restrict__ tab, int ninst,
                 int ntiles, int it, const int* __restrict__ it_dev, int* queues) {
  // tile shape: TZW x TYH cells (64 x 8, or 32 x 16); every solve of a
  // launch uses the launch's shape
  constexpr int TYH = TmaF32::TZ * TmaF32::TY / TZW;
  static_assert(TZW == 64 || TZW == 32, "tile widths 64 and 32");
  if (it_dev != nullptr) it += *it_dev;  // step counter kept on the device (graph replays)
  // with a queue, CTAs take tiles from it (the last CTA to finish resets it
  // for the next launch); without, tiles go in a fixed stride
  int* queue = queues;
  constexpr int NA = F32Ring<KR>::NA, NB = F32Ring<KR>::NB;
  constexpr int HWB = TmaF32::box_cells(TZW);           // halo-box cells per component
  constexpr uint32_t A_BYTES = (uint32_t)HWB * 6 * 4;  // one plane's u and d
  constexpr int TZ = TmaF32::TZ, TY = TmaF32::TY;
  constexpr int SF = F32Ring<KR>::STAGE / 4, SFB = F32Ring<KR>::B_STAGE / 4;  // floats
  constexpr int CF = F32Ring<KR>::C_OFF / 4, MF = F32Ring<KR>::M_OFF / 4;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  WsHeader* hd = reinterpret_cast<WsHeader*>(base);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(base + kAbortFlagOffset);
  float* ring = reinterpret_cast<float*>(base + kRingOffset);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto flags_of = [&](int k) -> int* { return BATCH ? tab[k].flags : one.flags; };
  if ((smem_addr(ring) & 127u) != 0u) {  // never issue a TMA to a misaligned destination
    if (threadIdx.x == 0)
      for (int k = 0; k < (BATCH ? ninst : 1); ++k)
        if (int* fl = flags_of(k)) atomicOr(fl, kFlagRefused);
    queue_cta_done(queue);
    return;
  }
  AbortLog* lg = abort_log(base);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NA; ++s) {
      mbar_init(&hd->fullA[s], 1);
      mbar_init(&hd->emptyA[s], TmaF32::CONSUMER_WARPS);
    }
    for (int s = 0; s < NB; ++s) {
      mbar_init(&hd->fullB[s], 1);
      mbar_init(&hd->emptyB[s], TmaF32::CONSUMER_WARPS);
    }
    *abort_flag = 0;
    abort_flag[1] = BATCH ? (ninst > 0 ? tab[0].wait_k : 1) : one.wait_k;
    lg->n_taken = 0;
    lg->armedA = lg->parA = lg->armedB = lg->parB = 0;
    for (int w = 0; w < 16; ++w) lg->done[w] = 0;
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == TmaF32::CONSUMER_WARPS) {
    // ------------------------------- producer -----------------------------
    if (lane == 0) {
      RingPos<NA> pa;  // next stage of ring A / ring B to load
      RingPos<NB> pb;
      int stride_next = blockIdx.x;
      while (!*abort_flag) {
        const int t = next_tile(queue, stride_next);
        if (t >= ntiles) {  // end of this CTA's work: arm one stage without a copy
          if (!ws_wait(&hd->emptyA[pa.s], pa.ph ^ 1u, abort_flag)) break;
          tile_slots(base)[pa.s] = -1;
          mbar_arrive(&hd->fullA[pa.s]);
          pa.next();
          break;
        }
        const int k = BATCH ? find_solve(tab, ninst, t) : 0;
        const TmaF32* in = BATCH ? &tab[k] : &one;
        const int local = BATCH ? t - in->tile_base : t;
        const int lit = it - in->it_begin;
        if (lit < 0 || lit >= in->n_steps || solve_abandoned(in->flags)) continue;
        lg->solve[lg->n_taken & 7] = k;
        ++lg->n_taken;
        const TileCoord tc = tile_coord_t(in->g, in->ts, local, TZW, TYH);
        const CUtensorMap* tma = &in->tm[lit % 3];
        const CUtensorMap* tmc = &in->tmc[lit % 3];
        const bool kahan = KR && in->kahan;  // the compact ring never carries c
        const uint32_t pbytes = (kahan ? TmaF32::C_BYTES : 0) + TZ * TY * 4 * in->ncoef;
        for (int p = tc.x0 - 1; p <= tc.x1 && !*abort_flag; ++p) {
          const int sa = pa.s;
          if (!ws_wait(&hd->emptyA[sa], pa.ph ^ 1u, abort_flag)) break;
          // the testing switch leaves the tile's first stage unarmed
          if (!(p == tc.x0 - 1 && in->stall_test)) {
            if (p == tc.x0 - 1) {
              tile_slots(base)[sa] = t;
              solve_slots(base)[sa] = k;
            }
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&hd->fullA[sa], A_BYTES);
            tma_load_4d(ring + sa * SF, tma, &hd->fullA[sa], tc.z0 - 4, tc.y0 - 1, p, 0);
            arm_record(lg->armedA, lg->parA, sa, pa.ph);
          }
          pa.next();
          if (p >= tc.x0 && p < tc.x1) {  // planes x0..x1-1 also need their point-wise inputs
            const int sb = pb.s;
            if (!ws_wait(&hd->emptyB[sb], pb.ph ^ 1u, abort_flag)) break;
            float* sbp = ring + NA * SF + sb * SFB;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&hd->fullB[sb], pbytes);
            if (kahan) tma_load_4d(sbp + CF, tmc, &hd->fullB[sb], tc.z0, tc.y0, p, 6);
            tma_load_4d(sbp + MF, &in->tmm, &hd->fullB[sb], tc.z0, tc.y0, p, 0);
            arm_record(lg->armedB, lg->parB, sb, pb.ph);
            pb.next();
          }
        }
      }
    }
  } else {
    // ------------------------------- consumers ----------------------------
    F32Consumer<KR> q{ring, hd, abort_flag};
    while (true) {
      // the tile's first plane (its halo plane x0-1)
      if (!ws_wait(&hd->fullA[q.a.s], q.a.ph, abort_flag)) break;
      const int t = tile_slots(base)[q.a.s];
      if (t < 0) break;
      const TmaF32* in = BATCH ? &tab[solve_slots(base)[q.a.s]] : &one;
      const int local = BATCH ? t - in->tile_base : t;
      const int lit = it - in->it_begin;
      if (!f32_tile_any<TZW, KR>(in, local, lit, q, warp, lane)) break;
      if (lane == 0) ++lg->done[warp];
    }
  }
  __syncthreads();
  if (*abort_flag && warp == TmaF32::CONSUMER_WARPS && lane == 0) {
    // let every copy still in flight land, then flag the abandoned tiles' solves
    drain_ring(hd->fullA, lg->armedA, lg->parA, NA);
    drain_ring(hd->fullB, lg->armedB, lg->parB, NB);
    flag_unfinished(lg, TmaF32::CONSUMER_WARPS, BATCH ? ninst : 1, kFlagTimeout, flags_of);
  }
  queue_cta_done(queue);
}

// ---------------------------------------------------------------------------
// plain FP64 step: warp-specialised TMA pipeline
// ---------------------------------------------------------------------------
template <bool BATCH>
__global__ void __launch_bounds__(TmaF64::THREADS, 2)
    step_f64_tma(const __grid_constant__ TmaF64 one, const TmaF64* __restrict__ tab, int ninst,
                 int ntiles, int it, const int* __restrict__ it_dev, int* queues) {
  if (it_dev != nullptr) it += *it_dev;  // step counter kept on the device (graph replays)
  int* queue = queues;  // see step_f32_tma
  constexpr int NA = TmaF64::NA, NB = TmaF64::NB, W = TmaF64::W, H = TmaF64::H;
  constexpr int TZ = TmaF64::TZ, TY = TmaF64::TY;
  constexpr int AD = TmaF64::A_STAGE / 8, BD = TmaF64::B_STAGE / 8, HALF = TmaF64::HALF / 8;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  WsHeader* hd = reinterpret_cast<WsHeader*>(base);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(base + kAbortFlagOffset);
  double* ringA = reinterpret_cast<double*>(base + kRingOffset);
  double* ringB = ringA + NA * AD;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto flags_of = [&](int k) -> int* { return BATCH ? tab[k].flags : one.flags; };
  if ((smem_addr(ringA) & 127u) != 0u) {
    if (threadIdx.x == 0)
      for (int k = 0; k < (BATCH ? ninst : 1); ++k)
        if (int* fl = flags_of(k)) atomicOr(fl, kFlagRefused);
    queue_cta_done(queue);
    return;
  }
  AbortLog* lg = abort_log(base);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NA; ++s) {
      mbar_init(&hd->fullA[s], 1);
      mbar_init(&hd->emptyA[s], TmaF64::CONSUMER_WARPS);
    }
    for (int s = 0; s < NB; ++s) {
      mbar_init(&hd->fullB[s], 1);
      mbar_init(&hd->emptyB[s], TmaF64::CONSUMER_WARPS);
    }
    *abort_flag = 0;
    abort_flag[1] = BATCH ? (ninst > 0 ? tab[0].wait_k : 1) : one.wait_k;
    lg->n_taken = 0;
    lg->armedA = lg->parA = lg->armedB = lg->parB = 0;
    for (int w = 0; w < 16; ++w) lg->done[w] = 0;
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == TmaF64::CONSUMER_WARPS) {
    if (lane == 0) {
      RingPos<NA> pa;
      RingPos<NB> pb;
      int stride_next = blockIdx.x;
      while (!*abort_flag) {
        const int t = next_tile(queue, stride_next);
        if (t >= ntiles) {  // end of this CTA's work: arm one stage without a copy
          if (!ws_wait(&hd->emptyA[pa.s], pa.ph ^ 1u, abort_flag)) break;
          tile_slots(base)[pa.s] = -1;
          mbar_arrive(&hd->fullA[pa.s]);
          pa.next();
          break;
        }
        const int k = BATCH ? find_solve(tab, ninst, t) : 0;
        const TmaF64* in = BATCH ? &tab[k] : &one;
        const int local = BATCH ? t - in->tile_base : t;
        const int lit = it - in->it_begin;
        if (lit < 0 || lit >= in->n_steps || solve_abandoned(in->flags)) continue;
        lg->solve[lg->n_taken & 7] = k;
        ++lg->n_taken;
        const TileCoord tc = tile_coord_t(in->g, in->ts, local, TZ, TY);
        const CUtensorMap* tmp = &in->tm[lit % 3];
        const CUtensorMap* tmc = &in->tm[(lit + 1) % 3];
        const uint32_t bbytes = TZ * TY * 8 * in->ncoef;
        for (int p = tc.x0 - 1; p <= tc.x1 && !*abort_flag; ++p) {
          const int sa = pa.s;
          if (!ws_wait(&hd->emptyA[sa], pa.ph ^ 1u, abort_flag)) break;
          // the testing switch leaves the tile's first stage unarmed
          if (!(p == tc.x0 - 1 && in->stall_test)) {
            if (p == tc.x0 - 1) {
              tile_slots(base)[sa] = t;
              solve_slots(base)[sa] = k;
            }
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&hd->fullA[sa], 2 * TmaF64::BOX_BYTES);
            tma_load_4d(ringA + sa * AD, tmp, &hd->fullA[sa], tc.z0 - 2, tc.y0 - 1, p, 0);
            tma_load_4d(ringA + sa * AD + HALF, tmc, &hd->fullA[sa], tc.z0 - 2, tc.y0 - 1, p,
                        0);
            arm_record(lg->armedA, lg->parA, sa, pa.ph);
          }
          pa.next();
          if (p >= tc.x0 && p < tc.x1) {
            const int sb = pb.s;
            if (!ws_wait(&hd->emptyB[sb], pb.ph ^ 1u, abort_flag)) break;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&hd->fullB[sb], bbytes);
            tma_load_4d(ringB + sb * BD, &in->tmm, &hd->fullB[sb], tc.z0, tc.y0, p, 0);
            arm_record(lg->armedB, lg->parB, sb, pb.ph);
            pb.next();
          }
        }
      }
    }
  } else {
    const int ly = warp;
    RingPos<NA> ca;
    RingPos<NB> cb;
    while (true) {
      int s_cur = ca.s;  // the tile's first plane (its halo plane x0-1)
      if (!ws_wait(&hd->fullA[s_cur], ca.ph, abort_flag)) break;
      const int t = tile_slots(base)[s_cur];
      if (t < 0) break;
      const TmaF64* in = BATCH ? &tab[solve_slots(base)[s_cur]] : &one;
      const int local = BATCH ? t - in->tile_base : t;
      const int lit = it - in->it_begin;
      const Geom& g = in->g;  // hot switches in registers (see step_f32_tma)
      const TileCoord tc = tile_coord_t(g, in->ts, local, TZ, TY);
      double* __restrict__ un = in->state[(lit + 2) % 3];
      const bool use_damp = in->use_damp != 0;
      const double dt2 = in->dt2, damp = in->damp;
      const int y = tc.y0 + ly, z = tc.z0 + lane;
      const bool act = (y >= 1 && y <= g.ny - 2 && z >= 1 && z <= g.nz - 2);
      const int j0 = in->term_off ? in->term_off[lit] : 0;
      const int j1 = in->term_off ? in->term_off[lit + 1] : 0;
      const bool snap =
          in->snap_stride > 0 && in->snaps != nullptr && ((lit + 1) % in->snap_stride) == 0;
      const int slot = snap ? (lit + 1) / in->snap_stride - 1 : 0;
      const long long nc = g.ncell;
      const bool visc = in->ncoef > 1;
      const double ihx2 = in->ihx2, ihy2 = in->ihy2, ihz2 = in->ihz2, inv_dt = in->inv_dt;
      // plane x-1 enters through its centre values only, kept in registers
      // (u_curr and u_prev per component), so a plane's stage is released as
      // soon as the plane is computed (see step_f32_tma)
      double qc[3], qp[3];
      bool ok = true;
      ca.next();  // plane x0-1 (waited for above): centres only
      {
        const double* P0 = ringA + s_cur * AD;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int op = (c * H + ly + 1) * W + lane + 2;
          qp[c] = P0[op];
          qc[c] = P0[op + HALF];
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&hd->emptyA[s_cur]);
      s_cur = ca.s;
      ok &= ws_wait(&hd->fullA[s_cur], ca.ph, abort_flag);
      ca.next();
      long long i = (long long)tc.x0 * g.sxy + (long long)y * g.pz + z;
      for (int x = tc.x0; x < tc.x1 && ok; ++x, i += g.sxy) {
        const int s_next = ca.s;
        ok &= ws_wait(&hd->fullA[s_next], ca.ph, abort_flag);
        ca.next();
        const int sb = cb.s;
        ok &= ws_wait(&hd->fullB[sb], cb.ph, abort_flag);
        cb.next();
        if (!ok) break;
        const double* Pc = ringA + s_cur * AD;
        const double* Pn = ringA + s_next * AD;
        if (act) {
          const double* Bm = ringB + sb * BD;
          const double m = Bm[ly * TZ + lane];
          const double e = visc ? Bm[(TY + ly) * TZ + lane] : 0.0;
          const double rinv = (j1 > j0) ? in->ir[i] : 0.0;
          bool bad = false;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int op = (c * H + ly + 1) * W + lane + 2;  // u_prev component c
            const int oc = op + HALF;                        // u_curr component c
            const double ucc = Pc[oc];
            const double lap_u = ((Pn[oc] - 2.0 * ucc) + qc[c]) * ihx2 +
                                 ((Pc[oc + W] - 2.0 * ucc) + Pc[oc - W]) * ihy2 +
                                 ((Pc[oc + 1] - 2.0 * ucc) + Pc[oc - 1]) * ihz2;
            double f = 0.0;
            for (int j = j0; j < j1; ++j) {
              const double fj =
                  in->pat[((long long)in->term_pat[j] * 3 + c) * nc + i] * in->term_scale[j];
              f = (j == j0) ? fj : f + fj;
            }
            double acc = m * lap_u + f * rinv;
            const double upc = Pc[op];
            if (visc) {
              const double vc = (ucc - upc) * inv_dt;
              const double lap_v =
                  (((Pn[oc] - Pn[op]) * inv_dt - 2.0 * vc) + (qc[c] - qp[c]) * inv_dt) * ihx2 +
                  (((Pc[oc + W] - Pc[op + W]) * inv_dt - 2.0 * vc) +
                   (Pc[oc - W] - Pc[op - W]) * inv_dt) *
                      ihy2 +
                  (((Pc[oc + 1] - Pc[op + 1]) * inv_dt - 2.0 * vc) +
                   (Pc[oc - 1] - Pc[op - 1]) * inv_dt) *
                      ihz2;
              acc += e * lap_v;
            }
            qc[c] = ucc;
            qp[c] = upc;
            double unew = (2.0 * ucc - upc) + dt2 * acc;
            if (use_damp) unew = ucc + damp * (unew - ucc);
            un[c * nc + i] = unew;
            bad |= !isfinite(unew);
            if (snap)
              in->snaps[((((long long)slot * g.nx + x) * g.ny + y) * g.nz + z) * 3 + c] = unew;
          }
          if (bad && in->flags) atomicOr(in->flags, 1);
        } else {  // keep the centres for the next plane
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const int op = (c * H + ly + 1) * W + lane + 2;
            qp[c] = Pc[op];
            qc[c] = Pc[op + HALF];
          }
        }
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&hd->emptyA[s_cur]);  // plane x is done
          mbar_arrive(&hd->emptyB[sb]);
        }
        s_cur = s_next;
      }
      if (!ok) break;
      __syncwarp();
      if (lane == 0) mbar_arrive(&hd->emptyA[s_cur]);  // the closing halo plane x1
      if (lane == 0) ++lg->done[warp];
    }
  }
  __syncthreads();
  if (*abort_flag && warp == TmaF64::CONSUMER_WARPS && lane == 0) {
    // let every copy still in flight land, then flag the abandoned tiles' solves
    drain_ring(hd->fullA, lg->armedA, lg->parA, NA);
    drain_ring(hd->fullB, lg->armedB, lg->parB, NB);
    flag_unfinished(lg, TmaF64::CONSUMER_WARPS, BATCH ? ninst : 1, kFlagTimeout, flags_of);
  }
  queue_cta_done(queue);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// dynamic shared memory: alignment slack + header + ring A + ring B
size_t tma_smem_bytes(int precision) {
  if (precision == SW_PLAIN_F64)
    return 128 + kRingOffset + (size_t)TmaF64::NA * TmaF64::A_STAGE + (size_t)TmaF64::NB * TmaF64::B_STAGE;
  return F32Ring<true>::SMEM;  // the larger of the two mixed layouts
}

// The mixed step kernel for a launch: batched or not, tile width, ring layout.
static const void* f32_kernel(bool batch, int tzw, bool kr) {
  if (batch) {
    if (tzw == 32) return kr ? (const void*)step_f32_tma<true, 32, true>
                             : (const void*)step_f32_tma<true, 32, false>;
    return kr ? (const void*)step_f32_tma<true, 64, true> : (const void*)step_f32_tma<true, 64, false>;
  }
  if (tzw == 32) return kr ? (const void*)step_f32_tma<false, 32, true>
                           : (const void*)step_f32_tma<false, 32, false>;
  return kr ? (const void*)step_f32_tma<false, 64, true> : (const void*)step_f32_tma<false, 64, false>;
}

static size_t f32_smem(bool kr) { return kr ? F32Ring<true>::SMEM : F32Ring<false>::SMEM; }

static void launch_f32(const void* fn, int grid, size_t smem, cudaStream_t s, const TmaF32& one,
                       const TmaF32* tab, int ninst, int ntiles, int it, int* queues) {
  const int* itd = nullptr;
  void* args[] = {(void*)&one, (void*)&tab, (void*)&ninst, (void*)&ntiles, (void*)&it,
                  (void*)&itd, (void*)&queues};
  cudaLaunchKernel(fn, dim3(grid), dim3(TmaF32::THREADS), args, smem, s);
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
    e = cudaSuccess;
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) {
      const bool kr = i & 1;
      e = cudaFuncSetAttribute(f32_kernel(i & 4, (i & 2) ? 32 : 64, kr),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)f32_smem(kr));
    }
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(step smem)");
  done[k] = true;
  return SW_OK;
}

// Planes per x chunk for a launch over one grid with `slots` resident CTAs:
// minimise (waves of tiles) x (planes a CTA loads per tile, including the
// two halo planes every chunk starts with).
int tma_xchunk(const Geom& g, int tz, int ty, long long slots) {
  const long long ntz = (g.nz + tz - 1) / tz, nty = (g.ny + ty - 1) / ty;
  const long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0) return 1;
  const long long cols = ntz * nty;
  long long best_nc = 1, best_cost = -1;
  for (long long nc = 1; nc <= nxi; ++nc) {
    const long long xc = (nxi + nc - 1) / nc;
    const long long nchunks = (nxi + xc - 1) / xc;
    const long long waves = (cols * nchunks + slots - 1) / slots;
    const long long cost = waves * (xc + 2);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best_nc = nc;
    }
  }
  return (int)((nxi + best_nc - 1) / best_nc);
}

// Planes per x chunk for a queue-fed launch over one grid: about
// SW_TUNE_BATCH_TILES_PER_CTA tiles per CTA slot, at least 8 planes, the
// interior split into equal chunks.
static int queue_xchunk(const Geom& g, int tz, int ty, long long slots) {
  const long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0) return 1;
  const long long cols = (long long)((g.nz + tz - 1) / tz) * ((g.ny + ty - 1) / ty);
  // when whole waves of equal chunks already fill >= 90 % of the slots, keep
  // them (fewer chunks, fewer re-read halo planes)
  const int xw = tma_xchunk(g, tz, ty, slots);
  const long long tiles = cols * ((nxi + xw - 1) / xw);
  const long long waves = (tiles + slots - 1) / slots;
  if (10 * tiles >= 9 * waves * slots) return xw;
  const long long want = (long long)tune_get(SW_TUNE_BATCH_TILES_PER_CTA) * slots;
  const long long xc = std::max<long long>(8, (cols * nxi + want - 1) / want);
  const long long nch = (nxi + xc - 1) / xc;
  return (int)((nxi + nch - 1) / nch);
}

// Material coefficients must be one allocation: component 0 = mu term,
// component 1 (optional) = eta term, ncell elements apart.
static int coef_components(const StepArgs& a, size_t es, int* ncoef) {
  if (a.coef_e == nullptr) {
    *ncoef = 1;
    return SW_OK;
  }
  if ((const char*)a.coef_e != (const char*)a.coef_m + a.g.ncell * es) {
    set_error("TMA step kernels need coef_e == coef_m + ncell (one 2-component allocation)");
    return SW_EINVAL;
  }
  *ncoef = 2;
  return SW_OK;
}

// Tile shape of the mixed step kernel for a grid: 64 x 8 or 32 x 16,
// whichever covers the (z, y) plane with fewer cells (ties: 64 x 8), unless
// the SW_TUNE_TILE_SHAPE knob forces one.
long long f32_tile_cover(const Geom& g, int tzw) {
  const int tyh = TmaF32::TZ * TmaF32::TY / tzw;
  return (long long)((g.nz + tzw - 1) / tzw) * tzw * (long long)((g.ny + tyh - 1) / tyh) * tyh;
}

int f32_tile_width(const Geom& g) {
  const int knob = tune_get(SW_TUNE_TILE_SHAPE);
  if (knob == 1) return 64;
  if (knob == 2) return 32;
  return f32_tile_cover(g, 32) < f32_tile_cover(g, 64) ? 32 : 64;
}

int make_tma_f32(const StepArgs& a, int xchunk, TmaF32* t, int tzw) {
  *t = TmaF32{};
  if (a.g.ncell >= (1LL << 32)) {  // the kernel offsets components by a 32-bit cell count
    set_error("grid too large for the TMA step kernel (%lld cells)", a.g.ncell);
    return SW_ERANGE;
  }
  t->g = a.g;
  t->tzw = tzw > 0 ? tzw : f32_tile_width(a.g);
  t->tyh = TmaF32::TZ * TmaF32::TY / t->tzw;
  const int xt = xchunk > 0 ? xchunk : tune_get(SW_TUNE_XCHUNK);
  const int xc = xt > 0 ? xt
                        : (a.queue ? queue_xchunk(a.g, t->tzw, t->tyh, step_slots())
                                   : tma_xchunk(a.g, t->tzw, t->tyh, step_slots()));
  t->ts = make_tiles_t(a.g, xc, t->tzw, t->tyh);
  int rc = coef_components(a, 4, &t->ncoef);
  if (rc != SW_OK) return rc;
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 9};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 4, (uint64_t)a.g.sxy * 4,
                               (uint64_t)a.g.ncell * 4};
  const uint32_t box_halo[4] = {(uint32_t)t->tzw + 8, (uint32_t)t->tyh + 2, 1, 6};
  const uint32_t box_pt[4] = {(uint32_t)t->tzw, (uint32_t)t->tyh, 1, 3};
  for (int b = 0; b < 3; ++b) {
    t->state[b] = (float*)a.state[b];
    rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                        box_halo);
    if (rc == SW_OK)
      rc = encode_tmap_4d(&t->tmc[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                          box_pt);
    if (rc != SW_OK) return rc;
  }
  const uint64_t mdims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx,
                             (uint64_t)t->ncoef};
  const uint32_t box_m[4] = {(uint32_t)t->tzw, (uint32_t)t->tyh, 1, (uint32_t)t->ncoef};
  rc = encode_tmap_4d(&t->tmm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (void*)a.coef_m, mdims, strides,
                      box_m);
  if (rc != SW_OK) return rc;
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
  t->wait_k = tune_get(SW_TUNE_WAIT_BUDGET);
  t->stall_test = a.stall_test;
  return SW_OK;
}

int make_tma_f64(const StepArgs& a, int xchunk, TmaF64* t) {
  *t = TmaF64{};
  t->g = a.g;
  const int xt = xchunk > 0 ? xchunk : tune_get(SW_TUNE_XCHUNK);
  const int xc = xt > 0 ? xt
                        : (a.queue ? queue_xchunk(a.g, TmaF64::TZ, TmaF64::TY, step_slots(false))
                                   : tma_xchunk(a.g, TmaF64::TZ, TmaF64::TY, step_slots(false)));
  t->ts = make_tiles_t(a.g, xc, TmaF64::TZ, TmaF64::TY);
  int rc = coef_components(a, 8, &t->ncoef);
  if (rc != SW_OK) return rc;
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 3};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 8, (uint64_t)a.g.sxy * 8,
                               (uint64_t)a.g.ncell * 8};
  const uint32_t box[4] = {TmaF64::W, TmaF64::H, 1, 3};
  for (int b = 0; b < 3; ++b) {
    t->state[b] = (double*)a.state[b];
    rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, a.state[b], dims, strides,
                        box);
    if (rc != SW_OK) return rc;
  }
  const uint64_t mdims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx,
                             (uint64_t)t->ncoef};
  const uint32_t box_m[4] = {TmaF64::TZ, TmaF64::TY, 1, (uint32_t)t->ncoef};
  rc = encode_tmap_4d(&t->tmm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (void*)a.coef_m, mdims, strides,
                      box_m);
  if (rc != SW_OK) return rc;
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
  t->wait_k = tune_get(SW_TUNE_WAIT_BUDGET);
  t->stall_test = a.stall_test;
  return SW_OK;
}

__global__ void clock_set(int* c, int v) { *c = v; }
__global__ void clock_add(int* c, int by) { *c += by; }

// Replay the step loop as one instantiated CUDA graph per segment: the graph
// holds `seg` launches of `func` (each advancing `per_launch` steps, offsets
// 0, per_launch, ...) reading the step counter `clock`, then a node that
// advances the counter.  Returns the number of steps enqueued this way (0
// when the run is too short to be worth a graph).  Kernel nodes are built
// explicitly, so the caller's stream may be the legacy default stream.  A
// batched launch passes its device table (`tab`, `ninst` solves, `ntiles`
// tiles; `t` unused); a lone solve passes `t` and tab = nullptr.
template <typename Inst>
int graph_loop(void* func, const Inst& t, int grid, int threads, size_t smem, int per_launch,
               int seg, int* clock, int* queue, int it0, int nsteps, cudaStream_t s, int* done,
               const Inst* tab = nullptr, int ninst = 1, int ntiles = -1) {
  *done = 0;
  const int seg_steps = per_launch * seg;
  const int reps = nsteps / seg_steps;
  if (reps < 2 || clock == nullptr) return SW_OK;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  cudaGraphNode_t prev = nullptr;
  if (ntiles < 0) ntiles = t.ts.count;
  const int* itd = clock;
  int* queues = queue;
  std::vector<int> offs(seg);
  for (int k = 0; k < seg && e == cudaSuccess; ++k) {
    offs[k] = k * per_launch;
    void* args[] = {(void*)&t,        (void*)&tab, (void*)&ninst, (void*)&ntiles,
                    (void*)&offs[k], (void*)&itd, (void*)&queues};
    cudaKernelNodeParams p{};
    p.func = func;
    p.gridDim = dim3(grid);
    p.blockDim = dim3(threads);
    p.sharedMemBytes = (unsigned)smem;
    p.kernelParams = args;
    cudaGraphNode_t node;
    e = cudaGraphAddKernelNode(&node, g, prev ? &prev : nullptr, prev ? 1 : 0, &p);
    prev = node;
  }
  int by = seg_steps;
  int* cl = clock;
  if (e == cudaSuccess) {
    void* args[] = {(void*)&cl, (void*)&by};
    cudaKernelNodeParams p{};
    p.func = (void*)clock_add;
    p.gridDim = dim3(1);
    p.blockDim = dim3(1);
    p.kernelParams = args;
    cudaGraphNode_t node;
    e = cudaGraphAddKernelNode(&node, g, &prev, 1, &p);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
  if (e == cudaSuccess) {
    clock_set<<<1, 1, 0, s>>>(clock, it0);
    e = cudaGetLastError();
  }
  for (int r = 0; r < reps && e == cudaSuccess; ++r) e = cudaGraphLaunch(ex, s);
  if (ex) cudaGraphExecDestroy(ex);  // freed once the enqueued replays complete
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_status(e, "step-loop graph");
  count_launches((unsigned long long)reps * (seg + 1) + 1, (unsigned long long)reps + 1);
  *done = reps * seg_steps;
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
    const int grid = std::min(t.ts.count, step_slots(false));
    int done = 0;
    rc = graph_loop(reinterpret_cast<void*>(step_f64_tma<false>), t, grid, TmaF64::THREADS, smem,
                    1, 32, a.clock, a.queue, it0, nsteps, s, &done);
    if (rc != SW_OK) return rc;
    for (int it = it0 + done; it < it0 + nsteps; ++it)
      step_f64_tma<false><<<grid, TmaF64::THREADS, smem, s>>>(t, nullptr, 1, t.ts.count, it,
                                                              nullptr, a.queue);
    count_launches((unsigned long long)(nsteps - done));
    SW_CHECK_LAUNCH("step (tma)");
    return SW_OK;
  } else {
    // two steps per pass: two steps per launch where two remain (one step
    // otherwise) unless the compensated sum is on (the default: 116 against
    // 93 Gcell-steps/s at 192^3).
    const bool fuse = steps_per_pass_of(a.steps_per_pass, false) == 2 && !a.kahan && nsteps >= 2;
    TmaF32 t;
    rc = make_tma_f32(a, xchunk, &t, 0);
    if (rc != SW_OK) return rc;
    if (t.ts.count == 0) return SW_OK;
    TmaF32TB tb;
    if (fuse) {
      rc = make_tma_f32_tb(a, 0, &tb, 0);
      if (rc != SW_OK) return rc;
      rc = launch_fused2_prepare();
      if (rc != SW_OK) return rc;
    }
    const int grid = std::min(t.ts.count, step_slots());
    unsigned long long n_launch = 0;
    int done = 0;
    if (fuse && tb.ts.count > 0)
      rc = graph_loop(const_cast<void*>(step_f32_fused2_ptr(tb.lz)), tb,
                      std::min(tb.ts.count, kNumSMs), TmaF32TB::THREADS, tb_smem_bytes(), 2, 16,
                      a.clock, a.queue, it0, nsteps, s, &done);
    else
      rc = graph_loop(const_cast<void*>(f32_kernel(false, t.tzw, t.kahan != 0)), t, grid,
                      TmaF32::THREADS, f32_smem(t.kahan != 0), 1, 32, a.clock, a.queue, it0,
                      nsteps, s, &done);
    if (rc != SW_OK) return rc;
    for (int it = it0 + done; it < it0 + nsteps;) {
      if (fuse && it + 1 < it0 + nsteps) {
        launch_fused2_raw(tb, it, s);
        it += 2;
      } else {
        launch_f32(f32_kernel(false, t.tzw, t.kahan != 0), grid, f32_smem(t.kahan != 0), s, t,
                   nullptr, 1, t.ts.count, it, a.queue);
        it += 1;
      }
      ++n_launch;
    }
    count_launches(n_launch);
    SW_CHECK_LAUNCH("step (tma)");
    return SW_OK;
  }
  count_launches((unsigned long long)nsteps);
  SW_CHECK_LAUNCH("step (tma)");
  return SW_OK;
}

int launch_steps_tma_batch(int precision, const void* d_tab, int ninst, int ntiles, int it,
                           int* queues, int tzw, bool kahan_ring, cudaStream_t s) {
  int rc = set_smem_attr(precision);
  if (rc != SW_OK) return rc;
  if (ntiles == 0) return SW_OK;
  const size_t smem = tma_smem_bytes(precision);
  const int grid = std::min(ntiles, step_slots(precision != SW_PLAIN_F64));
  if (precision == SW_PLAIN_F64) {
    TmaF64 dummy{};
    step_f64_tma<true><<<grid, TmaF64::THREADS, smem, s>>>(dummy, (const TmaF64*)d_tab, ninst,
                                                          ntiles, it, nullptr, queues);
  } else {
    TmaF32 dummy{};
    launch_f32(f32_kernel(true, tzw, kahan_ring), grid, f32_smem(kahan_ring), s, dummy,
               (const TmaF32*)d_tab, ninst, ntiles, it, queues);
  }
  count_launches(1);
  SW_CHECK_LAUNCH("step (tma, batch)");
  return SW_OK;
}

}  // namespace sw

// ---------------------------------------------------------------------------
// batched time loop: one launch per global step over every active solve
// ---------------------------------------------------------------------------
namespace sw {
namespace {

// Order in which the running solves enter a batched launch's tile range:
// solves with the longest x columns first, so that the launch-wide tile
// queue hands out the longest tiles first.
static std::vector<int> batch_order(const sw_fdtd_desc* descs, const std::vector<int>& run) {
  std::vector<int> ord(run);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](int a, int b) { return descs[a].nx > descs[b].nx; });
  return ord;
}

// Target planes per x chunk for a batched launch: about
// SW_TUNE_BATCH_TILES_PER_CTA (8) tiles per resident CTA over all running
// solves, at least 8 planes (each chunk re-reads two halo planes).
static int batch_xchunk(const sw_fdtd_desc* descs, const std::vector<int>& run, int tz, int ty,
                        bool mixed) {
  long long work = 0;
  for (int i : run) {
    const long long cols = (long long)((descs[i].nz + tz - 1) / tz) * ((descs[i].ny + ty - 1) / ty);
    work += cols * std::max(0, descs[i].nx - 2);
  }
  const long long want = (long long)tune_get(SW_TUNE_BATCH_TILES_PER_CTA) * step_slots(mixed);
  return (int)std::max<long long>(8, (work + want - 1) / want);
}

// A solve's chunk length for target `xc`: the interior planes split into
// equal chunks no longer than xc.  The solve's own xchunk, then the
// SW_TUNE_XCHUNK knob, when set, win.
static int solve_xchunk(const sw_fdtd_desc& d, int xc) {
  if (d.xchunk > 0) return d.xchunk;
  if (tune_get(SW_TUNE_XCHUNK) > 0) return tune_get(SW_TUNE_XCHUNK);
  const int nxi = std::max(1, d.nx - 2);
  const int nch = (nxi + xc - 1) / xc;
  return (nxi + nch - 1) / nch;
}

template <typename Inst>
int make_inst(const StepArgs& a, int xchunk, Inst* t, int shape);
template <>
int make_inst<TmaF32>(const StepArgs& a, int xchunk, TmaF32* t, int shape) {
  return make_tma_f32(a, xchunk, t, shape);
}
template <>
int make_inst<TmaF64>(const StepArgs& a, int xchunk, TmaF64* t, int) {
  return make_tma_f64(a, xchunk, t);
}

// Tile width shared by every solve of a batched mixed launch: the one that
// covers the running solves' planes with fewer cells (or the knob's).
static int batch_tile_width(const sw_fdtd_desc* descs, const std::vector<int>& run) {
  const int knob = tune_get(SW_TUNE_TILE_SHAPE);
  if (knob == 1) return 64;
  if (knob == 2) return 32;
  long long c64 = 0, c32 = 0;
  for (int i : run) {
    Geom g;
    g.nx = descs[i].nx;
    g.ny = descs[i].ny;
    g.nz = descs[i].nz;
    const long long nxi = std::max(0, descs[i].nx - 2) * (long long)descs[i].n_steps;
    c64 += f32_tile_cover(g, 64) * nxi;
    c32 += f32_tile_cover(g, 32) * nxi;
  }
  return c32 < c64 ? 32 : 64;
}

// Tile width of a batched two-step launch: 0 = each solve's own (the shape
// whose tiles compute fewer cells on its grid; on the config-3 batch 1.33
// computed cells per output cell against 1.38 for the best single shape), or
// the SW_TUNE_TILE_SHAPE knob's for all.
static int batch_tb_width() {
  const int knob = tune_get(SW_TUNE_TILE_SHAPE);
  if (knob == 1) return 64;
  if (knob == 2) return 32;
  return 0;
}

// Table of the solves running at step `it`, in batch_order, with their tile
// ranges laid end to end.
template <typename Inst>
int build_batch(const sw_fdtd_desc* descs, const int32_t* begins, int n, int it,
                std::vector<Inst>& tab, int* ntiles) {
  tab.clear();
  std::vector<int> run;
  for (int i = 0; i < n; ++i) {
    const int lit = it - (begins ? begins[i] : 0);
    if (lit >= 0 && lit < descs[i].n_steps) run.push_back(i);
  }
  const int shape = std::is_same<Inst, TmaF32>::value ? batch_tile_width(descs, run) : 0;
  const int xc = batch_xchunk(descs, run, Inst::TZ, Inst::TY, std::is_same<Inst, TmaF32>::value);
  int nt = 0;
  for (int i : batch_order(descs, run)) {
    StepArgs a;
    int rc = make_step_args(&descs[i], &a);
    if (rc != SW_OK) return rc;
    Inst t;
    rc = make_inst<Inst>(a, solve_xchunk(descs[i], xc), &t, shape);
    if (rc != SW_OK) return rc;
    t.it_begin = begins ? begins[i] : 0;
    t.tile_base = nt;
    nt += t.ts.count;
    tab.push_back(t);
  }
  *ntiles = nt;
  return SW_OK;
}

// A batch table starts with the launch-wide tile queue and its finish count
// (zeroed at the start of every call) and the step counter of graph
// replays; the solve arrays follow at kBatchHeader.
constexpr size_t kBatchHeader = 256;

// Mixed form: two steps per launch whenever every running solve runs both
// steps of the pair (unless a solve asks for one step per launch or for the
// compensated sum); one-step launches around starts and ends.  Two steps per
// pass are the default here: a batch keeps the GPU under its power cap long
// enough that the one-step kernel runs at about 1.55 GHz, while the two-step
// kernel, with 2.5x less DRAM traffic, keeps the full clock (48 solves of
// 64^3..160x160x224 cells: 99 against 91 Gcell-steps/s).  The table
// holds the one-step instance array, then the fused-kernel array.
int batch_steps_mixed(const sw_fdtd_desc* descs, const int32_t* begins, int n, int it0,
                      int nsteps, void* table, cudaStream_t s) {
  int* queues = (int*)table;
  char* tab_single = (char*)table + kBatchHeader;
  char* tab_fused = tab_single + (size_t)n * sizeof(TmaF32);
  cudaError_t e0 = cudaMemsetAsync(queues, 0, 4 * sizeof(int), s);
  if (e0 != cudaSuccess) return cuda_status(e0, "batch queue reset");
  bool fuse_ok = true;
  for (int i = 0; i < n; ++i)
    fuse_ok &= (steps_per_pass_of(descs[i].steps_per_pass, true) == 2 && !descs[i].kahan);
  auto active = [&](int i, int it) {
    const int lit = it - (begins ? begins[i] : 0);
    return lit >= 0 && lit < descs[i].n_steps;
  };
  std::vector<int> cur(n, -1);
  int cur_kind = -1;  // 0 single, 1 fused
  std::vector<TmaF32> tsingle;
  std::vector<TmaF32TB> tfused;
  int tb_lz = 64;  // tile width of the fused launches (per rebuild)
  int ntiles = 0;
  if (fuse_ok) {
    int rc = launch_fused2_prepare();
    if (rc != SW_OK) return rc;
  }
  const int end = it0 + nsteps;
  for (int it = it0; it < end;) {
    bool any = false, pair = fuse_ok && it + 1 < end;
    for (int i = 0; i < n; ++i) {
      const bool a0 = active(i, it);
      any |= a0;
      if (pair && a0 != active(i, it + 1)) pair = false;
    }
    if (!any) {
      ++it;
      continue;
    }
    const int kind = pair ? 1 : 0;
    bool rebuild = kind != cur_kind;
    for (int i = 0; i < n && !rebuild; ++i) rebuild = (cur[i] != (active(i, it) ? 1 : 0));
    if (rebuild) {
      tsingle.clear();
      tfused.clear();
      ntiles = 0;
      for (int i = 0; i < n; ++i) cur[i] = active(i, it) ? 1 : 0;
      if (kind == 1) {
        std::vector<int> run;
        for (int i = 0; i < n; ++i)
          if (cur[i]) run.push_back(i);
        tb_lz = batch_tb_width();
        for (int i : batch_order(descs, run)) {
          StepArgs a;
          int rc = make_step_args(&descs[i], &a);
          if (rc != SW_OK) return rc;
          TmaF32TB t;
          // planes per x chunk: the solve's own, else the SW_TUNE_XCHUNK knob,
          // else 32 (each chunk re-reads four halo planes of level 0)
          const int kx = tune_get(SW_TUNE_XCHUNK);
          rc = make_tma_f32_tb(a, descs[i].xchunk > 0 ? descs[i].xchunk : (kx > 0 ? kx : 32), &t,
                               tb_lz);
          if (rc != SW_OK) return rc;
          t.it_begin = begins ? begins[i] : 0;
          t.tile_base = ntiles;
          ntiles += t.ts.count;
          tfused.push_back(t);
        }
      } else {
        int rc = build_batch<TmaF32>(descs, begins, n, it, tsingle, &ntiles);
        if (rc != SW_OK) return rc;
      }
      const int urc = kind == 1 ? upload_staged(tab_fused, tfused.data(),
                                                tfused.size() * sizeof(TmaF32TB), s)
                                : upload_staged(tab_single, tsingle.data(),
                                                tsingle.size() * sizeof(TmaF32), s);
      if (urc != SW_OK) return urc;
      cur_kind = kind;
    }
    int rc;
    if (kind == 1) {
      // the steps from `it` on that keep this set of running solves (in
      // pairs): long runs replay one CUDA graph of 16 fused launches that
      // reads the step counter in the table header
      int stop = it;
      while (stop + 1 < end) {
        bool same = true;
        for (int i = 0; i < n && same; ++i)
          same = active(i, stop) == (cur[i] != 0) && active(i, stop + 1) == (cur[i] != 0);
        if (!same) break;
        stop += 2;
      }
      if (stop - it >= 64) {
        int done = 0;
        TmaF32TB dummy{};
        rc = graph_loop<TmaF32TB>(const_cast<void*>(step_f32_fused2_batch_ptr(tb_lz)), dummy,
                                  std::min(ntiles, kNumSMs), TmaF32TB::THREADS, tb_smem_bytes(),
                                  2, 16, queues + 2, queues, it, stop - it, s, &done,
                                  (const TmaF32TB*)tab_fused, (int)tfused.size(), ntiles);
        if (rc != SW_OK) return rc;
        if (done > 0) {
          it += done;
          continue;
        }
      }
      rc = launch_fused2_batch(tab_fused, (int)tfused.size(), ntiles, it, queues, tb_lz, s);
      it += 2;
    } else {
      bool kr = false;  // the compensation ring layout if any running solve needs it
      for (const TmaF32& t : tsingle) kr |= t.kahan != 0;
      rc = launch_steps_tma_batch(SW_MIXED_F32, tab_single, (int)tsingle.size(), ntiles, it,
                                  queues, tsingle.empty() ? 64 : tsingle[0].tzw, kr, s);
      it += 1;
    }
    if (rc != SW_OK) return rc;
  }
  return SW_OK;
}

template <typename Inst>
int batch_steps(int precision, const sw_fdtd_desc* descs, const int32_t* begins, int n, int it0,
                int nsteps, void* table_base, cudaStream_t s) {
  int* queues = (int*)table_base;
  char* table = (char*)table_base + kBatchHeader;
  cudaError_t e0 = cudaMemsetAsync(queues, 0, 2 * sizeof(int), s);
  if (e0 != cudaSuccess) return cuda_status(e0, "batch queue reset");
  std::vector<Inst> tab;
  std::vector<int> active(n, -1);
  int ntiles = 0;
  bool have = false;
  for (int it = it0; it < it0 + nsteps; ++it) {
    // rebuild the table only when the set of running solves changes
    bool changed = !have;
    for (int i = 0; i < n && !changed; ++i) {
      const int lit = it - (begins ? begins[i] : 0);
      const int act = (lit >= 0 && lit < descs[i].n_steps) ? 1 : 0;
      changed = (act != active[i]);
    }
    if (changed) {
      for (int i = 0; i < n; ++i) {
        const int lit = it - (begins ? begins[i] : 0);
        active[i] = (lit >= 0 && lit < descs[i].n_steps) ? 1 : 0;
      }
      int rc = build_batch<Inst>(descs, begins, n, it, tab, &ntiles);
      if (rc != SW_OK) return rc;
      if (!tab.empty()) {
        const int urc = upload_staged(table, tab.data(), tab.size() * sizeof(Inst), s);
        if (urc != SW_OK) return urc;
      }
      have = true;
    }
    if (tab.empty()) continue;
    if (std::is_same<Inst, TmaF64>::value) {
      // the steps from `it` on that keep this set of running solves replay
      // one CUDA graph of 32 launches reading the counter in the table header
      int stop = it;
      while (stop < it0 + nsteps) {
        bool same = true;
        for (int i = 0; i < n && same; ++i) {
          const int lit = stop - (begins ? begins[i] : 0);
          same = ((lit >= 0 && lit < descs[i].n_steps) ? 1 : 0) == active[i];
        }
        if (!same) break;
        ++stop;
      }
      if (stop - it >= 64) {
        int rc = set_smem_attr(precision);
        if (rc != SW_OK) return rc;
        int done = 0;
        TmaF64 dummy{};
        rc = graph_loop<TmaF64>(reinterpret_cast<void*>(step_f64_tma<true>), dummy,
                                std::min(ntiles, step_slots(false)), TmaF64::THREADS,
                                tma_smem_bytes(precision), 1, 32, queues + 2, queues, it,
                                stop - it, s, &done, (const TmaF64*)table, (int)tab.size(),
                                ntiles);
        if (rc != SW_OK) return rc;
        if (done > 0) {
          it += done - 1;  // the loop's ++it advances the last one
          continue;
        }
      }
    }
    int rc = launch_steps_tma_batch(precision, table, (int)tab.size(), ntiles, it, queues, 0,
                                    false, s);
    if (rc != SW_OK) return rc;
  }
  return SW_OK;
}

}  // namespace
}  // namespace sw

using namespace sw;

extern "C" size_t sw_fdtd_batch_table_bytes(int n) {
  if (n <= 0) return 0;
  return kBatchHeader + (size_t)n * std::max(sizeof(TmaF32) + sizeof(TmaF32TB), sizeof(TmaF64));
}

extern "C" int sw_fdtd_batch_steps(const sw_fdtd_desc* descs, const int32_t* begins, int n,
                                   int32_t it0, int32_t nsteps, void* table, size_t table_bytes,
                                   void* stream) {
  if (descs == nullptr || n <= 0 || table == nullptr || nsteps < 0) {
    set_error("sw_fdtd_batch_steps: bad arguments");
    return SW_EINVAL;
  }
  if (table_bytes < sw_fdtd_batch_table_bytes(n) || ((uintptr_t)table & 63u) != 0u) {
    set_error("sw_fdtd_batch_steps: table must be >= %zu bytes and 64-byte aligned",
              sw_fdtd_batch_table_bytes(n));
    return SW_EWORKSPACE;
  }
  const int prec = descs[0].precision;
  for (int i = 0; i < n; ++i) {
    if (descs[i].precision != prec || descs[i].kernel != 0 || descs[i].n_traces > 0) {
      set_error("sw_fdtd_batch_steps: solve %d differs in precision, asks for the direct "
                "kernels or records traces (unsupported in a batch)", i);
      return SW_EINVAL;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (prec == SW_PLAIN_F64)
    return batch_steps<TmaF64>(prec, descs, begins, n, it0, nsteps, table, s);
  return batch_steps_mixed(descs, begins, n, it0, nsteps, table, s);
}
