// Mixed-form step kernel that advances two time steps per pass over HBM.
//
// Same per-cell update as the one-step kernels (src/shearwave/solver.py:
// 195-226 in increment form with a compensated displacement), applied twice:
//
//   level 0  the state at step t, streamed by TMA: u and d of a plane with two
//            cells of halo around the 62 x 6 output tile (one 72 x 10 x 1 x 6
//            box per plane, 6-stage ring: three planes in use, three in
//            flight), and the point-wise data of the 64 x 8 level-1 region
//            (Kahan c, material coefficients; 4-stage ring);
//   level 1  step t+1 on the 64 x 8 region (the output tile plus one cell of
//            halo), written to a 4-slot shared-memory ring of planes;
//   level 2  step t+2 on the output tile, read from the level-1 ring and
//            written to global memory.
//
// The CTA marches along x: when level-0 plane q+1 lands, level 1 computes
// plane q and level 2 plane q-1.  Level-1 cells outside the grid interior
// are the zero shell.  Each consumer thread owns the same two columns at
// both levels, so the level-1 Kahan compensation and the material
// coefficients carry over in registers.  One named barrier per plane (with
// an or-reduction of the failure flag, so an abort is decided by all
// consumers together) separates the level-1 writes from the level-2 reads;
// four level-1 slots make a second barrier unnecessary.  A step reads the
// state in buffer t mod 3 and writes buffer (t+2) mod 3.
//
// Per output cell and pair of steps the kernel moves about 78 bytes of DRAM
// traffic (u, d, c in and out, coefficients once) instead of 160 for two
// one-step passes.
#include <math.h>

#include <algorithm>

#include "sw_common.cuh"
#include "sw_step.cuh"
#include "sw_step_tma.cuh"
#include "sw_tma.cuh"

namespace sw {

namespace {

struct TbCoord {
  int z_start, y_start, x0, x1;
};

__host__ __device__ inline TileSpace make_tiles_tb(const Geom& g, int xc) {
  TileSpace t;
  const int nzi = g.nz > 2 ? g.nz - 2 : 0, nyi = g.ny > 2 ? g.ny - 2 : 0;
  const int nxi = g.nx > 2 ? g.nx - 2 : 0;
  t.ntz = (nzi + TmaF32TB::OZ - 1) / TmaF32TB::OZ;
  t.nty = (nyi + TmaF32TB::OY - 1) / TmaF32TB::OY;
  t.xc = xc < 1 ? 1 : xc;
  t.nxc = nxi > 0 ? (nxi + t.xc - 1) / t.xc : 0;
  t.count = t.ntz * t.nty * t.nxc;
  return t;
}

__device__ inline TbCoord tb_coord(const Geom& g, const TileSpace& t, int local) {
  TbCoord c;
  const int zt = local % t.ntz;
  const int rest = local / t.ntz;
  const int yt = rest % t.nty;
  const int xt = rest / t.nty;
  c.z_start = 1 + TmaF32TB::OZ * zt;
  c.y_start = 1 + TmaF32TB::OY * yt;
  c.x0 = 1 + xt * t.xc;
  c.x1 = min(c.x0 + t.xc, g.nx - 1);
  return c;
}

__device__ inline int floor4(int v) { return v & ~3; }  // floor to a multiple of 4 (v >= -4)

template <bool BATCH>
__global__ void __launch_bounds__(TmaF32TB::THREADS, 1)
    step_f32_fused2(const __grid_constant__ TmaF32TB one, const TmaF32TB* __restrict__ tab,
                    int ninst, int ntiles, int it, const int* __restrict__ it_dev,
                    int* /*queues: unused; keeps the step kernels' parameters alike*/) {
  if (it_dev != nullptr) it += *it_dev;  // step counter kept on the device (graph replays)
  using T = TmaF32TB;
  constexpr int NA = T::NA, NB = T::NB, NL = T::NL, W = T::W, H = T::H, WB = T::WB, HB = T::HB;
  constexpr int LZ = T::LZ, LY = T::LY, NC = T::CONSUMER_WARPS * 32;
  constexpr int AF = T::A_STAGE / 4, BF = T::B_STAGE / 4, LF = T::L_STAGE / 4;
  constexpr int CF = round128(T::C_BYTES) / 4;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  WsHeader* hd = reinterpret_cast<WsHeader*>(base);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(base + kAbortFlagOffset);
  float* ringA = reinterpret_cast<float*>(base + kRingOffset);
  float* ringB = ringA + NA * AF;
  float* ringL = ringB + NB * BF;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((smem_addr(ringA) & 127u) != 0u) {
    int* fl = BATCH ? (ninst > 0 ? tab[0].flags : nullptr) : one.flags;
    if (threadIdx.x == 0 && fl) atomicOr(fl, 4);
    return;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < NA; ++s) {
      mbar_init(&hd->fullA[s], 1);
      mbar_init(&hd->emptyA[s], T::CONSUMER_WARPS);
    }
    for (int s = 0; s < NB; ++s) {
      mbar_init(&hd->fullB[s], 1);
      mbar_init(&hd->emptyB[s], T::CONSUMER_WARPS);
    }
    *abort_flag = 0;
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == T::CONSUMER_WARPS) {
    // ------------------------------- producer -----------------------------
    if (lane == 0) {
      uint32_t pa = 0, pb = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        const T* in;
        int local, lit;
        if (!resolve_tile<T, BATCH>(one, tab, ninst, t, it, in, local, lit)) continue;
        const Geom& g = in->g;
        const TbCoord tc = tb_coord(g, in->ts, local);
        const int zA0 = floor4(tc.z_start - 2), zB0 = floor4(tc.z_start - 1);
        const CUtensorMap* tma = &in->tm[lit % 3];
        const CUtensorMap* tmc = &in->tmc[lit % 3];
        const uint32_t bbytes = (in->kahan ? T::C_BYTES : 0) + WB * HB * 4 * in->ncoef;
        bool ok = true;
        auto issueA = [&](int p) {
          const int sa = pa % NA;
          ok = ok && ws_wait(&hd->emptyA[sa], ((pa / NA) & 1u) ^ 1u, abort_flag);
          if (!ok) return;
          const int pl = min(max(p, 0), g.nx - 1);  // planes outside the grid are never read
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&hd->fullA[sa], T::A_BYTES);
          tma_load_4d(ringA + sa * AF, tma, &hd->fullA[sa], zA0, tc.y_start - 2, pl, 0);
          ++pa;
        };
        auto issueB = [&](int q) {
          const int sb = pb % NB;
          ok = ok && ws_wait(&hd->emptyB[sb], ((pb / NB) & 1u) ^ 1u, abort_flag);
          if (!ok) return;
          const int ql = min(max(q, 0), g.nx - 1);
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&hd->fullB[sb], bbytes);
          if (in->kahan) tma_load_4d(ringB + sb * BF, tmc, &hd->fullB[sb], zB0, tc.y_start - 1, ql, 6);
          tma_load_4d(ringB + sb * BF + CF, &in->tmm, &hd->fullB[sb], zB0, tc.y_start - 1, ql, 0);
          ++pb;
        };
        issueA(tc.x0 - 2);
        issueA(tc.x0 - 1);
        for (int q = tc.x0 - 1; q <= tc.x1 && ok; ++q) {
          issueA(q + 1);
          issueB(q);
        }
        if (!ok) break;
      }
    }
  } else {
    // ------------------------------- consumers ----------------------------
    const int w = warp;
    uint32_t ca = 0, cb = 0, lcount = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
      const T* in;
      int local, lit;
      if (!resolve_tile<T, BATCH>(one, tab, ninst, t, it, in, local, lit)) continue;
      const Geom& g = in->g;  // hot switches in registers (see step_f32_tma)
      const TbCoord tc = tb_coord(g, in->ts, local);
      const bool use_damp = in->use_damp != 0;
      const float damp = in->damp;
      const int zA0 = floor4(tc.z_start - 2), zB0 = floor4(tc.z_start - 1);
      const int offA = tc.z_start - 1 - zA0;  // level-1 column 0 in the level-0 box
      const int offB = tc.z_start - 1 - zB0;  // level-1 column 0 in the point box
      float* __restrict__ D = in->state[(lit + 2) % 3];
      const long long nc = g.ncell;
      const int y = tc.y_start - 1 + w;  // this warp's level-1 row
      const bool yin = (y >= 1 && y <= g.ny - 2);
      int zc[2];
      bool inyz[2], own[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int c = lane + 32 * k;
        zc[k] = tc.z_start - 1 + c;
        inyz[k] = yin && zc[k] >= 1 && zc[k] <= g.nz - 2;
        own[k] = inyz[k] && w >= 1 && w <= T::OY && c >= 1 && c <= T::OZ;
      }
      const int ja0 = in->term_off ? in->term_off[lit] : 0;
      const int ja1 = in->term_off ? in->term_off[lit + 1] : 0;
      const int jb0 = in->term_off ? in->term_off[lit + 1] : 0;
      const int jb1 = in->term_off ? in->term_off[lit + 2] : 0;
      const bool snap1 =
          in->snap_stride > 0 && in->snaps != nullptr && ((lit + 1) % in->snap_stride) == 0;
      const bool snap2 =
          in->snap_stride > 0 && in->snaps != nullptr && ((lit + 2) % in->snap_stride) == 0;
      const int slot1 = snap1 ? (lit + 1) / in->snap_stride - 1 : 0;
      const int slot2 = snap2 ? (lit + 2) / in->snap_stride - 1 : 0;
      const bool visc = in->ncoef > 1, kahan = in->kahan != 0;
      const float hx = in->hx, hy = in->hy, hz = in->hz, hc = lap7_centre_coef(hx, hy, hz);
      float mp[2] = {0.f, 0.f}, ep[2] = {0.f, 0.f}, cp[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
      bool ok = true;
      int s_prev = ca % NA;
      ok = ok && ws_wait(&hd->fullA[s_prev], (ca / NA) & 1u, abort_flag);
      ++ca;
      int s_cur = ca % NA;
      ok = ok && ws_wait(&hd->fullA[s_cur], (ca / NA) & 1u, abort_flag);
      ++ca;
      for (int q = tc.x0 - 1; q <= tc.x1; ++q) {
        const int s_next = ca % NA;
        ok = ok && ws_wait(&hd->fullA[s_next], (ca / NA) & 1u, abort_flag);
        ++ca;
        const int sb = cb % NB;
        ok = ok && ws_wait(&hd->fullB[sb], (cb / NB) & 1u, abort_flag);
        ++cb;
        // ---- level 1: step lit+1 at plane q on the 64 x 8 region ----
        float* Lw = ringL + (lcount % NL) * LF;
        float mc[2] = {0.f, 0.f}, ec[2] = {0.f, 0.f}, cc[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        if (ok) {
          const float* Pp = ringA + s_prev * AF;
          const float* Pc = ringA + s_cur * AF;
          const float* Pn = ringA + s_next * AF;
          const float* Bc = ringB + sb * BF;
          const float* Bm = Bc + CF;
          const bool qin = (q >= 1 && q <= g.nx - 2);
          bool bad = false;
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int c = lane + 32 * k;
            const int ob = w * WB + c + offB;
            mc[k] = Bm[ob];
            ec[k] = visc ? Bm[HB * WB + ob] : 0.0f;
            const bool act = qin && inyz[k];
            const long long i = (long long)q * g.sxy + (long long)y * g.pz + zc[k];
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
              float unew = 0.f, inc = 0.f, cnew = 0.f;
              if (act) {
                const int o = (comp * H + w + 1) * W + c + offA;
                const int od = o + 3 * H * W;
                const float u0 = Pc[o], d0 = Pc[od];
                const float lu = lap7f(Pn[o] + Pp[o], Pc[o + W] + Pc[o - W],
                                       Pc[o + 1] + Pc[o - 1], u0, hx, hy, hz, hc);
                inc = d0 + mc[k] * lu;
                if (visc) {
                  const float ld = lap7f(Pn[od] + Pp[od], Pc[od + W] + Pc[od - W],
                                         Pc[od + 1] + Pc[od - 1], d0, hx, hy, hz, hc);
                  inc += ec[k] * ld;
                }
                for (int j = ja0; j < ja1; ++j)
                  inc += in->pat[((long long)in->term_pat[j] * 3 + comp) * nc + i] *
                         (float)in->term_scale[j];
                if (use_damp) inc *= damp;
                if (kahan) {
                  const float c0 = Bc[comp * HB * WB + ob];
                  const float yk = inc - c0;
                  unew = u0 + yk;
                  cnew = (unew - u0) - yk;
                } else {
                  unew = u0 + inc;
                }
                bad |= !isfinite(unew);
                if (snap1 && own[k] && q >= tc.x0 && q < tc.x1)
                  in->snaps[((((long long)slot1 * g.nx + q) * g.ny + y) * g.nz + zc[k]) * 3 +
                            comp] = unew;
              }
              Lw[(comp * LY + w) * LZ + c] = unew;
              Lw[((3 + comp) * LY + w) * LZ + c] = inc;
              cc[k][comp] = cnew;
            }
          }
          if (bad && in->flags) atomicOr(in->flags, 1);
        }
        __syncwarp();
        if (lane == 0 && ok) {
          mbar_arrive(&hd->emptyA[s_prev]);  // level-0 plane q-1 is no longer needed
          mbar_arrive(&hd->emptyB[sb]);
        }
        ++lcount;
        if (consumer_sync_or(!ok, NC)) {  // level-1 plane q visible to all consumers
          failed = true;
          break;
        }
        // ---- level 2: step lit+2 at plane x = q-1 on the output tile ----
        const int x = q - 1;
        if (x >= tc.x0) {
          const float* Lp = ringL + ((lcount - 3) % NL) * LF;
          const float* Lc = ringL + ((lcount - 2) % NL) * LF;
          const float* Ln = ringL + ((lcount - 1) % NL) * LF;
          bool bad = false;
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            if (!own[k]) continue;
            const int c = lane + 32 * k;
            const long long i = (long long)x * g.sxy + (long long)y * g.pz + zc[k];
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
              const int o = (comp * LY + w) * LZ + c;
              const int od = o + 3 * LY * LZ;
              const float u0 = Lc[o], d0 = Lc[od];
              const float lu = lap7f(Ln[o] + Lp[o], Lc[o + LZ] + Lc[o - LZ],
                                     Lc[o + 1] + Lc[o - 1], u0, hx, hy, hz, hc);
              float inc = d0 + mp[k] * lu;
              if (visc) {
                const float ld = lap7f(Ln[od] + Lp[od], Lc[od + LZ] + Lc[od - LZ],
                                       Lc[od + 1] + Lc[od - 1], d0, hx, hy, hz, hc);
                inc += ep[k] * ld;
              }
              for (int j = jb0; j < jb1; ++j)
                inc += in->pat[((long long)in->term_pat[j] * 3 + comp) * nc + i] *
                       (float)in->term_scale[j];
              if (use_damp) inc *= damp;
              float unew;
              if (kahan) {
                const float yk = inc - cp[k][comp];
                unew = u0 + yk;
                D[(6 + comp) * nc + i] = (unew - u0) - yk;
              } else {
                unew = u0 + inc;  // compensation planes unused
              }
              D[comp * nc + i] = unew;
              D[(3 + comp) * nc + i] = inc;
              bad |= !isfinite(unew);
              if (snap2)
                in->snaps[((((long long)slot2 * g.nx + x) * g.ny + y) * g.nz + zc[k]) * 3 +
                          comp] = unew;
            }
          }
          if (bad && in->flags) atomicOr(in->flags, 1);
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          mp[k] = mc[k];
          ep[k] = ec[k];
#pragma unroll
          for (int comp = 0; comp < 3; ++comp) cp[k][comp] = cc[k][comp];
        }
        s_prev = s_cur;
        s_cur = s_next;
      }
      if (failed) break;
      __syncwarp();
      if (lane == 0) {  // level-0 planes x1 and x1+1
        mbar_arrive(&hd->emptyA[s_prev]);
        mbar_arrive(&hd->emptyA[s_cur]);
      }
    }
  }
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) {
    int* fl = BATCH ? (ninst > 0 ? tab[0].flags : nullptr) : one.flags;
    if (fl) atomicOr(fl, 2);
    const long long t0 = clock64();
    while (clock64() - t0 < 200000000LL) {
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t tb_smem_bytes() {
  return 128 + 256 + (size_t)TmaF32TB::NA * TmaF32TB::A_STAGE +
         (size_t)TmaF32TB::NB * TmaF32TB::B_STAGE + (size_t)TmaF32TB::NL * TmaF32TB::L_STAGE;
}

static int tb_set_attr() {
  static bool done = false;
  if (done) return SW_OK;
  const int bytes = (int)tb_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(step_f32_fused2<false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(step_f32_fused2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
  if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(fused step smem)");
  done = true;
  return SW_OK;
}

// planes per x chunk: minimise waves x (level-1 planes per tile) on 148 SMs
static int tb_xchunk(const Geom& g) {
  const long long nzi = g.nz > 2 ? g.nz - 2 : 0, nyi = g.ny > 2 ? g.ny - 2 : 0;
  const long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0 || nzi == 0 || nyi == 0) return 1;
  const long long cols = ((nzi + TmaF32TB::OZ - 1) / TmaF32TB::OZ) *
                         ((nyi + TmaF32TB::OY - 1) / TmaF32TB::OY);
  const long long slots = 148;
  long long best_nc = 1, best = -1;
  for (long long nc = 1; nc <= nxi; ++nc) {
    const long long xc = (nxi + nc - 1) / nc;
    const long long nch = (nxi + xc - 1) / xc;
    const long long cost = ((cols * nch + slots - 1) / slots) * (xc + 2);
    if (best < 0 || cost < best) {
      best = cost;
      best_nc = nc;
    }
  }
  return (int)((nxi + best_nc - 1) / best_nc);
}

int make_tma_f32_tb(const StepArgs& a, int xchunk, TmaF32TB* t) {
  *t = TmaF32TB{};
  t->g = a.g;
  t->ts = make_tiles_tb(a.g, xchunk > 0 ? xchunk : tb_xchunk(a.g));
  if (a.coef_e == nullptr) {
    t->ncoef = 1;
  } else if ((const char*)a.coef_e == (const char*)a.coef_m + a.g.ncell * 4) {
    t->ncoef = 2;
  } else {
    set_error("the fused step kernel needs coef_e == coef_m + ncell");
    return SW_EINVAL;
  }
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 9};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 4, (uint64_t)a.g.sxy * 4,
                               (uint64_t)a.g.ncell * 4};
  const uint32_t boxA[4] = {TmaF32TB::W, TmaF32TB::H, 1, 6};
  const uint32_t boxC[4] = {TmaF32TB::WB, TmaF32TB::HB, 1, 3};
  for (int b = 0; b < 3; ++b) {
    t->state[b] = (float*)a.state[b];
    int rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                            boxA);
    if (rc == SW_OK)
      rc = encode_tmap_4d(&t->tmc[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                          boxC);
    if (rc != SW_OK) return rc;
  }
  const uint64_t mdims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx,
                             (uint64_t)t->ncoef};
  const uint32_t boxM[4] = {TmaF32TB::WB, TmaF32TB::HB, 1, (uint32_t)t->ncoef};
  int rc = encode_tmap_4d(&t->tmm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (void*)a.coef_m, mdims,
                          strides, boxM);
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
  return SW_OK;
}

int launch_fused2_prepare() { return tb_set_attr(); }

const void* step_f32_fused2_ptr() { return reinterpret_cast<const void*>(step_f32_fused2<false>); }

void launch_fused2_raw(const TmaF32TB& t, int it, cudaStream_t s) {
  if (t.ts.count == 0) return;
  step_f32_fused2<false><<<std::min(t.ts.count, 148), TmaF32TB::THREADS, tb_smem_bytes(), s>>>(
      t, nullptr, 1, t.ts.count, it, nullptr, nullptr);
}

int launch_fused2(const StepArgs& a, int xchunk, int it, cudaStream_t s) {
  int rc = tb_set_attr();
  if (rc != SW_OK) return rc;
  TmaF32TB t;
  rc = make_tma_f32_tb(a, xchunk, &t);
  if (rc != SW_OK) return rc;
  if (t.ts.count == 0) return SW_OK;
  const int grid = std::min(t.ts.count, 148);
  step_f32_fused2<false><<<grid, TmaF32TB::THREADS, tb_smem_bytes(), s>>>(
      t, nullptr, 1, t.ts.count, it, nullptr, nullptr);
  count_launches(1);
  SW_CHECK_LAUNCH("fused two-step kernel");
  return SW_OK;
}

int launch_fused2_batch(const void* d_tab, int ninst, int ntiles, int it, cudaStream_t s) {
  int rc = tb_set_attr();
  if (rc != SW_OK) return rc;
  if (ntiles == 0) return SW_OK;
  TmaF32TB dummy{};
  step_f32_fused2<true><<<std::min(ntiles, 148), TmaF32TB::THREADS, tb_smem_bytes(), s>>>(
      dummy, (const TmaF32TB*)d_tab, ninst, ntiles, it, nullptr, nullptr);
  count_launches(1);
  SW_CHECK_LAUNCH("fused two-step kernel (batch)");
  return SW_OK;
}

}  // namespace sw
