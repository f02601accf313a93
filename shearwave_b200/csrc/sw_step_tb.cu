// Mixed-form step kernel that advances two time steps per pass over HBM
// (the default of every mixed solve, batched or alone; runs without the
// compensated sum).
//
// Same per-cell update as the one-step kernels (src/shearwave/solver.py:
// 195-226 in increment form), applied twice in one pass.  For the 64-wide
// tile shape (TbShape<64>; the 32-wide shape has two rows of 16 pairs per
// warp and a 28 x 28 output tile):
//
//   level 0  the state at step t, streamed by TMA: u and d of a plane around
//            the 60 x 13 output tile (one 68 x 17 x 1 x 6 box per plane;
//            4-stage ring: planes q and q+1 held, two in flight) and the
//            material coefficients of the 64 x 15 level-1 region (2 stages);
//   level 1  step t+1 on the 64 x 15 region (the tile, one cell of halo, one
//            more column each side in z so z pairs stay aligned), written to
//            a 3-slot shared-memory ring of planes;
//   level 2  step t+2 on the output tile, read from the level-1 ring and
//            written to global memory.
//
// The CTA marches along x: when level-0 plane q+1 lands, level 1 computes
// plane q and level 2 plane q-1.  Fifteen consumer warps each own one
// level-1 row of 32 z pairs (8-byte shared loads and stores for both cells,
// packed .f32x2 arithmetic) and the same pairs at level 2, so the
// coefficients carry over in registers; the x neighbours at x-1 of both
// levels come from registers too (the centre values of the plane computed
// before), which frees a level-0 stage as soon as level 1 has used it.  The
// level-1 ring has a full and an empty mbarrier per slot (one arrival per
// warp): level 2 of plane q-1 waits until every warp has written plane q-1
// (it reads the rows above and below), and level 1 reuses a slot once every
// warp has read it, so warps drift up to a plane apart instead of meeting at
// a barrier; every wait is bounded and an abort stops each warp on its own.
// Level-1 cells outside the grid interior are the zero shell.  Both levels
// use lap7_pair, so two steps here equal two one-step launches bit for bit.
// A pass reads buffer t mod 3 and writes buffer (t+2) mod 3.  Batched
// launches give each solve its own tile shape; the force terms of push
// tiles come from a shared-memory term buffer the producer fills.
//
// It moves about 30 bytes of DRAM traffic per cell-step (u, d in and out
// once per two steps, coefficients once per two steps, halos), against 66
// for one-step launches.
#include <math.h>

#include <algorithm>

#include "sw_common.cuh"
#include "sw_step.cuh"
#include "sw_step_tma.cuh"
#include "sw_tma.cuh"

namespace sw {

namespace {

struct TbCoord {
  int z0, y0, x0, x1;  // output tile: z in [z0, z0+OZ), y in [y0, y0+OY), x in [x0, x1)
};

__host__ __device__ inline TileSpace make_tiles_tb(const Geom& g, int xc, int lz) {
  const int oz = lz == 32 ? TbShape<32>::OZ : TbShape<64>::OZ;
  const int oy = lz == 32 ? TbShape<32>::OY : TbShape<64>::OY;
  TileSpace t;
  // tiles [oz k, oz k + oz) and [oy k, oy k + oy) cover the interior 1..n-2
  t.ntz = g.nz > 2 ? (g.nz - 2) / oz + 1 : 0;
  t.nty = g.ny > 2 ? (g.ny - 2) / oy + 1 : 0;
  const int nxi = g.nx > 2 ? g.nx - 2 : 0;
  t.xc = xc < 1 ? 1 : xc;
  t.nxc = nxi > 0 ? (nxi + t.xc - 1) / t.xc : 0;
  t.count = t.ntz * t.nty * t.nxc;
  return t;
}

// Shape constants the producer needs per tile when a launch mixes shapes:
// the output tile, and the bytes of a level-0 box and cells of a point box.
struct TbDims {
  int oz, oy;
  uint32_t a_bytes, b_cells;
};
template <int LZ>
__device__ constexpr TbDims tb_dims() {
  using S = TbShape<LZ>;
  return TbDims{S::OZ, S::OY, (uint32_t)(S::W * S::H * 6 * 4), (uint32_t)(S::WB * S::HB)};
}

__device__ inline TbCoord tb_coord_rt(const Geom& g, const TileSpace& t, int local, int oz,
                                      int oy) {
  TbCoord c;
  const int zt = local % t.ntz;
  const int rest = local / t.ntz;
  const int yt = rest % t.nty;
  const int xt = rest / t.nty;
  c.z0 = oz * zt;
  c.y0 = oy * yt;
  c.x0 = 1 + xt * t.xc;
  c.x1 = min(c.x0 + t.xc, g.nx - 1);
  return c;
}

template <int OZ, int OY>
__device__ inline TbCoord tb_coord(const Geom& g, const TileSpace& t, int local) {
  TbCoord c;
  const int zt = local % t.ntz;
  const int rest = local / t.ntz;
  const int yt = rest % t.nty;
  const int xt = rest / t.nty;
  c.z0 = OZ * zt;
  c.y0 = OY * yt;
  c.x0 = 1 + xt * t.xc;
  c.x1 = min(c.x0 + t.xc, g.nx - 1);
  return c;
}

__device__ __forceinline__ float2 tb_ld2(const float* p) {
  return *reinterpret_cast<const float2*>(p);
}
__device__ __forceinline__ void tb_st2(float* p, float a, float b) {
  *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

// The force terms of a push tile's two steps, written by the producer when
// it takes the tile and read by the consumers: each term's pattern (its
// component 0) and scale, for step lit (level 1) and lit+1 (level 2).  Two
// buffers, by the parity of the tile's ordinal in the CTA: the producer
// fills the one of tile n+2 only after every consumer warp has released a
// plane of tile n+1 (a tile spans at least NA planes), so no warp still
// reads it.  A pair of steps with more than kTbTermCap terms at one step
// runs in one-step launches instead (the solver keeps such solves out of
// this kernel; the producer refuses the tile if one gets here).
constexpr int kTbTermCap = 32;
struct TbTermRef {
  const float* base;
  float scale;
  int pad;
};
struct TbTermBuf {
  int n[2];
  int pad[2];
  TbTermRef t[2][kTbTermCap];
};

// One level of the two-step pass for one thread's z pair: the step from the
// plane whose centre pair is at `P + o` (row stride `RS`, component stride
// `CS`), with the plane after it at `Pn` and the centre values of the plane
// before it in (pu, pd).  Writes the new u and the increment of each
// component to `out + c * ocs` and `out + (3 + c) * ocs` (inactive cells:
// 0) and, when `snap` is set, the new u of active cells to snap[3 c'] of the
// AoS snapshot.  (pu, pd) become this plane's centres.  The switches are
// template arguments fixed per tile: viscosity, damping, whether the pair of
// steps adds force terms, whether it writes a snapshot.
template <bool VISC, bool DAMP, bool PUSH, bool SNAP, int RS, int CS>
__device__ __forceinline__ void tb_pair_step(const float* __restrict__ P,
                                             const float* __restrict__ Pn, int o, float2 M,
                                             float2 E, float2 (&pu)[3], float2 (&pd)[3],
                                             bool act_a, bool act_b, const Lap7Pair& lk,
                                             float damp, const TbTermRef* __restrict__ terms,
                                             int nterms, unsigned nc, long long i, long long pf,
                                             float* __restrict__ out, unsigned ocs,
                                             float* __restrict__ snap) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int oc = o + c * CS, od = oc + 3 * CS;
    const float2 C = tb_ld2(P + oc), L = tb_ld2(P + oc - 2), R = tb_ld2(P + oc + 2);
    const float2 N = tb_ld2(P + oc + RS), S = tb_ld2(P + oc - RS), X = tb_ld2(Pn + oc);
    const float2 lu = lap7_pair(C, L, R, X, pu[c], N, S, lk);
    const float2 Cd = tb_ld2(P + od);
    float2 inc = ffma2(M, lu, Cd);
    if (VISC) {
      const float2 Ld = tb_ld2(P + od - 2), Rd = tb_ld2(P + od + 2);
      const float2 Nd = tb_ld2(P + od + RS), Sd = tb_ld2(P + od - RS), Xd = tb_ld2(Pn + od);
      inc = ffma2(E, lap7_pair(Cd, Ld, Rd, Xd, pd[c], Nd, Sd, lk), inc);
      pd[c] = Cd;
    }
    pu[c] = C;
    if (PUSH) {
      for (int j = 0; j < nterms; ++j) {
        const TbTermRef r = terms[j];
        const float* pp = r.base + (long long)c * nc + i;
        // the pattern is read with plain loads, outside the TMA ring: ask L2
        // for the next plane's now (pf: its offset, 0 when there is none)
        if (pf != 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(pp + pf));
        const float2 Pt = __ldg(reinterpret_cast<const float2*>(pp));
        inc = ffma2(Pt, splat2(r.scale), inc);
      }
    }
    if (DAMP) inc = fmul2(inc, splat2(damp));
    const float2 un = fadd2(C, inc);
    tb_st2(out + (size_t)c * ocs, act_a ? un.x : 0.f, act_b ? un.y : 0.f);
    tb_st2(out + (size_t)(3 + c) * ocs, act_a ? inc.x : 0.f, act_b ? inc.y : 0.f);
    if (SNAP && snap != nullptr) {
      if (act_a) snap[c] = un.x;
      if (act_b) snap[3 + c] = un.y;
    }
  }
}

// Where the two-step kernel's rings and barriers live.
struct TbRings {
  float* ringA;
  float* ringB;
  float* ringL;
  WsHeader* hd;
  uint64_t* Lfull;
  uint64_t* Lempty;
  volatile int* abort_flag;
  const TbTermBuf* terms;  // the two term buffers
};

// A consumer warp's next stage of each ring (level-0 planes, point-wise
// planes, level-1 slots), and whether its waits have all succeeded.
struct TbPos {
  RingPos<TmaF32TB::NA> ca;
  RingPos<TmaF32TB::NB> cb;
  RingPos<TmaF32TB::NL> lw;
  int ord = 0;  // tiles this warp has finished (picks the term buffer)
  bool ok = true;
};

// One tile of a consumer warp (level-1 row w): the tile's first plane x0-2
// (centres only; its full barrier waited on by the caller), then for every
// plane q = x0-1 .. x1 level 1 at q and level 2 at q-1.  Returns the ring
// positions after the tile, with ok = false when a wait gave up.
template <int LZ, bool VISC, bool DAMP, bool PUSH, bool SNAP>
__device__ __forceinline__ TbPos tb_tile(const TmaF32TB* __restrict__ in, int local, int lit,
                                         const TbRings& k, TbPos p, int w, int lane) {
  using T = TmaF32TB;
  using S = TbShape<LZ>;
  constexpr int W = S::W, H = S::H, WB = S::WB, HB = S::HB;
  constexpr int AF = T::A_STAGE / 4, BF = T::B_STAGE / 4, LF = T::L_STAGE / 4;
  constexpr int LP = LZ * S::LY;  // level-1 cells per component
  const Geom& g = in->g;
  const TbCoord tc = tb_coord<S::OZ, S::OY>(g, in->ts, local);
  float* __restrict__ D = in->state[(lit + 2) % 3];
  const unsigned nc = (unsigned)g.ncell;  // the host keeps ncell below 2^32
  const float damp = in->damp;
  const Lap7Pair lk =
      lap7_pair_coefs(in->hx, in->hy, in->hz, lap7_centre_coef(in->hx, in->hy, in->hz));
  // this thread: level-1 row r (y = y0-1+r), z pair zp, zp+1 (zp = z0-2+2 pl):
  // a warp owns one row of 32 pairs (LZ 64) or two rows of 16 (LZ 32)
  const int r = S::RPW == 1 ? w : 2 * w + (lane >> 4);
  const int pl = lane & (S::PAIRS - 1);
  const int y = tc.y0 - 1 + r, zp = tc.z0 - 2 + 2 * pl;
  const bool yin = y >= 1 && y <= g.ny - 2;
  const bool zin_a = zp >= 1 && zp <= g.nz - 2, zin_b = zp + 1 >= 1 && zp + 1 <= g.nz - 2;
  // a warp whose rows all lie outside the grid interior only writes zeros at
  // level 1 (the shell that level 2 reads)
  const bool warp_live = __any_sync(0xffffffffu, yin);
  // level 2: rows 1..OY and pairs 1..PAIRS-2 are the output tile
  const bool out_rc = r >= 1 && r <= S::OY && pl >= 1 && pl <= S::PAIRS - 2;
  const bool store = out_rc && yin && zp < g.pz;  // pz is even: the pair is in the row
  const int o = (r + 1) * W + 2 + 2 * pl, ob = r * WB + 2 + 2 * pl, ol = r * LZ + 2 * pl;
  // the force terms of steps lit (level 1) and lit+1 (level 2)
  const TbTermBuf& tbuf = k.terms[p.ord & 1];
  const int n1 = PUSH ? tbuf.n[0] : 0;
  const int n2 = PUSH ? tbuf.n[1] : 0;
  const bool snap1 = SNAP && ((lit + 1) % in->snap_stride) == 0;
  const bool snap2 = SNAP && ((lit + 2) % in->snap_stride) == 0;
  const int slot1 = snap1 ? (lit + 1) / in->snap_stride - 1 : 0;
  const int slot2 = snap2 ? (lit + 2) / in->snap_stride - 1 : 0;
  float2 pu[3], pd[3];  // level-0 centres of the plane before
  float2 qu[3], qd[3];  // level-1 centres of the plane before
  float2 Mp = make_float2(0.f, 0.f), Ep = Mp;  // coefficients of the previous plane
  {
    const float* P0 = k.ringA + p.ca.s * AF;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      pu[c] = tb_ld2(P0 + o + c * H * W);
      pd[c] = VISC ? tb_ld2(P0 + o + (3 + c) * H * W) : make_float2(0.f, 0.f);
      qu[c] = qd[c] = make_float2(0.f, 0.f);
    }
  }
  __syncwarp();
  if (lane == 0) mbar_arrive(&k.hd->emptyA[p.ca.s]);
  p.ca.next();
  RingPos<T::NA> cur = p.ca;  // plane q
  if (!ws_wait(&k.hd->fullA[cur.s], cur.ph, k.abort_flag)) {
      p.ok = false;
      return p;
    }
  p.ca.next();
  RingPos<T::NL> lprev = p.lw;  // slot of level-1 plane q-1 (meaningful from q = x0)
  for (int q = tc.x0 - 1; q <= tc.x1; ++q) {
    const RingPos<T::NA> nxt = p.ca;  // plane q+1
    if (!ws_wait(&k.hd->fullA[nxt.s], nxt.ph, k.abort_flag)) {
      p.ok = false;
      return p;
    }
    p.ca.next();
    const RingPos<T::NB> pt = p.cb;
    if (!ws_wait(&k.hd->fullB[pt.s], pt.ph, k.abort_flag)) {
      p.ok = false;
      return p;
    }
    p.cb.next();
    // the slot is free once every warp has read what it held before
    if (!ws_wait(&k.Lempty[p.lw.s], p.lw.ph ^ 1u, k.abort_flag)) {
      p.ok = false;
      return p;
    }
    float* Lw = k.ringL + p.lw.s * LF;
    // ---- level 1: step lit+1 at plane q on the level-1 region ----
    const float* Bm = k.ringB + pt.s * BF;
    const float2 Mc = tb_ld2(Bm + ob);
    const float2 Ec = VISC ? tb_ld2(Bm + HB * WB + ob) : make_float2(0.f, 0.f);
    const bool xin = q >= 1 && q <= g.nx - 2;
    if (!(xin && warp_live)) {
      // every cell of the warp's rows is outside the interior: level 1 is the
      // zero shell; keep this plane's level-0 centres for the next plane
      const float* P = k.ringA + cur.s * AF;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        pu[c] = tb_ld2(P + o + c * H * W);
        if (VISC) pd[c] = tb_ld2(P + o + (3 + c) * H * W);
        tb_st2(Lw + ol + c * LP, 0.f, 0.f);
        tb_st2(Lw + ol + (3 + c) * LP, 0.f, 0.f);
      }
    } else {
      const bool aa = xin && yin && zin_a, ab = xin && yin && zin_b;
      long long i = 0;  // the pair's cell, for the force patterns
      int nl = 0;
      if (PUSH) {
        i = (long long)min(max(q, 0), g.nx - 1) * g.sxy +
            (long long)min(max(y, 0), g.ny - 1) * g.pz + max(zp, 0);
        nl = (aa || ab) ? n1 : 0;
      }
      float* sp = nullptr;
      if (SNAP && snap1 && store && q >= tc.x0 && q < tc.x1)
        sp = in->snaps + ((((long long)slot1 * g.nx + q) * g.ny + y) * g.nz + zp) * 3;
      tb_pair_step<VISC, DAMP, PUSH, SNAP, W, H * W>(
          k.ringA + cur.s * AF, k.ringA + nxt.s * AF, o, Mc, Ec, pu, pd, aa, ab, lk, damp,
          tbuf.t[0], nl, nc, i, PUSH && q + 1 <= g.nx - 2 ? g.sxy : 0, Lw + ol, (unsigned)LP,
          sp);
    }
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&k.hd->emptyA[cur.s]);  // level-0 plane q is no longer needed
      mbar_arrive(&k.hd->emptyB[pt.s]);
      mbar_arrive(&k.Lfull[p.lw.s]);      // this warp's row of level-1 plane q is written
    }
    if (q >= tc.x0) {
      const float* Lc = k.ringL + lprev.s * LF;  // level-1 plane q-1
      if (q == tc.x0) {  // level-1 centres of plane x0-1 (own pair) for the first level 2
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          qu[c] = tb_ld2(Lc + ol + c * LP);
          qd[c] = VISC ? tb_ld2(Lc + ol + (3 + c) * LP) : make_float2(0.f, 0.f);
        }
      } else {
        // ---- level 2: step lit+2 at plane x = q-1 on the output tile ----
        // (reads rows r-1..r+1 of plane q-1: wait until every warp wrote it)
        if (!ws_wait(&k.Lfull[lprev.s], lprev.ph, k.abort_flag)) {
      p.ok = false;
      return p;
    }
        if (store) {
          const int x = q - 1;
          const long long i = (long long)x * g.sxy + (long long)y * g.pz + zp;
          float* sp = nullptr;
          if (SNAP && snap2)
            sp = in->snaps + ((((long long)slot2 * g.nx + x) * g.ny + y) * g.nz + zp) * 3;
          tb_pair_step<VISC, DAMP, PUSH, SNAP, LZ, LP>(Lc, Lw, ol, Mp, Ep, qu, qd, zin_a, zin_b,
                                                       lk, damp, tbuf.t[1], n2, nc, i, 0, D + i,
                                                       nc, sp);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&k.Lempty[lprev.s]);  // this warp is done with plane q-1
    }
    Mp = Mc;
    Ep = Ec;
    lprev = p.lw;
    p.lw.next();
    cur = nxt;
  }
  __syncwarp();
  if (lane == 0) {
    mbar_arrive(&k.hd->emptyA[cur.s]);  // the closing halo plane x1+1
    mbar_arrive(&k.Lempty[lprev.s]);    // the tile's last level-1 plane x1
  }
  return p;
}

// Whether the tile's pair of steps (lit+1, lit+2) adds force terms.
__device__ __forceinline__ bool tb_pushes(const TmaF32TB* __restrict__ in, int lit) {
  return in->term_off != nullptr && in->term_off[lit + 2] > in->term_off[lit];
}
// Whether the tile's pair of steps writes a snapshot.
__device__ __forceinline__ bool tb_snaps(const TmaF32TB* __restrict__ in, int lit) {
  return in->snap_stride > 0 && in->snaps != nullptr &&
         (((lit + 1) % in->snap_stride) == 0 || ((lit + 2) % in->snap_stride) == 0);
}

// The tile's switches (viscosity, damping, force terms, snapshot), resolved
// once per tile into a specialised loop, every path inlined.  Tiles of push
// or snapshot steps need more live values than the others; with their paths
// in called functions the common loop kept values on the stack around the
// calls (~3 local loads per warp and plane), and with the force terms read
// from the solve's tables inside the loop the push loop spilled (push tiles
// 4.9x slower).  With the terms in the shared term buffer the whole kernel
// fits 128 registers with nothing spilled.  (Running the push and snapshot
// tiles in a second launch of their own, which kept the first launch's
// variant at 102 registers, measured 1.4 % slower than this one launch.)
template <int LZ, bool VISC, bool DAMP>
__device__ __forceinline__ TbPos tb_tile_ps(bool push, bool snap, const TmaF32TB* __restrict__ in,
                                            int local, int lit, const TbRings& k, TbPos p, int w,
                                            int lane) {
  if (push) {
    if (snap) return tb_tile<LZ, VISC, DAMP, true, true>(in, local, lit, k, p, w, lane);
    return tb_tile<LZ, VISC, DAMP, true, false>(in, local, lit, k, p, w, lane);
  }
  if (snap) return tb_tile<LZ, VISC, DAMP, false, true>(in, local, lit, k, p, w, lane);
  return tb_tile<LZ, VISC, DAMP, false, false>(in, local, lit, k, p, w, lane);
}

template <int LZ>
__device__ __forceinline__ TbPos tb_tile_sw(const TmaF32TB* __restrict__ in, int local, int lit,
                                            const TbRings& k, TbPos p, int w, int lane) {
  const bool visc = in->ncoef > 1, damp = in->use_damp != 0;
  const bool push = tb_pushes(in, lit), snap = tb_snaps(in, lit);
  if (visc) {
    if (damp) return tb_tile_ps<LZ, true, true>(push, snap, in, local, lit, k, p, w, lane);
    return tb_tile_ps<LZ, true, false>(push, snap, in, local, lit, k, p, w, lane);
  }
  if (damp) return tb_tile_ps<LZ, false, true>(push, snap, in, local, lit, k, p, w, lane);
  return tb_tile_ps<LZ, false, false>(push, snap, in, local, lit, k, p, w, lane);
}


// LZ 0 (batched launches): each solve's tiles have the solve's own shape
// (TmaF32TB::lz), the one that computes fewer cells on its grid.
template <bool BATCH, int LZ>
__global__ void __launch_bounds__(TmaF32TB::THREADS, 1)
    step_f32_fused2(const __grid_constant__ TmaF32TB one, const TmaF32TB* __restrict__ tab,
                    int ninst, int ntiles, int it, const int* __restrict__ it_dev, int* queues) {
  static_assert(LZ != 0 || BATCH, "a single solve has one shape");
  if (it_dev != nullptr) it += *it_dev;  // step counter kept on the device (graph replays)
  // batched launches take tiles from a launch-wide queue (see step_f32_tma)
  int* queue = queues;
  using T = TmaF32TB;
  constexpr int NA = T::NA, NB = T::NB, NL = T::NL;
  constexpr int AF = T::A_STAGE / 4, BF = T::B_STAGE / 4, LF = T::L_STAGE / 4;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
  WsHeader* hd = reinterpret_cast<WsHeader*>(base);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(base + kAbortFlagOffset);
  float* ringA = reinterpret_cast<float*>(base + kRingOffset);
  float* ringB = ringA + NA * AF;
  float* ringL = ringB + NB * BF;
  uint64_t* Lfull = reinterpret_cast<uint64_t*>(ringL + NL * LF);  // after the rings
  uint64_t* Lempty = Lfull + NL;
  TbTermBuf* terms = reinterpret_cast<TbTermBuf*>(Lempty + NL);
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
      mbar_init(&hd->emptyA[s], T::CONSUMER_WARPS);
    }
    for (int s = 0; s < NB; ++s) {
      mbar_init(&hd->fullB[s], 1);
      mbar_init(&hd->emptyB[s], T::CONSUMER_WARPS);
    }
    for (int s = 0; s < NL; ++s) {
      mbar_init(&Lfull[s], T::CONSUMER_WARPS);
      mbar_init(&Lempty[s], T::CONSUMER_WARPS);
    }
    *abort_flag = 0;
    abort_flag[1] = BATCH ? (ninst > 0 ? tab[0].wait_k : 1) : one.wait_k;
    lg->n_taken = 0;
    lg->armedA = lg->parA = lg->armedB = lg->parB = 0;
    for (int w = 0; w < 16; ++w) lg->done[w] = 0;
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == T::CONSUMER_WARPS) {
    // ------------------------------- producer -----------------------------
    if (lane == 0) {
      RingPos<NA> pa;
      RingPos<NB> pb;
      int stride_next = blockIdx.x;
      bool ok = true;
      while (ok && !*abort_flag) {
        const int t = next_tile(queue, stride_next);
        if (t >= ntiles) {  // end of this CTA's work: arm one stage without a copy
          if (!ws_wait(&hd->emptyA[pa.s], pa.ph ^ 1u, abort_flag)) break;
          tile_slots(base)[pa.s] = -1;
          mbar_arrive(&hd->fullA[pa.s]);
          pa.next();
          break;
        }
        const int k = BATCH ? find_solve(tab, ninst, t) : 0;
        const T* in = BATCH ? &tab[k] : &one;
        const int local = BATCH ? t - in->tile_base : t;
        const int lit = it - in->it_begin;
        if (lit < 0 || lit + 1 >= in->n_steps || solve_abandoned(in->flags)) continue;
        const bool push = tb_pushes(in, lit);
        if (push && (in->term_off[lit + 1] - in->term_off[lit] > kTbTermCap ||
                     in->term_off[lit + 2] - in->term_off[lit + 1] > kTbTermCap)) {
          if (in->flags != nullptr) atomicOr(in->flags, kFlagRefused);  // see kTbTermCap
          continue;
        }
        const int ord = lg->n_taken;  // the tile's ordinal: its term buffer
        lg->solve[lg->n_taken & 7] = k;
        ++lg->n_taken;
        const Geom& g = in->g;
        const TbDims dm = LZ == 32 || (LZ == 0 && in->lz == 32) ? tb_dims<32>() : tb_dims<64>();
        const TbCoord tc = tb_coord_rt(g, in->ts, local, dm.oz, dm.oy);
        const CUtensorMap* tma = &in->tm[lit % 3];
        const uint32_t bbytes = dm.b_cells * 4 * in->ncoef;
        bool first = true;
        auto issueA = [&](int p) {
          const int sa = pa.s;
          ok = ok && ws_wait(&hd->emptyA[sa], pa.ph ^ 1u, abort_flag);
          if (!ok) return;
          if (first) {
            first = false;
            if (in->stall_test) {  // the testing switch leaves the tile's first stage unarmed
              pa.next();
              return;
            }
            tile_slots(base)[sa] = t;
            solve_slots(base)[sa] = k;
            if (push) {  // every warp has left tile ord-2, which used this buffer
              TbTermBuf& tb = terms[ord & 1];
              const unsigned nc = (unsigned)g.ncell;
              for (int lev = 0; lev < 2; ++lev) {
                const int j0 = in->term_off[lit + lev], j1 = in->term_off[lit + lev + 1];
                tb.n[lev] = j1 - j0;
                for (int j = j0; j < j1; ++j)
                  tb.t[lev][j - j0] = TbTermRef{in->pat + (long long)in->term_pat[j] * 3 * nc,
                                                (float)in->term_scale[j], 0};
              }
            }
          }
          const int pl = min(max(p, 0), g.nx - 1);  // planes outside the grid feed only the shell
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&hd->fullA[sa], dm.a_bytes);
          tma_load_4d(ringA + sa * AF, tma, &hd->fullA[sa], tc.z0 - 4, tc.y0 - 2, pl, 0);
          arm_record(lg->armedA, lg->parA, sa, pa.ph);
          pa.next();
        };
        auto issueB = [&](int q) {
          const int sb = pb.s;
          ok = ok && ws_wait(&hd->emptyB[sb], pb.ph ^ 1u, abort_flag);
          if (!ok) return;
          const int ql = min(max(q, 0), g.nx - 1);
          fence_proxy_async_smem();
          mbar_arrive_expect_tx(&hd->fullB[sb], bbytes);
          tma_load_4d(ringB + sb * BF, &in->tmm, &hd->fullB[sb], tc.z0 - 4, tc.y0 - 1, ql, 0);
          arm_record(lg->armedB, lg->parB, sb, pb.ph);
          pb.next();
        };
        issueA(tc.x0 - 2);
        issueA(tc.x0 - 1);
        for (int q = tc.x0 - 1; q <= tc.x1 && ok; ++q) {
          issueA(q + 1);
          issueB(q);
        }
      }
    }
  } else {
    // ------------------------------- consumers ----------------------------
    const TbRings k{ringA, ringB, ringL, hd, Lfull, Lempty, abort_flag, terms};
    TbPos p;
    while (true) {
      // the tile's first plane, x0-2: centres only
      if (!ws_wait(&hd->fullA[p.ca.s], p.ca.ph, abort_flag)) break;
      const int t = tile_slots(base)[p.ca.s];
      if (t < 0) break;
      const T* in = BATCH ? &tab[solve_slots(base)[p.ca.s]] : &one;
      const int local = BATCH ? t - in->tile_base : t;
      const int lit = it - in->it_begin;
      if (LZ == 0)
        p = in->lz == 32 ? tb_tile_sw<32>(in, local, lit, k, p, warp, lane)
                         : tb_tile_sw<64>(in, local, lit, k, p, warp, lane);
      else
        p = tb_tile_sw<LZ == 0 ? 64 : LZ>(in, local, lit, k, p, warp, lane);
      if (!p.ok) break;
      ++p.ord;
      if (lane == 0) ++lg->done[warp];
    }
  }
  __syncthreads();
  if (*abort_flag && warp == T::CONSUMER_WARPS && lane == 0) {
    // let every copy still in flight land, then flag the abandoned tiles' solves
    drain_ring(hd->fullA, lg->armedA, lg->parA, NA);
    drain_ring(hd->fullB, lg->armedB, lg->parB, NB);
    flag_unfinished(lg, T::CONSUMER_WARPS, BATCH ? ninst : 1, kFlagTimeout, flags_of);
  }
  queue_cta_done(queue);
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// alignment slack + header + rings + the level-1 ring's full / empty barriers
// + the two term buffers
size_t tb_smem_bytes() {
  return 128 + kRingOffset + (size_t)TmaF32TB::NA * TmaF32TB::A_STAGE +
         (size_t)TmaF32TB::NB * TmaF32TB::B_STAGE + (size_t)TmaF32TB::NL * TmaF32TB::L_STAGE +
         2 * TmaF32TB::NL * sizeof(uint64_t) + 2 * sizeof(TbTermBuf);
}

static int tb_set_attr() {
  static bool done = false;
  if (done) return SW_OK;
  const int bytes = (int)tb_smem_bytes();
  const void* fns[5] = {(const void*)step_f32_fused2<false, 64>,
                        (const void*)step_f32_fused2<true, 64>,
                        (const void*)step_f32_fused2<false, 32>,
                        (const void*)step_f32_fused2<true, 32>,
                        (const void*)step_f32_fused2<true, 0>};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(fused step smem)");
  }
  done = true;
  return SW_OK;
}

// planes per x chunk: minimise waves x (level-1 planes per tile) on 148 SMs
static int tb_xchunk(const Geom& g, int lz) {
  const long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0 || g.nz <= 2 || g.ny <= 2) return 1;
  const TileSpace one = make_tiles_tb(g, (int)nxi, lz);
  const long long cols = (long long)one.ntz * one.nty;
  const long long slots = kNumSMs;
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

// Cells the two levels compute per interior plane for tile width lz: the
// tiles times (level-1 region + output tile).
long long tb_work(const Geom& g, int lz) {
  const TileSpace t = make_tiles_tb(g, 1, lz);
  const long long per = lz == 32
                            ? (long long)TbShape<32>::LZ * TbShape<32>::LY +
                                  (long long)TbShape<32>::OZ * TbShape<32>::OY
                            : (long long)TbShape<64>::LZ * TbShape<64>::LY +
                                  (long long)TbShape<64>::OZ * TbShape<64>::OY;
  return (long long)t.ntz * t.nty * per;
}

int tb_tile_width(const Geom& g) {
  const int knob = tune_get(SW_TUNE_TILE_SHAPE);
  if (knob == 1) return 64;
  if (knob == 2) return 32;
  return tb_work(g, 32) < tb_work(g, 64) ? 32 : 64;
}

int make_tma_f32_tb(const StepArgs& a, int xchunk, TmaF32TB* t, int lz) {
  *t = TmaF32TB{};
  if (a.g.ncell >= (1LL << 32)) {  // the kernel offsets components by a 32-bit cell count
    set_error("grid too large for the two-step kernel (%lld cells)", a.g.ncell);
    return SW_ERANGE;
  }
  t->lz = lz == 32 || lz == 64 ? lz : tb_tile_width(a.g);
  t->g = a.g;
  t->ts = make_tiles_tb(a.g, xchunk > 0 ? xchunk : tb_xchunk(a.g, t->lz), t->lz);
  if (a.coef_e == nullptr) {
    t->ncoef = 1;
  } else if ((const char*)a.coef_e == (const char*)a.coef_m + a.g.ncell * 4) {
    t->ncoef = 2;
  } else {
    set_error("the fused step kernel needs coef_e == coef_m + ncell");
    return SW_EINVAL;
  }
  if (a.kahan) {
    set_error("the two-steps-per-pass kernel runs without the compensated sum");
    return SW_EINVAL;
  }
  const bool n32 = t->lz == 32;
  const uint32_t W = n32 ? TbShape<32>::W : TbShape<64>::W;
  const uint32_t H = n32 ? TbShape<32>::H : TbShape<64>::H;
  const uint32_t WB = n32 ? TbShape<32>::WB : TbShape<64>::WB;
  const uint32_t HB = n32 ? TbShape<32>::HB : TbShape<64>::HB;
  const uint64_t dims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx, 9};
  const uint64_t strides[3] = {(uint64_t)a.g.pz * 4, (uint64_t)a.g.sxy * 4,
                               (uint64_t)a.g.ncell * 4};
  const uint32_t boxA[4] = {W, H, 1, 6};
  for (int b = 0; b < 3; ++b) {
    t->state[b] = (float*)a.state[b];
    int rc = encode_tmap_4d(&t->tm[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, a.state[b], dims, strides,
                            boxA);
    if (rc != SW_OK) return rc;
  }
  const uint64_t mdims[4] = {(uint64_t)a.g.pz, (uint64_t)a.g.ny, (uint64_t)a.g.nx,
                             (uint64_t)t->ncoef};
  const uint32_t boxM[4] = {WB, HB, 1, (uint32_t)t->ncoef};
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

int launch_fused2_prepare() { return tb_set_attr(); }

const void* step_f32_fused2_ptr(int lz) {
  return lz == 32 ? reinterpret_cast<const void*>(step_f32_fused2<false, 32>)
                  : reinterpret_cast<const void*>(step_f32_fused2<false, 64>);
}

const void* step_f32_fused2_batch_ptr(int lz) {
  if (lz == 0) return reinterpret_cast<const void*>(step_f32_fused2<true, 0>);
  return lz == 32 ? reinterpret_cast<const void*>(step_f32_fused2<true, 32>)
                  : reinterpret_cast<const void*>(step_f32_fused2<true, 64>);
}

static void launch_tb(const void* fn, int grid, cudaStream_t s, const TmaF32TB& one,
                      const TmaF32TB* tab, int ninst, int ntiles, int it, int* queues) {
  const int* itd = nullptr;
  void* args[] = {(void*)&one, (void*)&tab, (void*)&ninst, (void*)&ntiles, (void*)&it,
                  (void*)&itd, (void*)&queues};
  cudaLaunchKernel(fn, dim3(grid), dim3(TmaF32TB::THREADS), args, tb_smem_bytes(), s);
}

void launch_fused2_raw(const TmaF32TB& t, int it, cudaStream_t s) {
  if (t.ts.count == 0) return;
  launch_tb(step_f32_fused2_ptr(t.lz), std::min(t.ts.count, kNumSMs), s, t, nullptr, 1,
            t.ts.count, it, nullptr);
}

int launch_fused2(const StepArgs& a, int xchunk, int it, cudaStream_t s) {
  int rc = tb_set_attr();
  if (rc != SW_OK) return rc;
  TmaF32TB t;
  rc = make_tma_f32_tb(a, xchunk, &t, 0);
  if (rc != SW_OK) return rc;
  if (t.ts.count == 0) return SW_OK;
  launch_fused2_raw(t, it, s);
  count_launches(1);
  SW_CHECK_LAUNCH("fused two-step kernel");
  return SW_OK;
}

int launch_fused2_batch(const void* d_tab, int ninst, int ntiles, int it, int* queues, int lz,
                        cudaStream_t s) {
  int rc = tb_set_attr();
  if (rc != SW_OK) return rc;
  if (ntiles == 0) return SW_OK;
  TmaF32TB dummy{};
  launch_tb(step_f32_fused2_batch_ptr(lz), std::min(ntiles, kNumSMs), s, dummy,
            (const TmaF32TB*)d_tab, ninst, ntiles, it, queues);
  count_launches(1);
  SW_CHECK_LAUNCH("fused two-step kernel (batch)");
  return SW_OK;
}

}  // namespace sw
