// Helmholtz-Hodge projection and its FP64 conjugate-gradient Poisson solve.
//
// Reference: project_vector_field (src/shearwave/solver.py:644-683) and
// poisson_cg (src/shearwave/solver.py:1010-1050).
//
// The operator is A x = -div_c(grad_c x) with both 2h central differences
// zero on the shell, so per axis an interior row reads x at i-2, i, i+2 and
// drops the gradient term whose centre i+-1 lies on the shell.  One CG
// iteration is two launches:
//   cg_apply  : p_k = r + beta p_{k-1} (fused, written to the other p buffer),
//               Ap = A p_k, partial p_k.Ap
//   cg_update : x += alpha p_k, r -= alpha Ap, partial r.r
// Each launch ends with a "last block" step: the block that takes the final
// ticket of an instance sums that instance's per-tile partials in a fixed
// order (deterministic) and advances the instance's scalar CG state, with the
// reference's stopping rule.  No block ever waits for another one.
// Every kernel works on a table of instances so that one launch can advance
// many independent solves (the batched path) as well as a single one.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "sw_common.cuh"
#include "sw_project.cuh"

namespace sw {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ inline int find_inst(const CgInst* __restrict__ tab, int ninst, int t) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {  // last instance with tile_base <= t
    int mid = (lo + hi + 1) >> 1;
    if (tab[mid].tile_base <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Take a ticket for instance `in`; returns true in every thread of the block
// that took the last ticket.  The caller has written its partial already.
__device__ inline bool last_block(const CgInst& in, unsigned int* flag_smem) {
  __syncthreads();
  if (flat_tid() == 0) {
    __threadfence();
    unsigned int t = atomicAdd(&in.st->ticket, 1u);
    *flag_smem = (t == (unsigned int)(in.ts.count - 1)) ? 1u : 0u;
  }
  __syncthreads();
  bool last = *flag_smem != 0u;
  if (last) __threadfence();
  return last;
}

// Sum (and max) of this instance's per-tile partials, fixed order.
__device__ inline double2 reduce_partials(const CgInst& in, double* red) {
  double s = 0.0, m = 0.0;
  const int tid = flat_tid(), nthr = blockDim.x * blockDim.y;
  for (int i = tid; i < in.ts.count; i += nthr) {
    double2 v = __ldcg(&in.partials[i]);
    s += v.x;
    m = fmax(m, v.y);
  }
  double2 out;
  out.x = block_sum(s, red);
  __syncthreads();
  out.y = block_max(m, red);
  return out;
}

template <typename T>
__device__ inline double ld_masked(const T* __restrict__ f, const CgInst& in, const InStride& s,
                                   int x, int y, int z) {
  if (f == nullptr || !interior(in.g, x, y, z)) return 0.0;
  return (double)f[(long long)x * s.sx + (long long)y * s.sy + (long long)z * s.sz];
}

// ---------------------------------------------------------------------------
// prep: rhs = -div_c(mask f), r = p0 = rhs, rs0, max|div|
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) cg_prep(const CgInst* __restrict__ tab, int ninst,
                                                        int ntiles, const T* const* __restrict__ fin,
                                                        const InStride* __restrict__ fstride) {
  __shared__ double red[32];
  __shared__ unsigned int lastflag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ii = find_inst(tab, ninst, t);
    const CgInst& in = tab[ii];
    const Geom& g = in.g;
    const T* fx = fin[3 * ii + 0];
    const T* fy = fin[3 * ii + 1];
    const T* fz = fin[3 * ii + 2];
    const InStride s = fstride[ii];
    const int local = t - in.tile_base;
    const TileCoord tc = tile_coord(g, in.ts, local);
    const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
    double acc = 0.0, mx = 0.0;
    if (in.op == 1) {  // static elastic solve: r = p = mask b, mu to FP64
      const T* mu = fin[3 * ii + 1];
      for (int x = tc.x0; x < tc.x1; ++x) {
        if (!interior(g, x, y, z)) continue;
        const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
        const double b = ld_masked(fx, in, s, x, y, z);
        in.r[i] = b;
        in.p0[i] = b;
        in.muf[i] = mu ? ld_masked(mu, in, s, x, y, z) : in.mu_s;
        acc += b * b;
      }
    }
    for (int x = tc.x0; x < tc.x1 && in.op == 0; ++x) {
      if (!interior(g, x, y, z)) continue;
      double tx = (ld_masked(fx, in, s, x + 1, y, z) - ld_masked(fx, in, s, x - 1, y, z)) * in.c2x;
      double ty = (ld_masked(fy, in, s, x, y + 1, z) - ld_masked(fy, in, s, x, y - 1, z)) * in.c2y;
      double tz = (ld_masked(fz, in, s, x, y, z + 1) - ld_masked(fz, in, s, x, y, z - 1)) * in.c2z;
      double div = (tx + ty) + tz;
      double rhs = -div;
      long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
      in.r[i] = rhs;
      in.p0[i] = rhs;
      acc += rhs * rhs;
      mx = fmax(mx, fabs(div));
    }
    double bs = block_sum(acc, red);
    __syncthreads();
    double bm = block_max(mx, red);
    if (flat_tid() == 0) in.partials[local] = make_double2(bs, bm);
    if (last_block(in, &lastflag)) {
      double2 tot = reduce_partials(in, red);
      if (flat_tid() == 0) {
        CgState* st = in.st;
        st->ticket = 0u;
        st->rs = tot.x;
        st->rs0 = fmax(tot.x, 2.220446049250313e-16);
        st->maxdiv = tot.y;
        st->iters = 0;
        st->k = 0;
        st->rel = nan("");
        if (in.op == 0 && tot.y < 1e-12) st->reason = SW_CG_EARLY_EXIT;
        else if (st->max_iters <= 0) st->reason = SW_CG_MAXITERS;
        else st->reason = SW_CG_RUNNING;
        __threadfence();
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// apply: p_k (fused update), Ap = A p_k, partial p_k.Ap
// ---------------------------------------------------------------------------
// The per-solve scalars (state, step scalars) that another block's last-block
// step wrote: the persistent kernel (COH) reads them from L2 (ld.global.cg);
// separate launches may use L1.
template <bool COH, typename T>
__device__ __forceinline__ T ldv(const T* p) {
  if (COH) return __ldcg(p);
  return *p;
}

// The stencil's vectors (r, the previous p) are read with plain, L1-cached
// loads in both forms: in the persistent kernel every block writes them
// before a grid barrier (release: a gpu-scope fence, then the arrival) and
// reads them after it (acquire: the wait, a gpu-scope fence, then the block
// barrier), so the memory model makes every write before the barrier visible
// to every load after it, and within a phase the vectors a block reads are
// not written.  Each value then comes from L2 once per block instead of at
// each of the stencil's 7 points (5 % faster than ld.global.cg at 192^3).
template <bool COH>
struct PView {
  const double* r;
  const double* pold;
  double beta;
  bool first;
  __device__ inline double operator()(long long i) const {
    return first ? pold[i] : fma(beta, pold[i], r[i]);
  }
};

// A = -div_c grad_c (op 0) at interior cell i with p read through `pv` and
// pc = p at i: the one expression both phases evaluate (the update phase
// recomputes Ap from the stored p instead of reading an Ap vector the apply
// phase wrote), so the two agree bit for bit.
template <typename PV>
__device__ __forceinline__ double op0_ap(const PV& pv, const CgInst& in, const Geom& g,
                                         long long i, int x, int y, int z, double pc) {
  double gp, gm, tx, ty, tz;
  gp = (x + 1 <= g.nx - 2) ? (pv(i + 2 * g.sxy) - pc) * in.c2x : 0.0;
  gm = (x - 1 >= 1) ? (pc - pv(i - 2 * g.sxy)) * in.c2x : 0.0;
  tx = (gp - gm) * in.c2x;
  gp = (y + 1 <= g.ny - 2) ? (pv(i + 2 * g.pz) - pc) * in.c2y : 0.0;
  gm = (y - 1 >= 1) ? (pc - pv(i - 2 * g.pz)) * in.c2y : 0.0;
  ty = (gp - gm) * in.c2y;
  gp = (z + 1 <= g.nz - 2) ? (pv(i + 2) - pc) * in.c2z : 0.0;
  gm = (z - 1 >= 1) ? (pc - pv(i - 2)) * in.c2z : 0.0;
  tz = (gp - gm) * in.c2z;
  return -((tx + ty) + tz);
}

// Ask L2 for a line a few planes ahead of a column walk (the walk issues one
// plane's loads at a time; the hint keeps more DRAM reads in flight).  Only
// addresses inside the vector are passed.
constexpr int kCgPrefetchPlanes = 4;
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// One tile of the apply phase (every thread of the block; uniform control).
template <bool COH>
__device__ __forceinline__ void apply_tile(const CgInst* __restrict__ tab, int ninst, int t,
                                           double* red, unsigned int* lastflag) {
  const int ii = find_inst(tab, ninst, t);
  const CgInst& in = tab[ii];
  const CgState* st = in.st;
  if (ldv<COH>(&st->reason) != SW_CG_RUNNING) return;  // uniform across the block
  const Geom& g = in.g;
  const int k = ldv<COH>(&st->k);
  PView<COH> pv;
  pv.first = (k == 0);
  pv.r = in.r;
  pv.beta = ldv<COH>(&st->beta);
  pv.pold = pv.first ? in.p0 : ((k - 1) & 1 ? in.p1 : in.p0);
  double* pnew = (k & 1) ? in.p1 : in.p0;
  const int local = t - in.tile_base;
  const TileCoord tc = tile_coord(g, in.ts, local);
  const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
  double acc = 0.0;
  for (int x = tc.x0; x < tc.x1; ++x) {
    if (!interior(g, x, y, z)) continue;
    const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
    if (x + kCgPrefetchPlanes <= g.nx - 1) {
      const long long ia = i + kCgPrefetchPlanes * g.sxy;
      prefetch_l2(pv.pold + ia);
      if (!pv.first) prefetch_l2(pv.r + ia);
    }
    const double pc = pv(i);
    if (in.op == 1) {  // -mu L7(p), laplacian_center's operation order
      const double lap = ((pv(i + g.sxy) - 2.0 * pc) + pv(i - g.sxy)) * in.ihx2 +
                         ((pv(i + g.pz) - 2.0 * pc) + pv(i - g.pz)) * in.ihy2 +
                         ((pv(i + 1) - 2.0 * pc) + pv(i - 1)) * in.ihz2;
      const double ap = -in.muf[i] * lap;
      in.ap[i] = ap;
      if (!pv.first) pnew[i] = pc;
      acc += pc * ap;
      continue;
    }
    const double ap = op0_ap(pv, in, g, i, x, y, z, pc);  // not stored: the update recomputes it
    if (!pv.first) pnew[i] = pc;
    acc += pc * ap;
  }
  double bs = block_sum(acc, red);
  if (flat_tid() == 0) in.partials[local] = make_double2(bs, 0.0);
  if (last_block(in, lastflag)) {
    double2 tot = reduce_partials(in, red);
    if (flat_tid() == 0) {
      CgState* w = in.st;
      w->ticket = 0u;
      const double denom = tot.x;
      const bool stop = (in.op == 1) ? (denom <= 0.0) : (!isfinite(denom) || denom <= 0.0);
      if (stop) w->reason = SW_CG_BREAKDOWN;
      else w->alpha = w->rs / denom;
      __threadfence();
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(TILE_THREADS) cg_apply(const CgInst* __restrict__ tab, int ninst,
                                                         int ntiles) {
  __shared__ double red[32];
  __shared__ unsigned int lastflag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    apply_tile<false>(tab, ninst, t, red, &lastflag);
}

// ---------------------------------------------------------------------------
// update: x += alpha p_k, r -= alpha Ap, partial r.r, stopping rule
// ---------------------------------------------------------------------------
// Every vector read here was written by this same thread (x, r, Ap, p_k at
// its own cells), so plain loads are coherent even in the persistent kernel;
// the scalar state comes from L2 there.
template <bool COH>
__device__ __forceinline__ void update_tile(const CgInst* __restrict__ tab, int ninst, int t,
                                            double* red, unsigned int* lastflag) {
  const int ii = find_inst(tab, ninst, t);
  const CgInst& in = tab[ii];
  const CgState* st = in.st;
  if (ldv<COH>(&st->reason) != SW_CG_RUNNING) return;
  const Geom& g = in.g;
  const int k = ldv<COH>(&st->k);
  const double alpha = ldv<COH>(&st->alpha);
  const double* pk = (k & 1) ? in.p1 : in.p0;
  const int local = t - in.tile_base;
  const TileCoord tc = tile_coord(g, in.ts, local);
  const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
  double acc = 0.0;
  if (y >= 1 && y <= g.ny - 2 && z >= 1 && z <= g.nz - 2) {
    // the column's planes are independent: restrict lets the loads of later
    // planes go ahead of the stores of earlier ones
    double* __restrict__ X = in.x;
    double* __restrict__ R = in.r;
    const double* __restrict__ AP = in.ap;
    const double* __restrict__ PK = pk;
    const long long c0 = (long long)y * g.pz + z;
    if (in.op == 0) {
      // Ap from p_k (written before the barrier: plain loads, as in PView)
      auto pkv = [PK](long long j) { return PK[j]; };
#pragma unroll 1
      for (int x = tc.x0; x < tc.x1; ++x) {
        const long long i = (long long)x * g.sxy + c0;
        if (x + kCgPrefetchPlanes <= g.nx - 1) {
          const long long ia = i + kCgPrefetchPlanes * g.sxy;
          prefetch_l2(X + ia);
          prefetch_l2(R + ia);
          prefetch_l2(PK + ia);
        }
        const double pc = PK[i];
        const double ap = op0_ap(pkv, in, g, i, x, y, z, pc);
        X[i] = fma(alpha, pc, X[i]);
        const double rn = fma(-alpha, ap, R[i]);
        R[i] = rn;
        acc += rn * rn;
      }
    } else {
#pragma unroll 4
      for (int x = tc.x0; x < tc.x1; ++x) {
        const long long i = (long long)x * g.sxy + c0;
        X[i] = fma(alpha, PK[i], X[i]);
        const double rn = fma(-alpha, AP[i], R[i]);
        R[i] = rn;
        acc += rn * rn;
      }
    }
  }
  double bs = block_sum(acc, red);
  if (flat_tid() == 0) in.partials[local] = make_double2(bs, 0.0);
  if (last_block(in, lastflag)) {
    double2 tot = reduce_partials(in, red);
    if (flat_tid() == 0) {
      CgState* w = in.st;
      w->ticket = 0u;
      const double rs_new = tot.x;
      w->iters += 1;
      if (in.op == 0 && !isfinite(rs_new)) {
        w->reason = SW_CG_NONFINITE;
      } else {
        const double rel = sqrt(rs_new / w->rs0);
        w->rel = rel;
        if (rel < w->tol) {
          w->reason = SW_CG_CONVERGED;
        } else {
          w->beta = rs_new / fmax(w->rs, 2.220446049250313e-16);
          w->rs = rs_new;
          w->k += 1;
          if (w->iters >= w->max_iters) w->reason = SW_CG_MAXITERS;
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(TILE_THREADS) cg_update(const CgInst* __restrict__ tab, int ninst,
                                                          int ntiles) {
  __shared__ double red[32];
  __shared__ unsigned int lastflag;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    update_tile<false>(tab, ninst, t, red, &lastflag);
}

// ---------------------------------------------------------------------------
// persistent CG: every iteration of every instance in one cooperative launch
// ---------------------------------------------------------------------------
// The two phases of an iteration are separated by a grid-wide barrier; the
// per-instance scalars still advance in the "last block" of each phase, so
// the arithmetic (and the order of every sum) is the two-launch version's.
// The barrier's waits are bounded: one that runs out sets the error word and
// every block leaves the loop (the host reports it); nothing spins forever.
constexpr uint32_t kCgBarrierBudget = 1u << 20;  // units of 1024 cycles (~0.5 s)

__device__ bool cg_grid_sync(CgGrid* b) {
  __shared__ int ok_s;
  __syncthreads();
  if (flat_tid() == 0) {
    int ok = 1;
    volatile unsigned int* gen = &b->gen;
    const unsigned int g0 = *gen;
    __threadfence();
    if (atomicAdd(&b->count, 1u) + 1u == gridDim.x) {
      atomicExch(&b->count, 0u);
      __threadfence();
      atomicAdd(&b->gen, 1u);
    } else {
      const uint32_t t0 = (uint32_t)clock();
      while (*gen == g0) {
        if (*(volatile int*)&b->error) {
          ok = 0;
          break;
        }
        if ((((uint32_t)clock() - t0) >> 10) > kCgBarrierBudget) {
          atomicExch(&b->error, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

__global__ void __launch_bounds__(TILE_THREADS, 5) cg_persist(const CgInst* __restrict__ tab,
                                                           int ninst, int ntiles, CgGrid* bar) {
  __shared__ double red[32];
  __shared__ unsigned int lastflag;
  __shared__ int any_s;
  for (;;) {
    if (flat_tid() == 0) {
      int any = 0;
      for (int i = 0; i < ninst && !any; ++i) any = __ldcg(&tab[i].st->reason) == SW_CG_RUNNING;
      any_s = any;
    }
    __syncthreads();
    if (!any_s) break;  // the same answer in every block: the states changed before a barrier
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
      apply_tile<true>(tab, ninst, t, red, &lastflag);
    if (!cg_grid_sync(bar)) break;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
      update_tile<true>(tab, ninst, t, red, &lastflag);
    if (!cg_grid_sync(bar)) break;
  }
}

// ---------------------------------------------------------------------------
// finish: out = (mask f - grad_c x), zero shell
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TILE_THREADS) cg_finish(const CgInst* __restrict__ tab, int ninst,
                                                          int ntiles, const T* const* __restrict__ fin,
                                                          const InStride* __restrict__ fstride,
                                                          double* const* __restrict__ outs) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ii = find_inst(tab, ninst, t);
    const CgInst& in = tab[ii];
    const Geom& g = in.g;
    const InStride s = fstride[ii];
    double* out = outs[ii];
    const int local = t - in.tile_base;
    const TileCoord tc = tile_coord(g, in.ts, local);
    const int z = tc.z0 + threadIdx.x, y = tc.y0 + threadIdx.y;
    for (int x = tc.x0; x < tc.x1; ++x) {
      if (!interior(g, x, y, z)) continue;
      const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
      const double gx = (in.x[i + g.sxy] - in.x[i - g.sxy]) * in.c2x;
      const double gy = (in.x[i + g.pz] - in.x[i - g.pz]) * in.c2y;
      const double gz = (in.x[i + 1] - in.x[i - 1]) * in.c2z;
      out[i] = ld_masked(fin[3 * ii + 0], in, s, x, y, z) - gx;
      out[i + g.ncell] = ld_masked(fin[3 * ii + 1], in, s, x, y, z) - gy;
      out[i + 2 * g.ncell] = ld_masked(fin[3 * ii + 2], in, s, x, y, z) - gz;
    }
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

size_t cg_workspace_bytes(const Geom& g, const TileSpace& ts) {
  size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
  size_t b = 6 * vec;                                            // x r p0 p1 ap muf
  b += align_up((size_t)ts.count * sizeof(double2), 256);        // partials
  b += align_up(sizeof(CgState), 256);                           // state + grid barrier
  b += align_up(sizeof(CgInst), 256);                            // instance table
  b += align_up(3 * sizeof(void*) + sizeof(InStride) + sizeof(double*), 256);
  return b;
}

TileSpace cg_tiles(const Geom& g) { return make_tiles(g, choose_xchunk(g, 4 * 148)); }

int cg_layout(const Geom& g, char* ws, size_t ws_bytes, CgInst* in, CgState** st,
              char** tail) {
  in->g = g;
  in->ts = cg_tiles(g);
  size_t need = cg_workspace_bytes(g, in->ts);
  if (ws == nullptr || ws_bytes < need) {
    set_error("workspace of %zu bytes is smaller than the %zu bytes required", ws_bytes, need);
    return SW_EWORKSPACE;
  }
  size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
  char* p = ws;
  in->x = (double*)p;
  p += vec;
  in->r = (double*)p;
  p += vec;
  in->p0 = (double*)p;
  p += vec;
  in->p1 = (double*)p;
  p += vec;
  in->ap = (double*)p;
  p += vec;
  in->muf = (double*)p;
  p += vec;
  in->partials = (double2*)p;
  p += align_up((size_t)in->ts.count * sizeof(double2), 256);
  *st = (CgState*)p;
  in->st = *st;
  p += align_up(sizeof(CgState), 256);
  *tail = p;
  in->tile_base = 0;
  return SW_OK;
}

// Blocks of a cooperative cg_persist launch on the current device (all
// resident at once), or 0 when the device cannot launch one.
static int cg_coop_blocks() {
  int dev = 0, coop = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
    return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, cg_persist, TILE_THREADS, 0) !=
      cudaSuccess)
    return 0;
  return per * sms;
}

int cg_run(const CgInst* d_tab, int ninst, int ntiles, CgState* d_states, int nst,
           CgGrid* d_grid, cudaStream_t s) {
  // One cooperative launch runs every iteration (grid barriers between the
  // phases); without cooperative launch support, iterations are launched in
  // growing batches and the host polls the exit reasons between batches.
  const int coop = d_grid != nullptr ? cg_coop_blocks() : 0;
  if (coop > 0) {
    const int grid = std::max(1, std::min(ntiles, coop));
    cudaError_t e = cudaMemsetAsync(d_grid, 0, sizeof(CgGrid), s);
    void* args[] = {(void*)&d_tab, (void*)&ninst, (void*)&ntiles, (void*)&d_grid};
    if (e == cudaSuccess)
      e = cudaLaunchCooperativeKernel((const void*)cg_persist, dim3(grid),
                                      dim3(TILE_Z, TILE_Y), args, 0, s);
    if (e != cudaSuccess) return cuda_status(e, "cg_persist launch");
    count_launches(1);
    CgGrid hg{};
    e = cudaMemcpyAsync(&hg, d_grid, sizeof(hg), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "cg_persist readback");
    if (hg.error) {
      set_error("CG: a grid barrier of the persistent kernel timed out");
      return SW_ETIMEOUT;
    }
    return SW_OK;
  }
  const int grid = std::max(1, std::min(ntiles, 148 * 8));
  CgState local[4];  // a single solve polls without touching the heap
  std::vector<CgState> heap(nst > 4 ? nst : 0);
  CgState* h = nst > 4 ? heap.data() : local;
  int batch = 4;
  for (;;) {
    cudaError_t e = cudaMemcpyAsync(h, d_states, nst * sizeof(CgState),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "cg state readback");
    bool running = false;
    for (int i = 0; i < nst; ++i) running |= (h[i].reason == SW_CG_RUNNING);
    if (!running) return SW_OK;
    for (int b = 0; b < batch; ++b) {
      cg_apply<<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, ninst, ntiles);
      cg_update<<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, ninst, ntiles);
    }
    count_launches(2ull * batch);
    SW_CHECK_LAUNCH("cg iteration");
    batch = std::min(batch * 2, 64);
  }
}

template <typename T>
int project_one(const void* fx, const void* fy, const void* fz, InStride fs, const Geom& g,
                double dX, double dY, double dZ, double tol, int max_iters, double* out, void* ws,
                size_t ws_bytes, sw_cg_stats* stats, cudaStream_t s) {
  CgInst in{};
  CgState* st = nullptr;
  char* tail = nullptr;
  int rc = cg_layout(g, (char*)ws, ws_bytes, &in, &st, &tail);
  if (rc != SW_OK) return rc;
  in.c2x = 1.0 / (2.0 * dX);
  in.c2y = 1.0 / (2.0 * dY);
  in.c2z = 1.0 / (2.0 * dZ);
  CgInst* d_tab = (CgInst*)tail;
  tail += align_up(sizeof(CgInst), 256);
  const T** d_fin = (const T**)tail;
  InStride* d_fs = (InStride*)(tail + 3 * sizeof(void*));
  double** d_out = (double**)(tail + 3 * sizeof(void*) + sizeof(InStride));

  struct {
    const T* f[3];
    InStride st;
    double* out;
  } hostargs;
  hostargs.f[0] = (const T*)fx;
  hostargs.f[1] = (const T*)fy;
  hostargs.f[2] = (const T*)fz;
  hostargs.st = fs;
  hostargs.out = out;

  CgState hst{};
  hst.tol = tol;
  hst.max_iters = max_iters;
  hst.reason = SW_CG_RUNNING;
  cudaError_t e;
  // x r p0 p1 ap muf are consecutive 256-byte aligned vectors: zero all of them
  const size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
  e = cudaMemsetAsync(in.x, 0, 6 * vec, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st, &hst, sizeof(hst), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_tab, &in, sizeof(in), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_fin, hostargs.f, 3 * sizeof(void*), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_fs, &fs, sizeof(fs), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, &out, sizeof(out), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, (size_t)g.ncell * 3 * sizeof(double), s);
  if (e != cudaSuccess) return cuda_status(e, "projection setup");
  const int ntiles = in.ts.count;
  if (ntiles > 0) {
    const int grid = std::max(1, std::min(ntiles, 148 * 8));
    cg_prep<T><<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, 1, ntiles, d_fin, d_fs);
    count_launches(1);
    SW_CHECK_LAUNCH("cg_prep");
    rc = cg_run(d_tab, 1, ntiles, st, 1, cg_grid_of(st), s);
    if (rc != SW_OK) return rc;
    cg_finish<T><<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, 1, ntiles, d_fin, d_fs, d_out);
    count_launches(1);
    SW_CHECK_LAUNCH("cg_finish");
  }
  e = cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "projection readback");
  if (stats) {
    if (ntiles == 0) {
      hst.iters = 0;
      hst.reason = SW_CG_EARLY_EXIT;
      hst.rel = nan("");
      hst.maxdiv = 0.0;
    }
    stats->iters = hst.iters;
    stats->reason = hst.reason;
    stats->rel = hst.rel;
    stats->max_div = hst.maxdiv;
  }
  return SW_OK;
}

// Static elastic solve: CG on (-mu L7) u = b (solver.py:569-625) in FP64;
// u (padded FP64) is written to `out`.
template <typename T>
int static_one(const void* b, const void* mu, double mu_s, InStride fs, const Geom& g,
               double dX, double dY, double dZ, double tol, int max_iters, double* out,
               void* ws, size_t ws_bytes, sw_cg_stats* stats, cudaStream_t s) {
  CgInst in{};
  CgState* st = nullptr;
  char* tail = nullptr;
  int rc = cg_layout(g, (char*)ws, ws_bytes, &in, &st, &tail);
  if (rc != SW_OK) return rc;
  in.op = 1;
  in.ihx2 = 1.0 / (dX * dX);
  in.ihy2 = 1.0 / (dY * dY);
  in.ihz2 = 1.0 / (dZ * dZ);
  in.mu_s = mu_s;
  CgInst* d_tab = (CgInst*)tail;
  tail += align_up(sizeof(CgInst), 256);
  const T** d_fin = (const T**)tail;
  InStride* d_fs = (InStride*)(tail + 3 * sizeof(void*));
  const void* fin[3] = {b, mu, nullptr};
  CgState hst{};
  hst.tol = tol;
  hst.max_iters = max_iters;
  hst.reason = SW_CG_RUNNING;
  const size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
  cudaError_t e = cudaMemsetAsync(in.x, 0, 6 * vec, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st, &hst, sizeof(hst), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_tab, &in, sizeof(in), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_fin, fin, 3 * sizeof(void*), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_fs, &fs, sizeof(fs), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_status(e, "static solve setup");
  const int ntiles = in.ts.count;
  if (ntiles > 0) {
    const int grid = std::max(1, std::min(ntiles, 148 * 8));
    cg_prep<T><<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, 1, ntiles, d_fin, d_fs);
    count_launches(1);
    SW_CHECK_LAUNCH("static cg_prep");
    rc = cg_run(d_tab, 1, ntiles, st, 1, cg_grid_of(st), s);
    if (rc != SW_OK) return rc;
  }
  e = cudaMemcpyAsync(out, in.x, (size_t)g.ncell * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hst, st, sizeof(hst), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "static solve readback");
  if (stats) {
    stats->iters = hst.iters;
    stats->reason = ntiles > 0 ? hst.reason : SW_CG_MAXITERS;
    stats->rel = hst.rel;
    stats->max_div = 0.0;
  }
  return SW_OK;
}

int project_field(int dtype, const void* fx, const void* fy, const void* fz, InStride fs,
                  const Geom& g, double dX, double dY, double dZ, double tol, int max_iters,
                  double* out, void* ws, size_t ws_bytes, sw_cg_stats* stats, cudaStream_t s) {
  if (dtype == SW_F32)
    return project_one<float>(fx, fy, fz, fs, g, dX, dY, dZ, tol, max_iters, out, ws, ws_bytes,
                              stats, s);
  if (dtype == SW_F64)
    return project_one<double>(fx, fy, fz, fs, g, dX, dY, dZ, tol, max_iters, out, ws, ws_bytes,
                               stats, s);
  set_error("projection: unknown dtype %d", dtype);
  return SW_EINVAL;
}

}  // namespace sw

using namespace sw;

extern "C" size_t sw_project_workspace_bytes(int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  return cg_workspace_bytes(g, cg_tiles(g));
}

extern "C" int sw_project(int in_dtype, const void* fx, const void* fy, const void* fz,
                          int64_t in_sx, int64_t in_sy, int64_t in_sz, int nx, int ny, int nz,
                          double dX, double dY, double dZ, double tol, int max_iters, double* out,
                          void* workspace, size_t workspace_bytes, sw_cg_stats* stats,
                          void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || out == nullptr) {
    set_error("sw_project: bad grid or null output");
    return SW_EINVAL;
  }
  if (!(dX > 0 && dY > 0 && dZ > 0)) {
    set_error("sw_project: grid spacing must be positive");
    return SW_EINVAL;
  }
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  InStride fs{in_sx, in_sy, in_sz};
  return project_field(in_dtype, fx, fy, fz, fs, g, dX, dY, dZ, tol, max_iters, out, workspace,
                       workspace_bytes, stats, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// batched projection: many independent solves advance together, one launch
// per CG phase over all their tiles
// ---------------------------------------------------------------------------
namespace {
struct BatchTableLayout {
  size_t inst, state, fin, strides, outs, grid, total;
};
BatchTableLayout batch_layout(int n) {
  BatchTableLayout L;
  size_t off = 0;
  L.inst = off;
  off += align_up((size_t)n * sizeof(CgInst), 256);
  L.state = off;
  off += align_up((size_t)n * sizeof(CgState), 256);
  L.fin = off;
  off += align_up((size_t)3 * n * sizeof(void*), 256);
  L.strides = off;
  off += align_up((size_t)n * sizeof(InStride), 256);
  L.outs = off;
  off += align_up((size_t)n * sizeof(double*), 256);
  L.grid = off;
  off += align_up(sizeof(CgGrid), 256);
  L.total = off;
  return L;
}

template <typename T>
int project_batch_t(const sw_project_job* jobs, int n, char* table, sw_cg_stats* stats,
                    cudaStream_t s) {
  const BatchTableLayout L = batch_layout(n);
  std::vector<CgInst> insts(n);
  std::vector<CgState> hst(n);
  std::vector<const void*> fin(3 * (size_t)n);
  std::vector<InStride> strides(n);
  std::vector<double*> outs(n);
  CgState* d_states = (CgState*)(table + L.state);
  int ntiles = 0;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < n; ++i) {
    const sw_project_job& j = jobs[i];
    Geom g = make_geom(j.nx, j.ny, j.nz, pad_pitch(j.nz));
    CgState* st_unused = nullptr;
    char* tail = nullptr;
    int rc = cg_layout(g, (char*)j.workspace, j.workspace_bytes, &insts[i], &st_unused, &tail);
    if (rc != SW_OK) return rc;
    insts[i].st = d_states + i;
    insts[i].c2x = 1.0 / (2.0 * j.dX);
    insts[i].c2y = 1.0 / (2.0 * j.dY);
    insts[i].c2z = 1.0 / (2.0 * j.dZ);
    insts[i].tile_base = ntiles;
    ntiles += insts[i].ts.count;
    hst[i] = CgState{};
    hst[i].tol = j.tol;
    hst[i].max_iters = j.max_iters;
    hst[i].reason = insts[i].ts.count > 0 ? SW_CG_RUNNING : SW_CG_EARLY_EXIT;
    fin[3 * i + 0] = j.fx;
    fin[3 * i + 1] = j.fy;
    fin[3 * i + 2] = j.fz;
    strides[i] = InStride{j.sx, j.sy, j.sz};
    outs[i] = j.out;
    const size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
    if (e == cudaSuccess) e = cudaMemsetAsync(insts[i].x, 0, 6 * vec, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(j.out, 0, (size_t)g.ncell * 3 * sizeof(double), s);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(table + L.inst, insts.data(), n * sizeof(CgInst), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_states, hst.data(), n * sizeof(CgState), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(table + L.fin, fin.data(), fin.size() * sizeof(void*),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(table + L.strides, strides.data(), n * sizeof(InStride),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(table + L.outs, outs.data(), n * sizeof(double*), cudaMemcpyHostToDevice,
                        s);
  if (e != cudaSuccess) return cuda_status(e, "batched projection setup");
  const CgInst* d_tab = (const CgInst*)(table + L.inst);
  if (ntiles > 0) {
    const int grid = std::max(1, std::min(ntiles, 148 * 8));
    cg_prep<T><<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, n, ntiles, (const T* const*)(table + L.fin),
                                                     (const InStride*)(table + L.strides));
    count_launches(1);
    SW_CHECK_LAUNCH("cg_prep (batch)");
    int rc = cg_run(d_tab, n, ntiles, d_states, n, (CgGrid*)(table + L.grid), s);
    if (rc != SW_OK) return rc;
    cg_finish<T><<<grid, dim3(TILE_Z, TILE_Y), 0, s>>>(d_tab, n, ntiles,
                                                       (const T* const*)(table + L.fin),
                                                       (const InStride*)(table + L.strides),
                                                       (double* const*)(table + L.outs));
    count_launches(1);
    SW_CHECK_LAUNCH("cg_finish (batch)");
  }
  e = cudaMemcpyAsync(hst.data(), d_states, n * sizeof(CgState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "batched projection readback");
  if (stats)
    for (int i = 0; i < n; ++i) {
      stats[i].iters = hst[i].iters;
      stats[i].reason = hst[i].reason;
      stats[i].rel = hst[i].rel;
      stats[i].max_div = hst[i].maxdiv;
    }
  return SW_OK;
}
}  // namespace

extern "C" size_t sw_project_batch_table_bytes(int n) {
  return n > 0 ? batch_layout(n).total : 0;
}

extern "C" int sw_project_batch(const sw_project_job* jobs, int n, void* table,
                                size_t table_bytes, sw_cg_stats* stats, void* stream) {
  if (n <= 0 || jobs == nullptr || table == nullptr) {
    set_error("sw_project_batch: bad arguments");
    return SW_EINVAL;
  }
  if (table_bytes < batch_layout(n).total) {
    set_error("sw_project_batch: table of %zu bytes, %zu required", table_bytes,
              batch_layout(n).total);
    return SW_EWORKSPACE;
  }
  const int dt = jobs[0].in_dtype;
  for (int i = 0; i < n; ++i) {
    const sw_project_job& j = jobs[i];
    if (j.in_dtype != dt || j.nx <= 0 || j.ny <= 0 || j.nz <= 0 || j.out == nullptr ||
        !(j.dX > 0 && j.dY > 0 && j.dZ > 0)) {
      set_error("sw_project_batch: job %d is invalid (dtype, grid, output or spacing)", i);
      return SW_EINVAL;
    }
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (dt == SW_F32) return project_batch_t<float>(jobs, n, (char*)table, stats, s);
  if (dt == SW_F64) return project_batch_t<double>(jobs, n, (char*)table, stats, s);
  set_error("sw_project_batch: unknown dtype %d", dt);
  return SW_EINVAL;
}

extern "C" int sw_static_solve(int dtype, const void* b, const void* mu, double mu_s,
                               int64_t sx, int64_t sy, int64_t sz, int nx, int ny, int nz,
                               double dX, double dY, double dZ, double tol, int max_iters,
                               double* out, void* workspace, size_t workspace_bytes,
                               sw_cg_stats* stats, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || out == nullptr || b == nullptr ||
      !(dX > 0 && dY > 0 && dZ > 0)) {
    set_error("sw_static_solve: bad grid, spacing or null pointer");
    return SW_EINVAL;
  }
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  InStride fs{sx, sy, sz};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    return static_one<float>(b, mu, mu_s, fs, g, dX, dY, dZ, tol, max_iters, out, workspace,
                             workspace_bytes, stats, s);
  if (dtype == SW_F64)
    return static_one<double>(b, mu, mu_s, fs, g, dX, dY, dZ, tol, max_iters, out, workspace,
                              workspace_bytes, stats, s);
  set_error("sw_static_solve: unknown dtype %d", dtype);
  return SW_EINVAL;
}
