// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a, in inline PTX.
//
// Only non-multicast tile loads are used: every tensor map covers this GPU's
// own memory.  Every wait on an mbarrier is bounded by a clock64 deadline;
// a wait that runs out sets bit 1 of the caller's error word and returns
// false instead of spinning forever.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sw {

__device__ inline uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ inline void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ inline void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive once (the producer) and announce `bytes` of transaction.
__device__ inline void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One potentially blocking test of phase `parity`: the thread may be
// suspended (without issuing instructions) until the phase completes or
// about 10 ms pass, so waiting warps leave the issue slots to working ones.
__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity), "r"(10000000u)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar` to complete, at most ~`budget` cycles.
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                         long long budget = 4000000000LL) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > budget) return false;
  }
  return true;
}

// 4-D tiled TMA load into shared memory, completion on `bar`.
__device__ inline void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0,
                                   int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_addr(bar))
      : "memory");
}

__device__ inline void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------------------
// warp-specialised pipeline pieces shared by the step kernels
// ---------------------------------------------------------------------------
// mbarrier arrive (no transaction), used by consumer warps to free a stage.
__device__ inline void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Shared-memory header of the warp-specialised kernels: the mbarriers at
// offset 0, the control words (abort flag, wait budget) at offset 192, the
// tile hand-off slots at 200, the abort log at 256, the rings from offset 384.
struct WsHeader {
  uint64_t fullA[6], emptyA[6], fullB[4], emptyB[4];  // 160 bytes
};
static_assert(sizeof(WsHeader) <= 192, "header overlaps the abort flag");
constexpr int kAbortFlagOffset = 192;
constexpr int kTileSlotOffset = 200;  // int tile[6], then int solve[6]
constexpr int kLogOffset = 256;
constexpr int kRingOffset = 384;
static_assert(kTileSlotOffset + 48 <= kLogOffset, "tile slots overlap the abort log");

// What a CTA needs to know, after an abort, about the tiles it had taken:
// the producer records the solve (table index) of every tile it takes and
// will load, in take order; each consumer warp counts the tiles it has
// finished.  Tiles from the smallest finished count to the taken count are
// incomplete, and so are their solves.  A ring holds at most a few tiles, so
// eight entries cover the window between the slowest warp and the producer.
struct AbortLog {
  int solve[8];  // solve of taken tile n at n & 7
  int n_taken;
  int done[16];  // tiles finished by consumer warp w
  // the stages of rings A and B that the producer armed with a copy, and the
  // phase parity of each stage's latest copy (one bit per stage)
  uint32_t armedA, parA, armedB, parB;
};
static_assert(kLogOffset + (int)sizeof(AbortLog) <= kRingOffset, "abort log overlaps the rings");
__device__ inline AbortLog* abort_log(unsigned char* base) {
  return reinterpret_cast<AbortLog*>(base + kLogOffset);
}

// Record that the producer armed stage s of a ring with a copy whose phase
// has parity ph.  After an abort the producer waits (bounded) for the latest
// phase of every armed stage, so that no copy is still landing in shared
// memory when the CTA exits.  The record lives in shared memory, so it holds
// no register in the consumers' loops.
__device__ inline void arm_record(uint32_t& armed, uint32_t& par, int s, uint32_t ph) {
  armed |= 1u << s;
  par = (par & ~(1u << s)) | (ph << s);
}
constexpr long long kDrainBudget = 1LL << 28;
__device__ inline void drain_ring(uint64_t* full, uint32_t armed, uint32_t par, int n) {
  for (int s = 0; s < n; ++s)
    if ((armed >> s) & 1u) (void)mbar_wait_bounded(&full[s], (par >> s) & 1u, kDrainBudget);
}

// Tile hand-off: the producer picks the CTA's tiles (a fixed stride over the
// tile range, or the next tile of a launch-wide queue) and writes the tile
// index and its solve's table index into the slots of the A stage that holds
// the tile's first plane, before arming that stage's full barrier (the
// barrier's release / acquire orders the slot write before the consumers'
// reads).  Tile -1 (a stage armed without a copy) ends the CTA's work.
__device__ inline volatile int* tile_slots(unsigned char* base) {
  return reinterpret_cast<volatile int*>(base + kTileSlotOffset);
}
__device__ inline volatile int* solve_slots(unsigned char* base) {
  return reinterpret_cast<volatile int*>(base + kTileSlotOffset + 24);
}

// Next tile of this CTA: a launch-wide queue (`queue`, batched launches;
// tiles of the solves with the longest columns come first, so the queue
// balances like longest-processing-time-first) or the fixed stride
// blockIdx.x + k gridDim.x.
__device__ inline int next_tile(int* queue, int& stride_next) {
  if (queue != nullptr) return atomicAdd(queue, 1);
  const int t = stride_next;
  stride_next += gridDim.x;
  return t;
}

// End of a CTA of a queue-fed launch: the last CTA to finish resets the
// launch-wide queue (queues[0]) and the finish count (queues[1]) for the next
// launch of the stream.  Every CTA has taken its last tile by then.
__device__ inline void queue_cta_done(int* queues) {
  if (queues == nullptr || threadIdx.x != 0) return;
  __threadfence();
  if (atomicAdd(queues + 1, 1) == (int)gridDim.x - 1) {
    atomicExch(queues, 0);
    atomicExch(queues + 1, 0);
  }
}

// Position in a ring of N stages: the stage index and the phase parity of
// its barriers, advanced without divisions.
template <int N>
struct RingPos {
  int s = 0;
  uint32_t ph = 0;
  __device__ inline void next() {
    if (++s == N) {
      s = 0;
      ph ^= 1u;
    }
  }
};

// Table index of the solve that owns global tile t (tile_base ascending).
template <typename Inst>
__device__ inline int find_solve(const Inst* __restrict__ tab, int ninst, int t) {
  int lo = 0, hi = ninst - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tab[mid].tile_base <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// A bounded wait that also gives up as soon as another thread has aborted.
// `abort_flag` points at the CTA's two control words in shared memory: the
// abort flag, then the wait budget in units of 1024 cycles (read only once a
// test has failed, so the budget costs the fast path no register).
__device__ inline bool ws_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  // 32-bit cycle counter: differences are exact below 2^32 cycles, and the
  // budget stays below that (at most 4e6 units of 1024 cycles, under the
  // 2^22 - 1 units a 32-bit difference can reach, so every wait can end)
  const uint32_t t0 = (uint32_t)clock();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort_flag) return false;
    if ((((uint32_t)clock() - t0) >> 10) > (uint32_t)abort_flag[1]) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// After an abort: set `bit` in the flags of every solve with a tile this CTA
// took and did not finish (all solves when the log cannot tell).  `flags_of(k)`
// gives solve k's flag word (or null).
template <typename FlagsOf>
__device__ inline void flag_unfinished(const AbortLog* lg, int nwarps, int ninst, int bit,
                                       FlagsOf flags_of) {
  int lo = lg->n_taken;
  for (int w = 0; w < nwarps; ++w) lo = min(lo, lg->done[w]);
  if (lg->n_taken - lo > 8 || lo < 0) {
    for (int k = 0; k < ninst; ++k)
      if (int* fl = flags_of(k)) atomicOr(fl, bit);
    return;
  }
  for (int n = lo; n < lg->n_taken; ++n)
    if (int* fl = flags_of(lg->solve[n & 7])) atomicOr(fl, bit);
}

// Whether a solve has already been abandoned in an earlier launch (its
// state is incomplete, so its remaining steps are skipped).
__device__ inline bool solve_abandoned(const int* flags) {
  return flags != nullptr && ((*reinterpret_cast<const volatile int*>(flags)) &
                              (kFlagTimeout | kFlagRefused)) != 0;
}

// Resolve the tile's instance and local step; false if the tile is idle.
template <typename Inst, bool BATCH>
__device__ inline bool resolve_tile(const Inst& one, const Inst* __restrict__ tab, int ninst,
                                    int t, int it, const Inst*& in, int& local, int& lit) {
  if (BATCH) {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (tab[mid].tile_base <= t) lo = mid;
      else hi = mid - 1;
    }
    in = &tab[lo];
    local = t - in->tile_base;
  } else {
    in = &one;
    local = t;
  }
  lit = it - in->it_begin;
  return lit >= 0 && lit < in->n_steps;
}

// Barrier among the consumer warps only (named barrier 1, `nthreads`
// threads), reducing a failure flag: returns true in every participant when
// any participant passed true.  The producer warp never joins it.
__device__ inline bool consumer_sync_or(bool fail, int nthreads) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)fail), "r"(nthreads)
      : "memory");
  return r != 0u;
}

// Host: encode a 4-D tiled tensor map (dims innermost first, strides in
// bytes for dims 1..3).  Returns a CUDA driver status.
int encode_tmap_4d(CUtensorMap* map, CUtensorMapDataType dt, void* base, const uint64_t dims[4],
                   const uint64_t strides_bytes[3], const uint32_t box[4]);

}  // namespace sw
