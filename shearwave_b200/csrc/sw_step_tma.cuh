// Internal interface of the TMA-staged step kernels (see sw_step_tma.cu).
#pragma once

#include <cuda.h>

#include "sw_common.cuh"
#include "sw_step.cuh"

namespace sw {

constexpr int round128(int bytes) { return (bytes + 127) / 128 * 128; }

// Kernel-side view of one mixed-form solve (state after t steps in buffer t mod 3).
// The output tile is tzw x tyh cells of the (z, y) plane: 64 x TY or
// 32 x 2TY (per launch, whichever wastes fewer lanes on the grids); a CTA
// has TY consumer warps, one tile row of 32 z pairs each (64-wide) or two
// rows of 16 (32-wide).
//   tm[b]  : state buffer b as a 4-D tensor (pz, ny, nx, 9 components);
//            box (tzw + 8, tyh + 2, 1, 6) = the halo'd u and d of one plane
//   tmc[b] : the same tensor, box (tzw, tyh, 1, 3) = the Kahan compensation
//   tmm    : material coefficients (pz, ny, nx, ncoef), box (tzw, tyh, 1, ncoef)
constexpr int kF32TileRows = 8;  // TY: rows of a 64-wide tile = consumer warps
// halo-box cells per component of a mixed-step tile of width tzw
constexpr int f32_box_cells(int tzw) { return (tzw + 8) * (64 * kF32TileRows / tzw + 2); }

struct TmaF32 {
  static constexpr int TZ = 64, TY = kF32TileRows;  // the 64-wide shape; tzw * tyh == TZ * TY
  static constexpr int PT = TZ * TY;                // cells of a point box (per component)
  static constexpr int box_cells(int tzw) { return f32_box_cells(tzw); }
  static constexpr int A_BYTES_MAX =
      (f32_box_cells(64) > f32_box_cells(32) ? f32_box_cells(64) : f32_box_cells(32)) * 6 * 4;
  static constexpr int C_BYTES = PT * 3 * 4;
  static constexpr int M_BYTES = PT * 2 * 4;
  static constexpr int A_STAGE = round128(A_BYTES_MAX);
  static constexpr int CONSUMER_WARPS = TY;
  static constexpr int THREADS = 32 * (CONSUMER_WARPS + 1);
  static constexpr int MIN_CTAS = TY <= 8 ? 2 : 1;  // resident CTAs per SM the layout allows
  CUtensorMap tm[3];
  CUtensorMap tmc[3];
  CUtensorMap tmm;
  Geom g;
  TileSpace ts;
  float* state[3];
  const float* pat;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  float hx, hy, hz, damp;
  int ncoef;  // 1: mu only, 2: mu and eta
  int use_damp, kahan, n_steps, snap_stride;
  int tzw, tyh;   // output tile shape: 64 x TY or 32 x 2 TY
  float* snaps;
  int* flags;
  int it_begin;   // launch step index of this solve's step 0
  int tile_base;  // first global tile of this solve in a batched launch
  int wait_k;     // wait budget, units of 1024 cycles (SW_TUNE_WAIT_BUDGET)
  int stall_test; // testing switch: sw_fdtd_desc.stall_test
};

// Kernel-side view of one plain-FP64 solve.
//   tm[b] : rotating buffer b as a 4-D tensor (pz, ny, nx, 3); box (W, H, 1, 3)
//   tmm   : material coefficients (pz, ny, nx, ncoef), box (TZ, TY, 1, ncoef)
struct TmaF64 {
  static constexpr int TZ = 32, TY = 8;
  static constexpr int W = TZ + 4;  // 2 cells of halo each side in z (16-byte aligned)
  static constexpr int H = TY + 2;
  static constexpr int NA = 5, NB = 3;  // planes x, x+1 held, three in flight
  static constexpr int BOX_BYTES = W * H * 3 * 8;        // one buffer's box
  static constexpr int HALF = round128(BOX_BYTES);        // u_prev box, then u_curr box
  static constexpr int A_STAGE = 2 * HALF;
  static constexpr int M_BYTES = TZ * TY * 2 * 8;
  static constexpr int B_STAGE = round128(M_BYTES);
  static constexpr int CONSUMER_WARPS = TY;
  static constexpr int THREADS = 32 * (CONSUMER_WARPS + 1);
  CUtensorMap tm[3];
  CUtensorMap tmm;
  Geom g;
  TileSpace ts;
  double* state[3];
  const double* ir;
  const double* pat;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  double ihx2, ihy2, ihz2, inv_dt, dt2, damp;
  int ncoef;
  int use_damp, n_steps, snap_stride;
  double* snaps;
  int* flags;
  int it_begin;
  int tile_base;
  int wait_k;
  int stall_test;
};

// Tile shapes of the two-steps-per-pass kernel (one per solve): output
// tiles of OZ x OY cells starting at z = OZ kz, y = OY ky; step t+1 is
// computed on the LZ x LY region around the tile (z from z0-2, y from y0-1:
// the tile plus one cell of halo, and one more column each side in z so
// that z pairs stay 8-byte aligned), step t+2 on the tile.  Each of the 15
// consumer warps owns RPW level-1 rows of LZ/2 z pairs:
//   LZ 64: one row of 32 pairs per warp, 64 x 15 -> 60 x 13 output cells;
//   LZ 32: two rows of 16 pairs per warp, 32 x 30 -> 28 x 28 output cells
//          (the narrower tile wastes less of a grid whose interior is not a
//          multiple of 60 cells wide).
//   level-0 box (u and d, 6 components): W x H from (z0-4, y0-2);
//   coefficient box: WB x HB from (z0-4, y0-1).
template <int LZ_>
struct TbShape {
  static constexpr int LZ = LZ_;
  static constexpr int PAIRS = LZ / 2;  // z pairs per level-1 row
  static constexpr int RPW = 64 / LZ;   // level-1 rows per consumer warp
  static constexpr int LY = 15 * RPW;
  static constexpr int OZ = LZ - 4, OY = LY - 2;
  static constexpr int W = LZ + 4, H = OY + 4;
  static constexpr int WB = LZ + 4, HB = LY;
};

constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Kernel-side view of one mixed-form solve for the two-steps-per-pass kernel
// (no compensated sum).  The ring stages are sized for either tile shape.
//   tm[b]  : state buffer b (pz, ny, nx, 9), box (W, H, 1, 6) of the shape
//   tmm    : coefficients (pz, ny, nx, ncoef), box (WB, HB, 1, ncoef)
struct TmaF32TB {
  // 15 consumer warps + the producer = 16 warps: four per scheduler, which
  // leaves each thread up to 128 registers (17 warps would cap it at 96)
  // ring stages: level 0 (planes q, q+1 held, two in flight), points (the
  // plane in use, one in flight: a third stage measured 3 % slower on a
  // config-3 batch), level 1
  static constexpr int NA = 4, NB = 2, NL = 3;
  static constexpr int A_STAGE =
      round128(cmax(TbShape<64>::W * TbShape<64>::H, TbShape<32>::W * TbShape<32>::H) * 6 * 4);
  static constexpr int B_STAGE = round128(
      cmax(TbShape<64>::WB * TbShape<64>::HB, TbShape<32>::WB * TbShape<32>::HB) * 2 * 4);
  static constexpr int L_STAGE = round128(
      cmax(TbShape<64>::LZ * TbShape<64>::LY, TbShape<32>::LZ * TbShape<32>::LY) * 6 * 4);
  static constexpr int CONSUMER_WARPS = 15;
  static constexpr int THREADS = 32 * (CONSUMER_WARPS + 1);
  CUtensorMap tm[3];
  CUtensorMap tmm;
  Geom g;
  TileSpace ts;  // z tiles of OZ, y tiles of OY, x chunks
  float* state[3];
  const float* pat;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  float hx, hy, hz, damp;
  int ncoef;
  int use_damp, n_steps, snap_stride;
  float* snaps;
  int* flags;
  int it_begin;
  int tile_base;
  int wait_k;
  int stall_test;
  int lz;  // this solve's tile shape (TbShape<lz>); a batched launch may mix them
};

size_t tma_smem_bytes(int precision);
size_t tb_smem_bytes();
// Two-step tile width for a grid (64 or 32; the SW_TUNE_TILE_SHAPE knob can
// force one) and the cells both levels compute for a width (tiles x region).
int tb_tile_width(const Geom& g);
long long tb_work(const Geom& g, int lz);
// lz 0: tb_tile_width(a.g)
int make_tma_f32_tb(const StepArgs& a, int xchunk, TmaF32TB* t, int lz);
int launch_fused2(const StepArgs& a, int xchunk, int it, cudaStream_t s);
int launch_fused2_prepare();                                   // kernel attributes, once
void launch_fused2_raw(const TmaF32TB& t, int it, cudaStream_t s);  // enqueue one launch
const void* step_f32_fused2_ptr(int lz);        // the single-solve fused kernel (graph nodes)
const void* step_f32_fused2_batch_ptr(int lz);  // the batched fused kernel (graph nodes)
int launch_fused2_batch(const void* d_tab, int ninst, int ntiles, int it, int* queues, int lz,
                        cudaStream_t s);
int tma_xchunk(const Geom& g, int tz, int ty, long long want_tiles);
// Mixed-step tile width for a grid (64 or 32; the SW_TUNE_TILE_SHAPE knob
// can force one) and the plane cells a tile width covers.
int f32_tile_width(const Geom& g);
long long f32_tile_cover(const Geom& g, int tzw);
// tzw 0: f32_tile_width(a.g)
int make_tma_f32(const StepArgs& a, int xchunk, TmaF32* t, int tzw);
int make_tma_f64(const StepArgs& a, int xchunk, TmaF64* t);
int launch_steps_tma(const StepArgs& a, int xchunk, int it0, int nsteps, cudaStream_t s);
int launch_steps_tma_batch(int precision, const void* d_tab, int ninst, int ntiles, int it,
                           int* queues, int tzw, bool kahan_ring, cudaStream_t s);

}  // namespace sw
