// Internal interface of the TMA-staged step kernels (see sw_step_tma.cu).
#pragma once

#include <cuda.h>

#include "sw_common.cuh"
#include "sw_step.cuh"

namespace sw {

// Kernel-side view of one mixed-form solve.  The tensor maps cover the two
// FP32 state buffers as 4-D tensors (pz, ny, nx, 9 components).
struct TmaF32 {
  static constexpr int TZ = 64, TY = 8;    // output tile (z, y)
  static constexpr int W = TZ + 8;         // box width: 4 cells of halo each side in z
  static constexpr int H = TY + 2;         // box height: 1 row of halo each side in y
  static constexpr int NF = 6;             // halo'd components per plane: u, d
  static constexpr int NST = 4;            // plane stages in the ring
  static constexpr int PLANE = W * H * NF; // floats per stage (box of the one TMA load)
  static constexpr int STAGE = ((PLANE * 4 + 127) / 128) * 128 / 4;  // 128-byte aligned stride
  CUtensorMap tm[2];
  Geom g;
  TileSpace ts;
  float* state[2];
  const float* m;
  const float* e;
  const float* pat;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  float hx, hy, hz, damp;
  int use_damp, kahan, n_steps, snap_stride;
  float* snaps;
  int* flags;
  int it_begin;   // launch step index of this solve's step 0
  int tile_base;  // first global tile of this solve in a batched launch
};

// Kernel-side view of one plain-FP64 solve: three rotating buffers, each a
// 4-D tensor (pz, ny, nx, 3 components).
struct TmaF64 {
  static constexpr int TZ = 32, TY = 8;
  static constexpr int W = TZ + 4;  // 2 cells of halo each side in z (16-byte aligned)
  static constexpr int H = TY + 2;
  static constexpr int NF = 6;      // u_prev (3) then u_curr (3)
  static constexpr int NST = 4;
  static constexpr int PLANE = W * H * NF;  // doubles of the two boxes
  // each box lands on a 128-byte boundary (TMA destination alignment)
  static constexpr int HALF = ((W * H * 3 * 8 + 127) / 128) * 128 / 8;
  static constexpr int STAGE = 2 * HALF;
  CUtensorMap tm[3];
  Geom g;
  TileSpace ts;
  double* state[3];
  const double* m;
  const double* e;
  const double* ir;
  const double* pat;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  double ihx2, ihy2, ihz2, inv_dt, dt2, damp;
  int use_damp, n_steps, snap_stride;
  double* snaps;
  int* flags;
  int it_begin;
  int tile_base;
};

size_t tma_smem_bytes(int precision);
int tma_xchunk(const Geom& g, int tz, int ty, long long want_tiles);
int make_tma_f32(const StepArgs& a, int xchunk, TmaF32* t);
int make_tma_f64(const StepArgs& a, int xchunk, TmaF64* t);
int launch_steps_tma(const StepArgs& a, int xchunk, int it0, int nsteps, cudaStream_t s);
int launch_steps_tma_batch(int precision, const void* d_tab, int ninst, int ntiles, int it,
                           cudaStream_t s);

}  // namespace sw
