// Internal interface of the time-loop stage (see sw_step.cu).
#pragma once

#include "sw_common.cuh"

namespace sw {

// Kernel-side view of an sw_fdtd_desc (passed by value as a grid constant).
struct StepArgs {
  Geom g;
  TileSpace ts;
  int precision;
  void* state[3];
  const void* coef_m;
  const void* coef_e;
  const void* inv_rho;
  const void* patterns;
  const int* term_off;
  const int* term_pat;
  const double* term_scale;
  double ihx2, ihy2, ihz2;  // 1 / h^2
  double dT, inv_dt, dt2, damp;
  int use_damp, kahan, n_steps;
  int snap_stride;
  void* snaps;
  int n_traces;
  const int* trace_cells;
  void* traces;
  int* flags;
  int kernel;          // 0 TMA-staged, 1 direct loads
  int xchunk;          // requested planes per tile (0 automatic)
  int steps_per_pass;  // mixed form: 2 two steps per launch, 0 / 1 one
  int* clock;          // device step counter for graph replays (or null)
  int* queue;          // launch-wide tile queue of one-solve launches (or null)
  int stall_test;      // testing: leave one ring stage of every tile unarmed
};

// 7-point Laplacian of the mixed form from the three neighbour-pair sums
// (x+ + x-, y+ + y-, z+ + z-) and the centre value:
//   hx sx + hy sy + hz sz + hc c,  hc = -2 ((hx + hy) + hz),
// as one fixed chain of fused multiply-adds.  Every mixed-form kernel uses
// these two functions, so all of them agree bit for bit.
__device__ __forceinline__ float lap7_centre_coef(float hx, float hy, float hz) {
  return -2.0f * ((hx + hy) + hz);
}
__device__ __forceinline__ float lap7f(float sx, float sy, float sz, float c, float hx, float hy,
                                       float hz, float hc) {
  return fmaf(hz, sz, fmaf(hy, sy, fmaf(hx, sx, hc * c)));
}

int make_step_args(const sw_fdtd_desc* d, StepArgs* a);
int launch_steps(const StepArgs& a, int it0, int nsteps, cudaStream_t s);

}  // namespace sw
