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
  return __fmaf_rn(hz, sz, __fmaf_rn(hy, sy, __fmaf_rn(hx, sx, __fmul_rn(hc, c))));
}

// Packed FP32 pairs (sm_100 `.f32x2`: one instruction for both cells of a z
// pair, each half rounded to nearest as the scalar instruction rounds it).
// The pair kernels compute both cells with these and the direct kernel one
// cell with the scalar `__f*_rn` forms of the same sequence, so no result
// depends on which multiply-adds the compiler would have contracted.
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
// a * b + c with one rounding per half
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }

// lap7f on a z pair: sums of the x and y neighbour pairs, the z neighbour
// sums (z-1 + z+1 of each cell), the centre pair; the coefficients splatted.
struct Lap7Pair {
  float2 hx, hy, hz, hc;
};
__device__ __forceinline__ Lap7Pair lap7_pair_coefs(float hx, float hy, float hz, float hc) {
  return Lap7Pair{splat2(hx), splat2(hy), splat2(hz), splat2(hc)};
}
__device__ __forceinline__ float2 lap7f2(float2 sx, float2 sy, float2 sz, float2 c,
                                         const Lap7Pair& k) {
  return ffma2(k.hz, sz, ffma2(k.hy, sy, ffma2(k.hx, sx, fmul2(k.hc, c))));
}
// The 7-point Laplacian of a pair whose centre is C, with L and R the pairs
// either side in z, X and Xm the centre pairs of the next and previous
// planes, N and S the pairs of the rows either side.
__device__ __forceinline__ float2 lap7_pair(float2 C, float2 L, float2 R, float2 X, float2 Xm,
                                            float2 N, float2 S, const Lap7Pair& k) {
  const float2 sz = make_float2(__fadd_rn(C.y, L.y), __fadd_rn(R.x, C.x));
  return lap7f2(fadd2(X, Xm), fadd2(N, S), sz, C, k);
}

int make_step_args(const sw_fdtd_desc* d, StepArgs* a);
int launch_steps(const StepArgs& a, int it0, int nsteps, cudaStream_t s);

}  // namespace sw
