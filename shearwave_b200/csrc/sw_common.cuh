// Shared device-side helpers of the shearwave_b200 CUDA library (sm_100a).
//
// Data layout in HBM.  A scalar field on an (nx, ny, nz) grid is stored
// x-slowest / z-fastest, like the reference's C-ordered numpy arrays, with
// the z rows padded to a pitch `pz` (a multiple of 8 elements, so every row
// starts on a 32-byte sector for float and a 64-byte boundary for double).
// A vector field keeps its components as separate planes ("SoA"), component c
// at offset c * ncell with ncell = nx * ny * pz.  The one-voxel shell and the
// padding are zero and are never written by the time loop, so a kernel only
// ever updates interior cells 1..n-2 on every axis.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/shearwave_b200.h"

namespace sw {

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
struct Geom {
  int nx, ny, nz, pz;  // extents and padded z pitch (elements)
  long long sxy;       // plane stride = ny * pz
  long long ncell;     // component stride = nx * ny * pz
};

__host__ __device__ inline Geom make_geom(int nx, int ny, int nz, int pz) {
  Geom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.pz = pz;
  g.sxy = (long long)ny * pz;
  g.ncell = (long long)nx * g.sxy;
  return g;
}

__host__ __device__ inline int pad_pitch(int nz) { return (nz + 7) & ~7; }

// Solve flag bits (sw_fdtd_desc.flags): bit 0 a non-finite value, bit 1 a
// step kernel's bounded wait ran out and the CTA abandoned its tiles, bit 2
// a step launch refused to issue a TMA to a misaligned destination.
constexpr int kFlagNonFinite = 1, kFlagTimeout = 2, kFlagRefused = 4;

// Thread-block tile of the marching kernels: 32 cells along z (one warp, one
// coalesced 128 B / 256 B row segment) x TILE_Y rows along y; each thread
// marches along x over a chunk of planes.
constexpr int TILE_Z = 32;
constexpr int TILE_Y = 8;
constexpr int TILE_THREADS = TILE_Z * TILE_Y;

// Tile space of one instance: z tiles x y tiles x x chunks.  The tiles of all
// instances of a launch are numbered consecutively; `tile_base` is the first
// global tile index of the instance.
struct TileSpace {
  int ntz, nty, nxc, xc;  // tiles along z, y; x chunks and chunk length
  int count;              // ntz * nty * nxc
};

__host__ __device__ inline TileSpace make_tiles(const Geom& g, int xc) {
  TileSpace t;
  t.ntz = (g.nz + TILE_Z - 1) / TILE_Z;
  t.nty = (g.ny + TILE_Y - 1) / TILE_Y;
  int nxi = g.nx > 2 ? g.nx - 2 : 0;  // interior planes
  t.xc = xc < 1 ? 1 : xc;
  t.nxc = nxi > 0 ? (nxi + t.xc - 1) / t.xc : 0;
  t.count = t.ntz * t.nty * t.nxc;
  return t;
}

struct TileCoord {
  int z0, y0, x0, x1;  // z0/y0: first cell of the tile; [x0, x1): interior planes
};

__host__ __device__ inline TileCoord tile_coord(const Geom& g, const TileSpace& t, int local) {
  TileCoord c;
  int zt = local % t.ntz;
  int rest = local / t.ntz;
  int yt = rest % t.nty;
  int xt = rest / t.nty;
  c.z0 = zt * TILE_Z;
  c.y0 = yt * TILE_Y;
  c.x0 = 1 + xt * t.xc;
  int xe = c.x0 + t.xc;
  int xl = g.nx - 1;
  c.x1 = xe < xl ? xe : xl;
  return c;
}

// Tile space / coordinates for an arbitrary (tz, ty) output tile.
__host__ __device__ inline TileSpace make_tiles_t(const Geom& g, int xc, int tz, int ty) {
  TileSpace t;
  t.ntz = (g.nz + tz - 1) / tz;
  t.nty = (g.ny + ty - 1) / ty;
  int nxi = g.nx > 2 ? g.nx - 2 : 0;
  t.xc = xc < 1 ? 1 : xc;
  t.nxc = nxi > 0 ? (nxi + t.xc - 1) / t.xc : 0;
  t.count = t.ntz * t.nty * t.nxc;
  return t;
}

__host__ __device__ inline TileCoord tile_coord_t(const Geom& g, const TileSpace& t, int local,
                                                  int tz, int ty) {
  TileCoord c;
  int zt = local % t.ntz;
  int rest = local / t.ntz;
  int yt = rest % t.nty;
  int xt = rest / t.nty;
  c.z0 = zt * tz;
  c.y0 = yt * ty;
  c.x0 = 1 + xt * t.xc;
  int xe = c.x0 + t.xc;
  int xl = g.nx - 1;
  c.x1 = xe < xl ? xe : xl;
  return c;
}

// Chunk length along x so that a launch over one grid has roughly `want`
// tiles (at least one plane per chunk, at most the whole interior).
inline int choose_xchunk(const Geom& g, long long want) {
  long long ntz = (g.nz + TILE_Z - 1) / TILE_Z, nty = (g.ny + TILE_Y - 1) / TILE_Y;
  long long nxi = g.nx > 2 ? g.nx - 2 : 0;
  if (nxi == 0) return 1;
  long long per = ntz * nty;
  long long nchunks = (want + per - 1) / per;
  if (nchunks < 1) nchunks = 1;
  long long xc = (nxi + nchunks - 1) / nchunks;
  if (xc < 1) xc = 1;
  return (int)xc;
}

// ---------------------------------------------------------------------------
// Deterministic block reductions (fixed association for a fixed blockDim)
// ---------------------------------------------------------------------------
__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the block; result valid in thread 0.  `scratch` holds >= 32 doubles.
__device__ inline double block_sum(double v, double* scratch) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  v = warp_sum(v);
  __syncthreads();
  if ((tid & 31) == 0) scratch[tid >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (tid < 32) {
    r = tid < (nthr + 31) / 32 ? scratch[tid] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

__device__ inline double block_max(double v, double* scratch) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  v = warp_max(v);
  __syncthreads();
  if ((tid & 31) == 0) scratch[tid >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (tid < 32) {
    r = tid < (nthr + 31) / 32 ? scratch[tid] : 0.0;
    r = warp_max(r);
  }
  return r;
}

__device__ inline int flat_tid() { return threadIdx.x + threadIdx.y * blockDim.x; }

// Does (x, y, z) lie in the interior (mask == 1) of the grid?
__device__ inline bool interior(const Geom& g, int x, int y, int z) {
  return x >= 1 && y >= 1 && z >= 1 && x <= g.nx - 2 && y <= g.ny - 2 && z <= g.nz - 2;
}

// ---------------------------------------------------------------------------
// Host-side error plumbing
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
// Launch-shape knob (enum sw_tune_knob), process-wide.
int tune_get(int knob);
// Steps per pass of a mixed-form solve: its own setting (desc.steps_per_pass)
// when non-zero, else the SW_TUNE_STEPS_PER_PASS knob when non-zero, else two
// (batched or alone: configs 0, 1 and 2 alone ran 26 %, 25 % and 12 %
// faster than with one step per pass).
inline int steps_per_pass_of(int own, bool batched) {
  (void)batched;
  if (own != 0) return own;
  const int k = tune_get(SW_TUNE_STEPS_PER_PASS);
  if (k != 0) return k;
  return 2;
}
constexpr int kNumSMs = 148;  // B200
// CTA slots a step launch is sized for (SMs x CTAs per SM): the mixed
// kernel follows the SW_TUNE_STEP_CTAS_PER_SM knob, the plain FP64 kernel
// always fits two CTAs per SM.
inline int step_slots(bool mixed = true) {
  return kNumSMs * (mixed ? tune_get(SW_TUNE_STEP_CTAS_PER_SM) : 2);
}
int cuda_status(cudaError_t e, const char* what);
// Queue a host-to-device copy of a host-built table on stream s through a
// page-locked staging slot (src may be reused as soon as this returns).
int upload_staged(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Count kernels launched by this library (exported as sw_launch_count) and
// the host-side enqueue calls that launched them (sw_host_enqueue_count):
// `host` defaults to `n` (one call per kernel); a graph launch enqueues many
// kernels with one call.
void count_launches(unsigned long long n, unsigned long long host = ~0ull);

#define SW_CHECK_LAUNCH(what)                                   \
  do {                                                          \
    cudaError_t _e = cudaGetLastError();                        \
    if (_e != cudaSuccess) return ::sw::cuda_status(_e, what);  \
  } while (0)

template <typename T>
struct DType;
template <>
struct DType<float> {
  static constexpr int code = SW_F32;
};
template <>
struct DType<double> {
  static constexpr int code = SW_F64;
};

inline int grid_blocks(long long work, int per_block, int cap) {
  long long b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

}  // namespace sw
