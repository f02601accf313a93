// Collocated FD operators and the strain post-pass.
//
// Reference: laplacian_center / divergence_center / gradient_center
// (src/shearwave/solver.py:686-729), compute_strain_tensor and
// compute_strain_invariants (src/shearwave/strain.py:16-135).
//
// These kernels reproduce numpy's elementwise rounding: every operation is a
// separately rounded IEEE operation in the array dtype (no FMA contraction,
// true division by the same divisor numpy uses), so their outputs equal the
// reference's bit for bit in float32 and float64.
#include <math.h>

#include <algorithm>

#include "sw_common.cuh"

namespace sw {

template <typename T>
struct Ar;
template <>
struct Ar<float> {
  static __device__ inline float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ inline float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ inline float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ inline float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ inline float sqrt_(float a) { return __fsqrt_rn(a); }
};
template <>
struct Ar<double> {
  static __device__ inline double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ inline double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ inline double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ inline double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ inline double sqrt_(double a) { return __dsqrt_rn(a); }
};

// A dense (nx, ny, nz) grid, z fastest.  The stencil kernels give each
// thread one (z, y) column of a 32 x 8 block and walk x across the grid's z
// dimension of blocks, so a cell's coordinates cost no division.
constexpr int kCellBlockZ = 32, kCellBlockY = 8;
struct Dense {
  int nx, ny, nz;
  __device__ inline bool inner(int x, int y, int z) const {
    return x >= 1 && y >= 1 && z >= 1 && x <= nx - 2 && y <= ny - 2 && z <= nz - 2;
  }
};

template <typename T>
__global__ void laplacian_kernel(const T* __restrict__ f, T* __restrict__ out, Dense d, T hx2,
                                 T hy2, T hz2) {
  using A = Ar<T>;
  const long long sx = (long long)d.ny * d.nz, sy = d.nz;
  const int z = blockIdx.x * kCellBlockZ + threadIdx.x, y = blockIdx.y * kCellBlockY + threadIdx.y;
  if (z >= d.nz || y >= d.ny) return;
  for (int x = blockIdx.z; x < d.nx; x += gridDim.z) {
    {
      const long long q = ((long long)x * d.ny + y) * d.nz + z;
      T r = T(0);
      if (d.inner(x, y, z)) {
        const T c2 = A::mul(T(2), f[q]);
        const T tx = A::div(A::add(A::sub(f[q + sx], c2), f[q - sx]), hx2);
        const T ty = A::div(A::add(A::sub(f[q + sy], c2), f[q - sy]), hy2);
        const T tz = A::div(A::add(A::sub(f[q + 1], c2), f[q - 1]), hz2);
        r = A::add(A::add(tx, ty), tz);
      }
      out[q] = r;
    }
  }
}

template <typename T>
__global__ void divergence_kernel(const T* __restrict__ fx, const T* __restrict__ fy,
                                  const T* __restrict__ fz, T* __restrict__ out, Dense d, T h2x,
                                  T h2y, T h2z) {
  using A = Ar<T>;
  const long long sx = (long long)d.ny * d.nz, sy = d.nz;
  const int z = blockIdx.x * kCellBlockZ + threadIdx.x, y = blockIdx.y * kCellBlockY + threadIdx.y;
  if (z >= d.nz || y >= d.ny) return;
  for (int x = blockIdx.z; x < d.nx; x += gridDim.z) {
    {
      const long long q = ((long long)x * d.ny + y) * d.nz + z;
      T r = T(0);
      if (d.inner(x, y, z)) {
        const T tx = A::div(A::sub(fx[q + sx], fx[q - sx]), h2x);
        const T ty = A::div(A::sub(fy[q + sy], fy[q - sy]), h2y);
        const T tz = A::div(A::sub(fz[q + 1], fz[q - 1]), h2z);
        r = A::add(A::add(tx, ty), tz);
      }
      out[q] = r;
    }
  }
}

template <typename T>
__global__ void gradient_kernel(const T* __restrict__ p, T* __restrict__ gx, T* __restrict__ gy,
                                T* __restrict__ gz, Dense d, T h2x, T h2y, T h2z) {
  using A = Ar<T>;
  const long long sx = (long long)d.ny * d.nz, sy = d.nz;
  const int z = blockIdx.x * kCellBlockZ + threadIdx.x, y = blockIdx.y * kCellBlockY + threadIdx.y;
  if (z >= d.nz || y >= d.ny) return;
  for (int x = blockIdx.z; x < d.nx; x += gridDim.z) {
    {
      const long long q = ((long long)x * d.ny + y) * d.nz + z;
      T a = T(0), b = T(0), c = T(0);
      if (d.inner(x, y, z)) {
        a = A::div(A::sub(p[q + sx], p[q - sx]), h2x);
        b = A::div(A::sub(p[q + sy], p[q - sy]), h2y);
        c = A::div(A::sub(p[q + 1], p[q - 1]), h2z);
      }
      gx[q] = a;
      gy[q] = b;
      gz[q] = c;
    }
  }
}

// Invariants of one Voigt vector, in the reference's operation order
// (strain.py:110-128).  von Mises is float64: numpy multiplies the dtype
// `dev` by the float64 scalar sqrt(2/3).
template <typename T>
__device__ inline void invariants(const T e[6], T& vol, T& dev, T& msh, double& vm) {
  using A = Ar<T>;
  vol = A::div(A::add(A::add(e[0], e[1]), e[2]), T(3));
  const T dxx = A::sub(e[0], vol), dyy = A::sub(e[1], vol), dzz = A::sub(e[2], vol);
  const T nrm = A::add(A::add(A::mul(dxx, dxx), A::mul(dyy, dyy)), A::mul(dzz, dzz));
  const T shr = A::mul(T(0.5), A::add(A::add(A::mul(e[3], e[3]), A::mul(e[4], e[4])),
                                      A::mul(e[5], e[5])));
  const T s = A::add(nrm, shr);
  dev = A::sqrt_(s);
  const T j2 = A::mul(T(0.5), s);
  msh = A::sqrt_(j2 > T(0) ? j2 : T(0));
  vm = __dmul_rn(__dsqrt_rn(2.0 / 3.0), (double)dev);
}

template <typename T>
__global__ void strain_kernel(const T* __restrict__ ux, const T* __restrict__ uy,
                              const T* __restrict__ uz, long long sx, long long sy, long long sz,
                              Dense d, T h2x, T h2y, T h2z, T* __restrict__ eps,
                              T* __restrict__ vol, T* __restrict__ dev, T* __restrict__ msh,
                              double* __restrict__ vm) {
  using A = Ar<T>;
  const int z = blockIdx.x * kCellBlockZ + threadIdx.x, y = blockIdx.y * kCellBlockY + threadIdx.y;
  if (z >= d.nz || y >= d.ny) return;
  for (int x = blockIdx.z; x < d.nx; x += gridDim.z) {
    {
      const long long q = ((long long)x * d.ny + y) * d.nz + z;
      T e[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
      if (d.inner(x, y, z)) {
        const long long i = x * sx + y * sy + z * sz;
        // g[a][b] = d u_a / d x_b
        const T* u[3] = {ux, uy, uz};
        T g[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          g[a][0] = A::div(A::sub(u[a][i + sx], u[a][i - sx]), h2x);
          g[a][1] = A::div(A::sub(u[a][i + sy], u[a][i - sy]), h2y);
          g[a][2] = A::div(A::sub(u[a][i + sz], u[a][i - sz]), h2z);
        }
        e[0] = g[0][0];
        e[1] = g[1][1];
        e[2] = g[2][2];
        e[3] = A::add(g[1][2], g[2][1]);
        e[4] = A::add(g[0][2], g[2][0]);
        e[5] = A::add(g[0][1], g[1][0]);
      }
      if (eps) {
#pragma unroll
        for (int k = 0; k < 6; ++k) eps[6 * q + k] = e[k];
      }
      if (vol || dev || msh || vm) {
        T a, b, c;
        double v;
        invariants<T>(e, a, b, c, v);
        if (vol) vol[q] = a;
        if (dev) dev[q] = b;
        if (msh) msh[q] = c;
        if (vm) vm[q] = v;
      }
    }
  }
}

template <typename T>
__global__ void invariants_kernel(const T* __restrict__ eps, long long n, T* __restrict__ vol,
                                  T* __restrict__ dev, T* __restrict__ msh,
                                  double* __restrict__ vm) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    T e[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) e[k] = eps[6 * q + k];
    T a, b, c;
    double v;
    invariants<T>(e, a, b, c, v);
    if (vol) vol[q] = a;
    if (dev) dev[q] = b;
    if (msh) msh[q] = c;
    if (vm) vm[q] = v;
  }
}

static bool bad_grid(int nx, int ny, int nz) { return nx <= 0 || ny <= 0 || nz <= 0; }

}  // namespace sw

using namespace sw;

namespace {
// numpy's divisors: h**2 and 2.0*h computed in double, then cast to the dtype
template <typename T>
T sq(double h) {
  return (T)(h * h);
}
template <typename T>
T twice(double h) {
  return (T)(2.0 * h);
}
int blocks_for(long long n) { return grid_blocks(n, 256, 148 * 32); }
// blocks of 32 (z) x 8 (y) threads, one x plane per block in z (up to 65535)
dim3 cell_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nz + kCellBlockZ - 1) / kCellBlockZ),
              (unsigned)((ny + kCellBlockY - 1) / kCellBlockY), (unsigned)std::min(nx, 65535));
}
const dim3 kCellBlock(kCellBlockZ, kCellBlockY);
}  // namespace

extern "C" int sw_laplacian(int dtype, const void* f, void* out, int nx, int ny, int nz,
                            double dX, double dY, double dZ, void* stream) {
  if (bad_grid(nx, ny, nz) || !f || !out) {
    set_error("sw_laplacian: bad arguments");
    return SW_EINVAL;
  }
  Dense d{nx, ny, nz};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    laplacian_kernel<float><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const float*)f, (float*)out, d, sq<float>(dX), sq<float>(dY), sq<float>(dZ));
  else if (dtype == SW_F64)
    laplacian_kernel<double><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const double*)f, (double*)out, d, sq<double>(dX), sq<double>(dY), sq<double>(dZ));
  else {
    set_error("sw_laplacian: unknown dtype");
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("laplacian");
  return SW_OK;
}

extern "C" int sw_divergence(int dtype, const void* fx, const void* fy, const void* fz, void* out,
                             int nx, int ny, int nz, double dX, double dY, double dZ,
                             void* stream) {
  if (bad_grid(nx, ny, nz) || !fx || !fy || !fz || !out) {
    set_error("sw_divergence: bad arguments");
    return SW_EINVAL;
  }
  Dense d{nx, ny, nz};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    divergence_kernel<float><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const float*)fx, (const float*)fy, (const float*)fz, (float*)out, d, twice<float>(dX),
        twice<float>(dY), twice<float>(dZ));
  else if (dtype == SW_F64)
    divergence_kernel<double><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const double*)fx, (const double*)fy, (const double*)fz, (double*)out, d,
        twice<double>(dX), twice<double>(dY), twice<double>(dZ));
  else {
    set_error("sw_divergence: unknown dtype");
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("divergence");
  return SW_OK;
}

extern "C" int sw_gradient(int dtype, const void* phi, void* gx, void* gy, void* gz, int nx,
                           int ny, int nz, double dX, double dY, double dZ, void* stream) {
  if (bad_grid(nx, ny, nz) || !phi || !gx || !gy || !gz) {
    set_error("sw_gradient: bad arguments");
    return SW_EINVAL;
  }
  Dense d{nx, ny, nz};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    gradient_kernel<float><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const float*)phi, (float*)gx, (float*)gy, (float*)gz, d, twice<float>(dX),
        twice<float>(dY), twice<float>(dZ));
  else if (dtype == SW_F64)
    gradient_kernel<double><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const double*)phi, (double*)gx, (double*)gy, (double*)gz, d, twice<double>(dX),
        twice<double>(dY), twice<double>(dZ));
  else {
    set_error("sw_gradient: unknown dtype");
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("gradient");
  return SW_OK;
}

extern "C" int sw_strain(int dtype, const void* ux, const void* uy, const void* uz, int64_t sx,
                         int64_t sy, int64_t sz, int nx, int ny, int nz, double dX, double dY,
                         double dZ, void* eps, void* vol, void* dev, void* max_shear,
                         double* von_mises, void* stream) {
  if (bad_grid(nx, ny, nz) || !ux || !uy || !uz) {
    set_error("sw_strain: bad arguments");
    return SW_EINVAL;
  }
  if (!(dX > 0 && dY > 0 && dZ > 0)) {
    set_error("sw_strain: grid spacing must be positive");
    return SW_EINVAL;
  }
  Dense d{nx, ny, nz};
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    strain_kernel<float><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const float*)ux, (const float*)uy, (const float*)uz, sx, sy, sz, d, twice<float>(dX),
        twice<float>(dY), twice<float>(dZ), (float*)eps, (float*)vol, (float*)dev,
        (float*)max_shear, von_mises);
  else if (dtype == SW_F64)
    strain_kernel<double><<<cell_grid(nx, ny, nz), kCellBlock, 0, s>>>(
        (const double*)ux, (const double*)uy, (const double*)uz, sx, sy, sz, d,
        twice<double>(dX), twice<double>(dY), twice<double>(dZ), (double*)eps, (double*)vol,
        (double*)dev, (double*)max_shear, von_mises);
  else {
    set_error("sw_strain: unknown dtype");
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("strain");
  return SW_OK;
}

extern "C" int sw_strain_invariants(int dtype, const void* eps, int64_t n, void* vol, void* dev,
                                    void* max_shear, double* von_mises, void* stream) {
  if (n < 0 || (n > 0 && !eps)) {
    set_error("sw_strain_invariants: bad arguments");
    return SW_EINVAL;
  }
  if (n == 0) return SW_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == SW_F32)
    invariants_kernel<float><<<blocks_for(n), 256, 0, s>>>((const float*)eps, n, (float*)vol,
                                                           (float*)dev, (float*)max_shear,
                                                           von_mises);
  else if (dtype == SW_F64)
    invariants_kernel<double><<<blocks_for(n), 256, 0, s>>>((const double*)eps, n, (double*)vol,
                                                            (double*)dev, (double*)max_shear,
                                                            von_mises);
  else {
    set_error("sw_strain_invariants: unknown dtype");
    return SW_EINVAL;
  }
  count_launches(1);
  SW_CHECK_LAUNCH("strain invariants");
  return SW_OK;
}
