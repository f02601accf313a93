// Direct (spectral) solve of the projection's Poisson problem.
//
// The CG of src/shearwave/solver.py:1010-1050 inverts A = -div_c(grad_c .)
// with both central differences zeroed on the one-voxel shell.  Restricted to
// interior cells, A is a sum over axes of one-dimensional operators
//     A = A_x (x) I (x) I + I (x) A_y (x) I + I (x) I (x) A_z,
// because the gradient's shell mask along an axis only depends on the
// coordinate along that axis for the rows that matter.  Each 1-D operator is
// 1/(4h^2) times a matrix that couples index i to i+-2 only, i.e. two
// independent tridiagonal chains (even and odd grid indices) with -1
// off-diagonals, 2 on the diagonal, and 1 at a chain end that sits on grid
// index 1 or n-2 (the gradient term through the shell is dropped: a
// Neumann-like end) or 2 at an end next to the zero shell (Dirichlet).  The
// eigenvectors of such chains are the discrete sine / cosine bases, so
//     phi = Q_x Q_y Q_z  diag(1 / (lx_i + ly_j + lz_k))  Q_z^T Q_y^T Q_x^T rhs
// solves the problem exactly (pseudo-inverse on the constant modes of the
// all-Neumann sub-lattices, which is the solution CG converges to).
//
// The mixed form uses this exact solve in FP64: ~6 dense per-axis transforms
// instead of hundreds of CG iterations.  The plain FP64 form keeps the CG,
// whose truncated iterate is what the reference returns.
#include <math.h>

#include <algorithm>
#include <vector>

#include "sw_common.cuh"
#include "sw_project.cuh"

namespace sw {

// ---------------------------------------------------------------------------
// basis of one axis (host, closed form)
// ---------------------------------------------------------------------------
// Q (m x m, row-major Q[i*m + k]: interior index i = grid index i+1, mode k)
// and lam[k] (physical eigenvalues, 1/(4 h^2) included).  The interior
// indices form two chains, the even grid indices (columns 0..K0-1) and the
// odd ones (columns K0..); an entry is non-zero only where its row and
// column lie on the same chain.  One entry at a time, so that the host entry
// point and the device kernel share the formulas; `lam` (when not null)
// receives the column's eigenvalue.
__host__ __device__ inline double basis_entry(int n, double h, int row, int col, double* lam) {
  const int first0 = 2, first1 = 1;
  const int K0 = first0 > n - 2 ? 0 : (n - 2 - first0) / 2 + 1;
  const int par = col < K0 ? 0 : 1;
  const int first = par == 0 ? first0 : first1;
  const int k = par == 0 ? col : col - K0;
  const int last = first + 2 * ((n - 2 - first) / 2);
  const int K = (last - first) / 2 + 1;
  const bool nf = (first == 1), nl = (last == n - 2);  // Neumann-like ends
  if (lam != nullptr) {
    double lk;
    if (nf && nl) lk = 2.0 - 2.0 * cos(k * M_PI / K);
    else if (!nf && !nl) lk = 2.0 - 2.0 * cos((k + 1.0) * M_PI / (K + 1));
    else lk = 2.0 - 2.0 * cos((k + 0.5) * M_PI / (K + 0.5));
    *lam = lk * (1.0 / (4.0 * h * h));
  }
  const int gi = row + 1;  // grid index of the row
  if ((gi & 1) != (first & 1)) return 0.0;
  const int j = (gi - first) / 2;  // chain position
  if (nf && nl) {                  // N-N: cosines, k = 0..K-1
    const double c = (k == 0) ? sqrt(1.0 / K) : sqrt(2.0 / K);
    return c * cos((j + 0.5) * k * M_PI / K);
  }
  if (!nf && !nl)  // D-D: sines, k = 1..K
    return sqrt(2.0 / (K + 1)) * sin((j + 1.0) * (k + 1.0) * M_PI / (K + 1));
  const int jj = nf ? j : (K - 1 - j);  // one Neumann end: distance from it
  return sqrt(2.0 / (K + 0.5)) * cos((jj + 0.5) * (k + 0.5) * M_PI / (K + 0.5));
}

// The solve builds its bases on the device, one thread per entry (the host
// would spend ~1 ms per solve on the m^2 cosines, with the GPU waiting).
__global__ void axis_basis_kernel(int n, double h, double* __restrict__ Q,
                                  double* __restrict__ lam) {
  const int m = n - 2;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m <= 0 || e >= (long long)m * m) return;
  const int row = (int)(e / m), col = (int)(e % m);
  Q[e] = basis_entry(n, h, row, col, row == 0 ? lam + col : nullptr);
}

// ---------------------------------------------------------------------------
// strided batched FP64 GEMM: C = A B
// ---------------------------------------------------------------------------
struct Mat {
  const double* p;
  long long rs, cs, bs;  // row, column and batch strides (elements)
};

constexpr int GB_M = 64, GB_N = 64, GB_K = 16;

__global__ void __launch_bounds__(256) gemm_f64(Mat A, Mat B, double* C, long long crs,
                                                long long ccs, long long cbs, int M, int N,
                                                int K) {
  __shared__ double As[GB_K][GB_M + 1];
  __shared__ double Bs[GB_K][GB_N + 1];
  const int b = blockIdx.z;
  const double* Ab = A.p + b * A.bs;
  const double* Bb = B.p + b * B.bs;
  double* Cb = C + b * cbs;
  const int m0 = blockIdx.y * GB_M, n0 = blockIdx.x * GB_N;
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  double acc[4][4] = {};
  const bool a_rowmajor = (A.cs == 1);
  const bool b_rowmajor = (B.cs == 1);
  for (int k0 = 0; k0 < K; k0 += GB_K) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int e = t + 256 * q;
      int r, c;  // A tile element (r in M, c in K)
      if (a_rowmajor) {
        r = e / GB_K;
        c = e % GB_K;
      } else {
        r = e % GB_M;
        c = e / GB_M;
      }
      const int gr = m0 + r, gc = k0 + c;
      As[c][r] = (gr < M && gc < K) ? Ab[gr * A.rs + gc * A.cs] : 0.0;
      int rb, cb;  // B tile element (rb in K, cb in N)
      if (b_rowmajor) {
        rb = e / GB_N;
        cb = e % GB_N;
      } else {
        rb = e % GB_K;
        cb = e / GB_K;
      }
      const int gk = k0 + rb, gn = n0 + cb;
      Bs[rb][cb] = (gk < K && gn < N) ? Bb[gk * B.rs + gn * B.cs] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GB_K; ++kk) {
      double a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = m0 + ty * 4 + i;
    if (gr >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx * 4 + j;
      if (gn < N) Cb[gr * crs + gn * ccs] = acc[i][j];
    }
  }
}

// b_hat /= (lx_i + ly_j + lz_k) on interior cells; zero on the null modes
__global__ void spectral_scale(double* v, Geom g, const double* __restrict__ lx,
                               const double* __restrict__ ly, const double* __restrict__ lz,
                               double lam_floor) {
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % (g.nz - 2));
    const long long r = q / (g.nz - 2);
    const int j = (int)(r % (g.ny - 2));
    const int i = (int)(r / (g.ny - 2));
    const long long idx = (long long)(i + 1) * g.sxy + (long long)(j + 1) * g.pz + (k + 1);
    const double L = lx[i] + ly[j] + lz[k];
    v[idx] = (L > lam_floor) ? v[idx] / L : 0.0;
  }
}

static int launch_gemm(Mat A, Mat B, double* C, long long crs, long long ccs, long long cbs,
                       int M, int N, int K, int batch, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return SW_OK;
  dim3 grid((N + GB_N - 1) / GB_N, (M + GB_M - 1) / GB_M, batch);
  gemm_f64<<<grid, 256, 0, s>>>(A, B, C, crs, ccs, cbs, M, N, K);
  count_launches(1);
  SW_CHECK_LAUNCH("spectral transform");
  return SW_OK;
}

// Transform along `axis` (0 x, 1 y, 2 z) of the padded field src into dst:
// forward (dst = Q^T src) or inverse (dst = Q src) on interior indices.
static int axis_transform(const Geom& g, int axis, const double* Q, bool forward,
                          const double* src, double* dst, cudaStream_t s) {
  const int nax = axis == 0 ? g.nx : (axis == 1 ? g.ny : g.nz);
  const int m = nax - 2;
  if (m <= 0) return SW_OK;
  // operator as an m x m matrix: forward uses Q^T (row k, col i) = Q[i*m + k]
  Mat Op;
  Op.p = Q;
  Op.bs = 0;
  if (forward) {
    Op.rs = 1;
    Op.cs = m;
  } else {
    Op.rs = m;
    Op.cs = 1;
  }
  if (axis == 0) {  // C[k][l] = Op[k][i] D[i+1][l], l over all (y, z)
    Mat D{src + g.sxy, g.sxy, 1, 0};
    return launch_gemm(Op, D, dst + g.sxy, g.sxy, 1, 0, m, (int)g.sxy, m, 1, s);
  }
  if (axis == 1) {  // per x plane: C[k][z] = Op[k][j] D[x][j+1][z]
    Mat D{src + g.pz, g.pz, 1, g.sxy};
    return launch_gemm(Op, D, dst + g.pz, g.pz, 1, g.sxy, m, g.pz, m, g.nx, s);
  }
  // axis z: C[l][k] = D[l][i+1] Op^T[i][k], l over all (x, y) lines
  Mat D{src + 1, g.pz, 1, 0};
  Mat OpT;  // (i, k) -> Op[k][i]
  OpT.p = Q;
  OpT.bs = 0;
  OpT.rs = Op.cs;
  OpT.cs = Op.rs;
  return launch_gemm(D, OpT, dst + 1, g.pz, 1, 0, g.nx * g.ny, m, m, 1, s);
}

size_t spectral_extra_bytes(const Geom& g) {
  size_t b = 0;
  const int ns[3] = {g.nx, g.ny, g.nz};
  for (int a = 0; a < 3; ++a) {
    const size_t m = ns[a] > 2 ? ns[a] - 2 : 1;
    b += align_up(m * m * sizeof(double), 256) + align_up(m * sizeof(double), 256);
  }
  return b;
}

}  // namespace sw

using namespace sw;

namespace {

template <typename T>
__global__ void prep_rhs(const T* __restrict__ fx, const T* __restrict__ fy,
                         const T* __restrict__ fz, InStride s, Geom g, double c2x, double c2y,
                         double c2z, double* __restrict__ rhs, double* __restrict__ maxdiv) {
  // rhs = -div_c(mask f) on interior cells (the CG's r0); also max |div|
  double mx = 0.0;
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  auto ld = [&](const T* f, int x, int y, int z) -> double {
    if (f == nullptr || !interior(g, x, y, z)) return 0.0;
    return (double)f[(long long)x * s.sx + (long long)y * s.sy + (long long)z * s.sz];
  };
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = 1 + (int)(q % (g.nz - 2));
    const long long r = q / (g.nz - 2);
    const int y = 1 + (int)(r % (g.ny - 2));
    const int x = 1 + (int)(r / (g.ny - 2));
    const double tx = (ld(fx, x + 1, y, z) - ld(fx, x - 1, y, z)) * c2x;
    const double ty = (ld(fy, x, y + 1, z) - ld(fy, x, y - 1, z)) * c2y;
    const double tz = (ld(fz, x, y, z + 1) - ld(fz, x, y, z - 1)) * c2z;
    const double div = (tx + ty) + tz;
    rhs[(long long)x * g.sxy + (long long)y * g.pz + z] = -div;
    mx = fmax(mx, fabs(div));
  }
  // block max, then one atomic per block on the bit pattern (non-negative doubles)
  __shared__ double red[32];
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x + 31) / 32 ? red[threadIdx.x] : 0.0;
    v = warp_max(v);
    if (threadIdx.x == 0)
      atomicMax((unsigned long long*)maxdiv, (unsigned long long)__double_as_longlong(v));
  }
}

template <typename T>
__global__ void finish_spectral(const T* __restrict__ fx, const T* __restrict__ fy,
                                const T* __restrict__ fz, InStride s, Geom g, double c2x,
                                double c2y, double c2z, const double* __restrict__ phi,
                                double* __restrict__ out) {
  const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int z = 1 + (int)(q % (g.nz - 2));
    const long long r = q / (g.nz - 2);
    const int y = 1 + (int)(r % (g.ny - 2));
    const int x = 1 + (int)(r / (g.ny - 2));
    const long long i = (long long)x * g.sxy + (long long)y * g.pz + z;
    const long long f = (long long)x * s.sx + (long long)y * s.sy + (long long)z * s.sz;
    const double gx = (phi[i + g.sxy] - phi[i - g.sxy]) * c2x;
    const double gy = (phi[i + g.pz] - phi[i - g.pz]) * c2y;
    const double gz = (phi[i + 1] - phi[i - 1]) * c2z;
    out[i] = (fx ? (double)fx[f] : 0.0) - gx;
    out[i + g.ncell] = (fy ? (double)fy[f] : 0.0) - gy;
    out[i + 2 * g.ncell] = (fz ? (double)fz[f] : 0.0) - gz;
  }
}

template <typename T>
int spectral_one(const void* fx, const void* fy, const void* fz, InStride fs, const Geom& g,
                 double dX, double dY, double dZ, double* out, char* ws, size_t ws_bytes,
                 sw_cg_stats* stats, cudaStream_t s) {
  const size_t vec = align_up((size_t)g.ncell * sizeof(double), 256);
  const size_t need = 3 * vec + spectral_extra_bytes(g) + 256;
  if (ws == nullptr || ws_bytes < need) {
    set_error("spectral workspace of %zu bytes is smaller than the %zu bytes required", ws_bytes,
              need);
    return SW_EWORKSPACE;
  }
  double* v0 = (double*)ws;
  double* v1 = (double*)(ws + vec);
  double* v2 = (double*)(ws + 2 * vec);
  char* p = ws + 3 * vec;
  const int ns[3] = {g.nx, g.ny, g.nz};
  const double hs[3] = {dX, dY, dZ};
  double* Q[3];
  double* L[3];
  cudaError_t e = cudaSuccess;
  for (int a = 0; a < 3; ++a) {
    const int m = ns[a] > 2 ? ns[a] - 2 : 1;
    Q[a] = (double*)p;
    p += align_up((size_t)m * m * sizeof(double), 256);
    L[a] = (double*)p;
    p += align_up((size_t)m * sizeof(double), 256);
    if (ns[a] > 2) {
      const long long cnt = (long long)m * m;
      axis_basis_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(ns[a], hs[a], Q[a], L[a]);
      count_launches(1);
      SW_CHECK_LAUNCH("spectral basis");
    }
  }
  double* d_max = (double*)p;
  if (e == cudaSuccess) e = cudaMemsetAsync(ws, 0, 3 * vec, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_max, 0, sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, (size_t)g.ncell * 3 * sizeof(double), s);
  if (e != cudaSuccess) return cuda_status(e, "spectral setup");
  double maxdiv = 0.0;
  const bool has_interior = g.nx > 2 && g.ny > 2 && g.nz > 2;
  const double c2x = 1.0 / (2.0 * dX), c2y = 1.0 / (2.0 * dY), c2z = 1.0 / (2.0 * dZ);
  if (has_interior) {
    const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
    const int grid = grid_blocks(n, 256, 148 * 16);
    prep_rhs<T><<<grid, 256, 0, s>>>((const T*)fx, (const T*)fy, (const T*)fz, fs, g, c2x, c2y,
                                     c2z, v0, d_max);
    count_launches(1);
    SW_CHECK_LAUNCH("spectral prep");
    e = cudaMemcpyAsync(&maxdiv, d_max, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, "spectral readback");
  }
  const bool solve = has_interior && !(maxdiv < 1e-12);
  if (solve) {
    // v0 -> v1 (x) -> v2 (y) -> v1 (z), scale, v1 -> v2 (z) -> v1 (y) -> v2 (x)
    int rc = axis_transform(g, 0, Q[0], true, v0, v1, s);
    if (rc == SW_OK) rc = axis_transform(g, 1, Q[1], true, v1, v2, s);
    if (rc == SW_OK) rc = axis_transform(g, 2, Q[2], true, v2, v1, s);
    if (rc != SW_OK) return rc;
    double lmax = 0.0;
    for (int a = 0; a < 3; ++a) lmax += 4.0 / (hs[a] * hs[a]);
    const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
    spectral_scale<<<grid_blocks(n, 256, 148 * 16), 256, 0, s>>>(v1, g, L[0], L[1], L[2],
                                                                 1e-13 * lmax);
    count_launches(1);
    SW_CHECK_LAUNCH("spectral scale");
    rc = axis_transform(g, 2, Q[2], false, v1, v2, s);
    if (rc == SW_OK) rc = axis_transform(g, 1, Q[1], false, v2, v1, s);
    if (rc == SW_OK) rc = cudaMemsetAsync(v2, 0, vec, s) == cudaSuccess ? SW_OK : SW_ECUDA;
    if (rc == SW_OK) rc = axis_transform(g, 0, Q[0], false, v1, v2, s);
    if (rc != SW_OK) return rc;
  }
  if (has_interior) {
    const long long n = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
    finish_spectral<T><<<grid_blocks(n, 256, 148 * 16), 256, 0, s>>>(
        (const T*)fx, (const T*)fy, (const T*)fz, fs, g, c2x, c2y, c2z,
        solve ? v2 : v1 /* zero field when no solve */, out);
    count_launches(1);
    SW_CHECK_LAUNCH("spectral finish");
  }
  if (stats) {
    stats->iters = 0;
    stats->reason = solve ? SW_CG_CONVERGED : SW_CG_EARLY_EXIT;
    stats->rel = 0.0;
    stats->max_div = maxdiv;
  }
  return SW_OK;
}

}  // namespace

extern "C" size_t sw_project_spectral_workspace_bytes(int nx, int ny, int nz) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  return 3 * align_up((size_t)g.ncell * sizeof(double), 256) + spectral_extra_bytes(g) + 256;
}

extern "C" int sw_project_spectral(int in_dtype, const void* fx, const void* fy, const void* fz,
                                   int64_t in_sx, int64_t in_sy, int64_t in_sz, int nx, int ny,
                                   int nz, double dX, double dY, double dZ, double* out,
                                   void* workspace, size_t workspace_bytes, sw_cg_stats* stats,
                                   void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || out == nullptr || !(dX > 0 && dY > 0 && dZ > 0)) {
    set_error("sw_project_spectral: bad grid, spacing or null output");
    return SW_EINVAL;
  }
  Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  InStride fs{in_sx, in_sy, in_sz};
  cudaStream_t s = (cudaStream_t)stream;
  if (in_dtype == SW_F32)
    return spectral_one<float>(fx, fy, fz, fs, g, dX, dY, dZ, out, (char*)workspace,
                               workspace_bytes, stats, s);
  if (in_dtype == SW_F64)
    return spectral_one<double>(fx, fy, fz, fs, g, dX, dY, dZ, out, (char*)workspace,
                                workspace_bytes, stats, s);
  set_error("sw_project_spectral: unknown dtype %d", in_dtype);
  return SW_EINVAL;
}

extern "C" int sw_spectral_basis(int n, double h, double* Q, double* lam) {
  if (n < 3 || !(h > 0) || Q == nullptr || lam == nullptr) {
    set_error("sw_spectral_basis: need n >= 3, h > 0 and host buffers");
    return SW_EINVAL;
  }
  const int m = n - 2;
  for (int row = 0; row < m; ++row)
    for (int col = 0; col < m; ++col)
      Q[(size_t)row * m + col] = basis_entry(n, h, row, col, row == 0 ? lam + col : nullptr);
  return SW_OK;
}
