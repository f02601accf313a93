// The projection for callers that cannot allocate device memory.
//
// Some hosts of this library hand it only their own input and output
// buffers: applications that reserve all device memory up front through a
// pool or budget of their own and forbid any later cudaMalloc, and bindings
// (ctypes, cgo, JNI ...) that expose no way to allocate device memory for a
// workspace.  sw_project needs a caller-provided workspace for its CG
// vectors; sw_project_noalloc runs the same solve with that scratch taken
// from a fixed array compiled into the library instead.
//
// The array lives in every GPU's memory from the moment the library's code
// is loaded on that GPU until the process exits.  Its device address is
// looked up once per device, on the first call made while that device is
// current.  All calls share the one array: each call re-initialises
// everything it reads, but two calls whose work overlaps on the GPU (for
// example on two streams) overwrite each other's scratch.
#include <mutex>

#include "sw_common.cuh"
#include "sw_project.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array on the current device.
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sw::cuda_status(e, "sw_project_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    sw::set_error("sw_project_noalloc: device ordinal %d is above %d", dev, kMaxDevices - 1);
    return SW_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return sw::cuda_status(e, "sw_project_noalloc: cudaGetSymbolAddress(scratch)");
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return SW_OK;
}

}  // namespace

extern "C" size_t sw_project_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int sw_project_noalloc(int in_dtype, const void* fx, const void* fy, const void* fz,
                                  int64_t in_sx, int64_t in_sy, int64_t in_sz, int nx, int ny,
                                  int nz, double dX, double dY, double dZ, double tol,
                                  int max_iters, double* out, sw_cg_stats* stats,
                                  void* stream) {
  using namespace sw;
  if (nx <= 0 || ny <= 0 || nz <= 0 || out == nullptr || !(dX > 0 && dY > 0 && dZ > 0)) {
    set_error("sw_project_noalloc: bad grid, spacing or null output");
    return SW_EINVAL;
  }
  const Geom g = make_geom(nx, ny, nz, pad_pitch(nz));
  const size_t need = cg_workspace_bytes(g, cg_tiles(g));
  if (need > kNoAllocScratchBytes) {
    set_error(
        "sw_project_noalloc: a %d x %d x %d grid needs %zu bytes of scratch, above the %zu "
        "bytes this entry point holds (about %zu padded cells); use sw_project with a "
        "caller-provided workspace",
        nx, ny, nz, need, kNoAllocScratchBytes, kNoAllocScratchBytes / 48);
    return SW_ERANGE;
  }
  void* ws = nullptr;
  int rc = scratch_address(&ws);
  if (rc != SW_OK) return rc;
  InStride fs{in_sx, in_sy, in_sz};
  return project_field(in_dtype, fx, fy, fz, fs, g, dX, dY, dZ, tol, max_iters, out, ws,
                       kNoAllocScratchBytes, stats, (cudaStream_t)stream);
}
