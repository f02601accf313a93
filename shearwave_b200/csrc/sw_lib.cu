// Library-level entry points: version, error reporting, device selection.
#include <stdarg.h>
#include <stdio.h>

#include <string.h>

#include <atomic>
#include <map>
#include <mutex>
#include <vector>

#include "sw_common.cuh"

namespace sw {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

static std::atomic<unsigned long long> g_launches{0}, g_enqueues{0};

void count_launches(unsigned long long n, unsigned long long host) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  g_enqueues.fetch_add(host == ~0ull ? n : host, std::memory_order_relaxed);
}

static std::atomic<int> g_tune[SW_TUNE_COUNT] = {{2}, {8}, {0}, {0}, {0}, {3906250}};

int tune_get(int knob) { return (knob >= 0 && knob < SW_TUNE_COUNT) ? g_tune[knob].load() : -1; }

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
  return SW_ECUDA;
}

// Page-locked staging of the small tables the host builds between launches
// (batched solve tables).  A copy from pageable memory may wait for the
// stream, which would stop the host from running ahead of the GPU; from a
// page-locked slot the copy is queued and the call returns.  Each device has
// a ring of slots, each with an event recorded after its copy: a slot is
// refilled once that copy has run (the wait only happens when the host is
// kRingSlots uploads ahead of the GPU).
namespace {
constexpr int kRingSlots = 32;
struct StageSlot {
  void* host = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
};
struct StageRing {
  StageSlot slot[kRingSlots];
  int next = 0;
};
std::mutex g_stage_mu;
std::map<int, StageRing> g_stage;
}  // namespace

int upload_staged(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return SW_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lock(g_stage_mu);
  StageRing& ring = g_stage[dev];
  StageSlot& sl = ring.slot[ring.next];
  ring.next = (ring.next + 1) % kRingSlots;
  if (sl.pending) {
    e = cudaEventSynchronize(sl.done);  // the copy that last used this slot
    if (e != cudaSuccess) return cuda_status(e, "table staging wait");
    sl.pending = false;
  }
  if (sl.done == nullptr) {
    e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_status(e, "table staging event");
  }
  if (sl.cap < bytes) {
    if (sl.host != nullptr) cudaFreeHost(sl.host);
    sl.host = nullptr;
    sl.cap = 0;
    const size_t cap = bytes < 65536 ? 65536 : 2 * bytes;
    e = cudaHostAlloc(&sl.host, cap, cudaHostAllocPortable);
    if (e != cudaSuccess) return cuda_status(e, "table staging buffer");
    sl.cap = cap;
  }
  memcpy(sl.host, src, bytes);
  e = cudaMemcpyAsync(dst, sl.host, bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_status(e, "table upload");
  e = cudaEventRecord(sl.done, s);
  if (e != cudaSuccess) return cuda_status(e, "table staging event");
  sl.pending = true;
  return SW_OK;
}

}  // namespace sw

extern "C" int sw_abi_version(void) { return SW_ABI_VERSION; }

extern "C" const char* sw_last_error(void) { return sw::g_err; }

extern "C" int sw_set_device(int device) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return sw::cuda_status(e, "cudaSetDevice");
  return SW_OK;
}

extern "C" int sw_pitch(int nz) { return nz > 0 ? sw::pad_pitch(nz) : 0; }

extern "C" size_t sw_fdtd_desc_size(void) { return sizeof(sw_fdtd_desc); }

extern "C" uint64_t sw_launch_count(void) { return sw::g_launches.load(); }

extern "C" uint64_t sw_host_enqueue_count(void) { return sw::g_enqueues.load(); }

extern "C" int sw_tune_set(int knob, int value) {
  static const int lo[SW_TUNE_COUNT] = {1, 1, 0, 0, 0, 1};
  static const int hi[SW_TUNE_COUNT] = {2, 64, 1 << 20, 2, 2, 4000000};
  if (knob < 0 || knob >= SW_TUNE_COUNT || value < lo[knob] || value > hi[knob]) {
    sw::set_error("sw_tune_set: knob %d does not take the value %d", knob, value);
    return SW_EINVAL;
  }
  sw::g_tune[knob].store(value);
  return SW_OK;
}

extern "C" int sw_tune_get(int knob) { return sw::tune_get(knob); }
