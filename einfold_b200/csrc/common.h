// Shared host-side machinery of the einfold_b200 library: errors, the
// budget, device buffers, the per-device context and its stream.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/einfold_b200.h"

namespace ef {

// An outcome other than success, carried to the ABI boundary.
struct Failure : std::runtime_error {
  int32_t status;
  Failure(int32_t s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(int32_t status, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw Failure(status, buf);
}

// The kernels' requirements don't hold: the caller runs the host's plan.
struct Declined {
  std::string why;
};
[[noreturn]] inline void decline(const std::string& why) { throw Declined{why}; }

#define EF_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      ::ef::fail(EINFOLD_DEVICE, "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
  } while (0)

#define EF_LAUNCH_CHECK() EF_CUDA(cudaGetLastError())

// The memory a call may take beyond its inputs (options.rs:56-65). Asked
// before allocating; a refusal fails the call with EINFOLD_BUDGET.
struct Budget {
  const einfold_options* o = nullptr;
  uint64_t taken = 0;
  bool try_reserve(uint64_t bytes) {
    if (!o || !o->budget_grow) return true;
    if (o->budget_grow(o->budget_ctx, bytes)) {
      taken += bytes;
      return true;
    }
    return false;
  }
  void reserve(uint64_t bytes, const char* what) {
    if (!try_reserve(bytes))
      fail(EINFOLD_BUDGET, "EinFold's budget can't give %llu bytes for %s", (unsigned long long)bytes, what);
  }
  void release(uint64_t bytes) {
    if (o && o->budget_shrink) o->budget_shrink(o->budget_ctx, bytes);
    taken = bytes > taken ? 0 : taken - bytes;
  }
};

// Saturating arithmetic on sizes, as the reference's usize::saturating_*.
inline uint64_t sat_add(uint64_t a, uint64_t b) { return a + b < a ? UINT64_MAX : a + b; }
inline uint64_t sat_mul(uint64_t a, uint64_t b) {
  if (a == 0 || b == 0) return 0;
  return a > UINT64_MAX / b ? UINT64_MAX : a * b;
}
// a * b, or false on overflow (checked_mul).
inline bool checked_mul(uint64_t a, uint64_t b, uint64_t* out) {
  if (a != 0 && b > UINT64_MAX / a) return false;
  *out = a * b;
  return true;
}

struct Context;

// Device scratch through a process-wide cache of freed blocks keyed by
// stream, device and size class: a block freed on a stream is reused in
// stream order on it; one freed after a device synchronization on any
// stream of its device. Misses go to the stream-ordered pool.
void* device_alloc(size_t bytes, cudaStream_t s);
void device_free(void* p, size_t bytes, cudaStream_t s);
void device_free_synchronized(void* p, size_t bytes, int device);
// Hands a stream's cached blocks over to any stream (the stream is about
// to be destroyed, its work done).
void device_cache_forget(cudaStream_t s);

// A device allocation (device_alloc), freed on the same stream when it goes
// out of scope.
template <class T>
struct DeviceBuffer {
  T* ptr = nullptr;
  size_t count = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffer() = default;
  DeviceBuffer(size_t n, cudaStream_t s) { allocate(n, s); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept { *this = std::move(o); }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    reset();
    ptr = o.ptr; count = o.count; stream = o.stream;
    o.ptr = nullptr; o.count = 0;
    return *this;
  }
  void allocate(size_t n, cudaStream_t s) {
    reset();
    stream = s;
    count = n;
    if (n) ptr = (T*)device_alloc(n * sizeof(T), s);
  }
  void zero() {
    if (count) EF_CUDA(cudaMemsetAsync(ptr, 0, count * sizeof(T), stream));
  }
  void reset() {
    if (ptr) device_free(ptr, count * sizeof(T), stream);
    ptr = nullptr;
    count = 0;
  }
  ~DeviceBuffer() { reset(); }
  T* get() const { return ptr; }
  size_t bytes() const { return count * sizeof(T); }
};

// Pinned host memory for staging copies, grown on demand and kept.
struct PinnedArena {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t n) {
    if (n > bytes) {
      if (ptr) cudaFreeHost(ptr);
      ptr = nullptr;
      size_t want = n < (64u << 20) ? (64u << 20) : n;
      EF_CUDA(cudaHostAlloc(&ptr, want, cudaHostAllocDefault));
      bytes = want;
    }
    return ptr;
  }
  ~PinnedArena() {
    if (ptr) cudaFreeHost(ptr);
  }
};

// Instantiated CUDA graphs of a context's launch sequences. An entry is
// replayed only when every argument its launches were captured with
// (pointers included) is the same. Arguments seen for the first time are
// launched directly, so that one-off arguments leave the cache alone; seen
// again, the sequence is captured and updated into the entry of the same
// shape (kernels, grids), or instantiated.
struct GraphCache {
  struct Entry {
    std::vector<uint8_t> shape, key;
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
  };
  std::vector<Entry> entries;
  uint64_t clock = 0;
  cudaStream_t capture = nullptr;  // the stream graphs are captured on (the context's device)
  std::vector<uint8_t> seen_shape, seen_key;  // the arguments last launched directly
  static constexpr size_t kMaxEntries = 8;
  // Launches `enqueue`'s work (queued on the stream it is given) on
  // `stream`: 0 directly, else through a graph, 1 replayed, 2 updated,
  // 3 instantiated.
  int run(const std::vector<uint8_t>& shape, const std::vector<uint8_t>& key, cudaStream_t stream,
          const std::function<void(cudaStream_t)>& enqueue);
  void clear();
};

struct Context {
  // With EINFOLD_TRACE set, phase() synchronizes the stream and prints the
  // milliseconds since the previous phase to stderr.
  bool tracing = false;
  double last_phase = 0;
  void phase(const char* name);
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex lock;
  int sm_count = 148;
  uint64_t kernels = 0;  // kernels launched by the current call
  double product_ms = 0, product_ops = 0;  // the split products' kernels in the current call
  PinnedArena pinned;
  // A second stream of the context, for work that overlaps the main
  // stream's within one call (created on first use, destroyed with the
  // context).
  cudaStream_t aux = nullptr;
  GraphCache graphs;
  // The current call's attention forward: its schedule (-1: none) and how
  // its tile phase ran (0 launched directly, else GraphCache::run's value).
  int schedule = -1, graph = 0;
  // Device-resident scratch kept across calls.
  void* status_word = nullptr;  // int32 status set by bounded device waits
};

// Makes `ctx`'s device current for the scope.
struct DeviceGuard {
  int old = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&old);
    if (old != dev) EF_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    if (old >= 0) cudaSetDevice(old);
  }
};

inline double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline void Context::phase(const char* name) {
  if (!tracing) return;
  cudaStreamSynchronize(stream);
  double t = now_ms();
  std::fprintf(stderr, "[einfold %p] %-28s %9.3f ms\n", (void*)stream, name, last_phase ? t - last_phase : 0.0);
  last_phase = t;
}

inline unsigned blocks_for(uint64_t n, unsigned threads, unsigned cap = 148u * 32u) {
  uint64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  return (unsigned)(b > cap ? cap : b);
}

}  // namespace ef
