// A process-wide cache of freed device blocks in front of the stream-ordered
// pool. A block freed on a stream is reused, in stream order, by the next
// allocation of its size on that stream; one freed after a device
// synchronization by an allocation on any stream of its device. Repeated
// calls of the same shapes then allocate without entering the driver.
#include <map>
#include <tuple>
#include <vector>

#include "common.h"

namespace ef {
namespace {

constexpr size_t kMaxCached = 24ull << 30;

// Sizes in classes: 512-byte steps up to 1 MiB, 2 MiB steps above.
size_t size_class(size_t bytes) {
  if (bytes == 0) bytes = 1;
  if (bytes <= (1u << 20)) return (bytes + 511) / 512 * 512;
  return (bytes + (2u << 20) - 1) / (2u << 20) * (2u << 20);
}

struct BlockCache {
  std::mutex m;
  // (stream or null for any stream, device, size class) -> free blocks
  std::map<std::tuple<cudaStream_t, int, size_t>, std::vector<void*>> free;
  size_t cached = 0;
};

BlockCache& cache() {
  static BlockCache* c = new BlockCache;  // outlives buffers released at exit
  return *c;
}

bool take(BlockCache& c, cudaStream_t s, int device, size_t cls, void** p) {
  auto it = c.free.find(std::make_tuple(s, device, cls));
  if (it == c.free.end() || it->second.empty()) return false;
  *p = it->second.back();
  it->second.pop_back();
  c.cached -= cls;
  return true;
}

}  // namespace

void* device_alloc(size_t bytes, cudaStream_t s) {
  const size_t cls = size_class(bytes);
  int device = 0;
  EF_CUDA(cudaGetDevice(&device));
  BlockCache& c = cache();
  {
    std::lock_guard<std::mutex> lock(c.m);
    void* p = nullptr;
    if (take(c, s, device, cls, &p) || take(c, nullptr, device, cls, &p)) return p;
  }
  void* p = nullptr;
  if (cudaMallocAsync(&p, cls, s) == cudaSuccess) return p;
  // Out of memory: return the device's cached blocks to the driver and try
  // again.
  cudaGetLastError();
  std::vector<void*> blocks;
  {
    std::lock_guard<std::mutex> lock(c.m);
    for (auto it = c.free.begin(); it != c.free.end();) {
      if (std::get<1>(it->first) != device) {
        ++it;
        continue;
      }
      blocks.insert(blocks.end(), it->second.begin(), it->second.end());
      c.cached -= std::get<2>(it->first) * it->second.size();
      it = c.free.erase(it);
    }
  }
  cudaDeviceSynchronize();
  for (void* b : blocks) cudaFree(b);
  EF_CUDA(cudaMallocAsync(&p, cls, s));
  return p;
}

void device_free(void* p, size_t bytes, cudaStream_t s) {
  if (!p) return;
  const size_t cls = size_class(bytes);
  int device = 0;
  cudaGetDevice(&device);
  BlockCache& c = cache();
  {
    std::lock_guard<std::mutex> lock(c.m);
    if (c.cached + cls <= kMaxCached) {
      c.free[std::make_tuple(s, device, cls)].push_back(p);
      c.cached += cls;
      return;
    }
  }
  cudaFreeAsync(p, s);
}

void device_free_synchronized(void* p, size_t bytes, int device) {
  if (!p) return;
  const size_t cls = size_class(bytes);
  BlockCache& c = cache();
  {
    std::lock_guard<std::mutex> lock(c.m);
    if (c.cached + cls <= kMaxCached) {
      c.free[std::make_tuple((cudaStream_t) nullptr, device, cls)].push_back(p);
      c.cached += cls;
      return;
    }
  }
  cudaFree(p);
}

void device_cache_forget(cudaStream_t s) {
  BlockCache& c = cache();
  std::lock_guard<std::mutex> lock(c.m);
  for (auto it = c.free.begin(); it != c.free.end();) {
    if (std::get<0>(it->first) == s) {
      auto& any = c.free[std::make_tuple((cudaStream_t) nullptr, std::get<1>(it->first), std::get<2>(it->first))];
      any.insert(any.end(), it->second.begin(), it->second.end());
      it = c.free.erase(it);
    } else {
      ++it;
    }
  }
}

}  // namespace ef
