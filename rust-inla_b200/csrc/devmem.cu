// Device memory for every handle of the library, with a cache of released blocks.
//
// Handles are often created and destroyed in loops (one solver per worker or per
// integration node, one Laplace model per fit); mapping and unmapping the
// multi-GB front buffers each time costs tens of milliseconds. Released blocks are
// therefore kept per device and handed to later requests of similar size (the
// smallest cached block of at least the requested size and at most 1.5x it plus
// 64 MiB). Releasing a block synchronizes the device first -- as cudaFree does --
// so no queued kernel of any stream can still use a block that is handed out
// again. The cache holds at most half of the device's memory; when cudaMalloc
// fails, the cached blocks of that device are returned to the driver and the
// allocation is retried once. INLA_NO_MEMORY_CACHE set in the environment turns
// the cache off; inla_release_cached_memory() empties it.
#include <cuda_runtime.h>

#include <cstdlib>
#include <string>
#include <map>
#include <mutex>
#include <unordered_map>

#include "gpu_factor.hpp"

namespace inla {

namespace {
constexpr int kMaxDevices = 64;

struct Block {
  size_t bytes;
  int dev;
};

struct MemCache {
  std::mutex mu;
  std::multimap<size_t, void*> free_blocks[kMaxDevices];
  size_t cached[kMaxDevices] = {};
  size_t limit[kMaxDevices] = {};
  std::unordered_map<void*, Block> live;
};

MemCache& cache() {
  static MemCache* c = new MemCache();  // outlives static destruction: the driver frees at exit
  return *c;
}

bool cache_enabled() {
  static const bool on = std::getenv("INLA_NO_MEMORY_CACHE") == nullptr;
  return on;
}

size_t round_bytes(size_t b) {
  if (b == 0) b = 1;
  const size_t g = b < (size_t(1) << 20) ? 512 : (size_t(2) << 20);
  return (b + g - 1) / g * g;
}

// return every cached block of `dev` to the driver (caller holds the lock)
void flush_locked(MemCache& c, int dev) {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  for (auto& kv : c.free_blocks[dev]) cudaFree(kv.second);
  c.free_blocks[dev].clear();
  c.cached[dev] = 0;
  if (cur != dev) cudaSetDevice(cur);
}
}  // namespace

void* device_alloc(size_t bytes) {
  bytes = round_bytes(bytes);
  int dev = 0;
  INLA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device index out of range");
  MemCache& c = cache();
  const bool use = cache_enabled();
  if (use) {
    std::lock_guard<std::mutex> lk(c.mu);
    auto& fl = c.free_blocks[dev];
    auto it = fl.lower_bound(bytes);
    if (it != fl.end() && it->first <= bytes + bytes / 2 + (size_t(64) << 20)) {
      void* p = it->second;
      const size_t b = it->first;
      c.cached[dev] -= b;
      fl.erase(it);
      c.live[p] = {b, dev};
      return p;
    }
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e == cudaErrorMemoryAllocation && use) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.cached[dev] > 0) {
      flush_locked(c, dev);
      e = cudaMalloc(&p, bytes);
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw CudaError(std::string("cudaMalloc: ") + cudaGetErrorString(e), (int)e);
  }
  if (use) {
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[p] = {bytes, dev};
  }
  return p;
}

void device_free(void* p) {
  if (!p) return;
  if (!cache_enabled()) {
    cudaFree(p);
    return;
  }
  MemCache& c = cache();
  Block blk{0, 0};
  {
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) {  // not ours: hand it back directly
      cudaFree(p);
      return;
    }
    blk = it->second;
    c.live.erase(it);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != blk.dev) cudaSetDevice(blk.dev);
  cudaDeviceSynchronize();  // as cudaFree: nothing queued may still read or write the block
  std::lock_guard<std::mutex> lk(c.mu);
  if (c.limit[blk.dev] == 0) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) c.limit[blk.dev] = tot / 2;
    else c.limit[blk.dev] = size_t(1) << 34;
  }
  if (c.cached[blk.dev] + blk.bytes > c.limit[blk.dev]) {
    cudaFree(p);
  } else {
    c.free_blocks[blk.dev].emplace(blk.bytes, p);
    c.cached[blk.dev] += blk.bytes;
  }
  if (cur != blk.dev) cudaSetDevice(cur);
}

void device_release_cached() {
  MemCache& c = cache();
  std::lock_guard<std::mutex> lk(c.mu);
  for (int d = 0; d < kMaxDevices; ++d)
    if (c.cached[d] > 0) flush_locked(c, d);
}

}  // namespace inla
