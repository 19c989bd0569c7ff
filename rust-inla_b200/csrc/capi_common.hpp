// Shared helpers for the extern "C" layer: error type, last-error slot,
// launch counter and pinned host staging.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "gpu_factor.hpp"

namespace inla {

struct InlaError : std::runtime_error {
  int code;
  InlaError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

extern thread_local std::string g_last_error;
extern std::atomic<int64_t> g_launches;
int fail(int code, const std::string& msg);
int map_exception();

template <class T>
struct PinnedBuf {
  T* p = nullptr;
  size_t n = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    INLA_CUDA(cudaMallocHost(&p, (count ? count : 1) * sizeof(T)));
    n = count;
  }
};

}  // namespace inla
