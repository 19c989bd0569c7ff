// Host-side parallel loop over an index range: the range is cut into contiguous
// chunks, one per hardware thread (at least `grain` indices each), and body(lo, hi)
// runs on each chunk. Bodies must write disjoint data; exceptions from a chunk
// are rethrown on the calling thread after all chunks finish.
#pragma once
#include <algorithm>
#include <cstdint>
#include <exception>
#include <thread>
#include <vector>

namespace inla {

template <class Body>
void parallel_for(int64_t n, Body&& body, int64_t grain = 8192) {
  const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
  const int64_t nt = std::min<int64_t>(hw, std::max<int64_t>(1, n / std::max<int64_t>(grain, 1)));
  if (nt <= 1) {
    body((int64_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  std::vector<std::exception_ptr> err(nt);
  const int64_t chunk = (n + nt - 1) / nt;
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([&, t, lo, hi] {
      try {
        body(lo, hi);
      } catch (...) {
        err[t] = std::current_exception();
      }
    });
  }
  for (auto& x : th) x.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

}  // namespace inla
