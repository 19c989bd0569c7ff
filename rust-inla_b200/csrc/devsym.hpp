// Device view of one symbolic analysis (plain pointers into device arrays).
#pragma once
#include <cstdint>

namespace inla {

struct DevSym {
  int n = 0, ns = 0;
  const int* first = nullptr;      // ns+1
  const int* rowptr = nullptr;     // ns+1
  const int* rows = nullptr;       // sum m : permuted row indices
  const int* relx = nullptr;       // sum m : position of below-row in parent's structure
  const int64_t* fptr = nullptr;   // ns+1 : front offsets
  const int64_t* lptr = nullptr;   // ns+1 : panel offsets (compact m*k numbering)
  const int* child_ptr = nullptr;  // ns+1
  const int* child_list = nullptr;
  const int* parent = nullptr;     // ns
  const int* uoff = nullptr;       // ns+1 : offsets of the per-supernode update vectors (sum r)
  const int64_t* dpos = nullptr;   // n : front offset of D_j
  const int* perm = nullptr;       // n : perm[new] = old
  // 64 x 64 inverse-block cache of the large fronts: block (s, j0 / 64) of
  // problem b at linv + (b * lstride + (lbo[s] + j0 / 64) * 4096); lbo[s] = -1
  // for fronts that have no cached blocks.
  const int* lbo = nullptr;        // ns
  int64_t lstride = 0;
  // Optional (independent models held block-diagonally): the factorization skips the fronts
  // of the (problem, model) pairs whose entry of active ([B][nseg]) is 0; fseg: model of
  // each front. Those fronts keep their previous contents.
  const unsigned char* active = nullptr;
  const int* fseg = nullptr;
  int nseg = 1;
};

__host__ __device__ inline bool front_skipped(const DevSym& S, int s, int b) {
  return S.active && !S.active[(int64_t)b * S.nseg + S.fseg[s]];
}

constexpr int kStatusOk = 0;
constexpr int kStatusSingular = 1;
constexpr int kStatusNotFinite = 2;
constexpr int kStatusSchedule = 4;  // the persistent schedule stopped early (a dependency wait ran out)

}  // namespace inla
