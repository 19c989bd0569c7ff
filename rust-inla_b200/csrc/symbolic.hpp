// Host-side symbolic analysis shared by every numeric factorization of one
// sparsity pattern: fill-reducing ordering, elimination tree, column counts,
// relaxed supernode partition, supernodal row structures, level schedule and
// the index maps the CUDA kernels use (value scatter, extend-add, selected
// inverse gather).
//
// Reference behaviour being replaced:
//   crates/inla_math/src/ordering.rs:149-162   choose_symmetric_order (restated bit-exact)
//   crates/inla_math/src/sparse_ldlt.rs:151-186 factorize_symbolic (faer AMD + supernodal
//                                               symbolic; faer itself is not vendored, the
//                                               AMD here is written from the published
//                                               Amestoy-Davis-Duff algorithm)
//   crates/inla_math/src/sparse_ldlt.rs:82-92  lower-triangle convention (row >= col)
//   crates/inla_math/src/scratch.rs:90-119     exact pattern match => numeric-only refactor
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace inla {

// Which branch the ordering choice took (values are part of the C ABI).
enum OrderKind : int {
  ORDER_AUTO = 0,        // reference choice: time-major -> RCM -> AMD
  ORDER_AMD = 1,
  ORDER_RCM = 2,
  ORDER_NATURAL = 3,
  ORDER_CUSTOM = 4,      // caller-provided permutation
  ORDER_TIME_MAJOR = 5,
  ORDER_ND = 6,          // nested dissection (nd.cpp)
};

struct SymbolicOptions {
  int ordering = ORDER_AUTO;
  // Relaxed supernode amalgamation: merge a child into its parent when the
  // merged width and the fraction of explicit zeros stay under these bounds.
  int nrelax0 = 4, nrelax1 = 16, nrelax2 = 48;
  double zrelax0 = 0.8, zrelax1 = 0.1, zrelax2 = 0.05;
  int max_width = 1 << 30;  // cap on supernode width (columns)
};

struct Symbolic {
  // Identity of the analysis: every analysis computed gets a new id, and the copies the
  // process-wide cache hands out keep the id of the analysis they copy, so equal ids mean equal
  // contents (tables derived from an analysis can be cached by id). 0: not from analyze().
  uint64_t id = 0;
  int64_t n = 0;
  int order_used = ORDER_AMD;
  // perm[new] = old ; iperm[old] = new (after postordering)
  std::vector<int64_t> perm, iperm;
  std::vector<int64_t> etree;     // column elimination tree (permuted indices), -1 = root
  std::vector<int64_t> colcount;  // nnz of column j of L incl. the diagonal (true structure)

  // Supernodes, in postorder of the supernodal tree.
  int64_t nsuper = 0;
  std::vector<int64_t> sn_first;   // nsuper+1: columns [sn_first[s], sn_first[s+1])
  std::vector<int64_t> sn_rowptr;  // nsuper+1: offsets into sn_rows
  std::vector<int64_t> sn_rows;    // sorted row structure incl. the supernode's own columns
  std::vector<int64_t> sn_parent;  // -1 for roots
  std::vector<int64_t> sn_lptr;    // nsuper+1: L panel offsets (m*k column-major panels)
  std::vector<int64_t> sn_uptr;    // nsuper+1: update-block offsets (r*r, r = m-k)
  std::vector<int32_t> sn_level;   // 0 = leaf
  std::vector<int64_t> col_to_sn;
  std::vector<int64_t> child_ptr, child_list;  // CSR children of each supernode
  std::vector<int64_t> rel_ptr;                // nsuper+1 offsets into rel
  std::vector<int32_t> rel;                    // below-row -> position in parent's structure
  int32_t nlevels = 0;
  std::vector<int64_t> level_ptr, level_list;  // supernodes grouped by level

  // Input pattern copy (full symmetric CSC, both triangles) and value map.
  std::vector<int64_t> colptr, rowidx;
  std::vector<int64_t> qmap;  // per input entry: L storage position (row>=col entries), -1 otherwise

  int64_t nnz_l_stored = 0;  // sum m*k over supernodes
  int64_t nnz_l = 0;         // true structural nnz(L) incl. diagonal
  int64_t u_total = 0;       // sum r*r
  int64_t max_m = 0, max_k = 0, max_r = 0;
  double flops_factor = 0;   // sum_j (c_j^2 + 2 c_j), c_j = colcount-1
  double flops_selinv = 0;   // sum_j (2 c_j^2 + 2 c_j)
  double flops_solve = 0;    // 4 nnz(L) + n
};

// Reference restatements (ordering.rs).
int64_t lower_bandwidth(int64_t n, const int64_t* colptr, const int64_t* rowidx);
int64_t bandwidth_with_fwd(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           const int64_t* fwd);
bool try_time_major_kronecker(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                              std::vector<int64_t>& fwd);
void reverse_cuthill_mckee(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           std::vector<int64_t>& fwd);
// Returns the branch taken; fills fwd (old->new) for custom branches.
int choose_symmetric_order(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           std::vector<int64_t>& fwd);

// Approximate minimum degree on the symmetric pattern; returns perm[new] = old.
void nd_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, std::vector<int64_t>& perm);
void amd_order(int64_t n, const int64_t* colptr, const int64_t* rowidx,
               std::vector<int64_t>& perm);

// Full analysis. Throws std::runtime_error on invalid input. Results are cached process-wide by
// exact inputs (see symbolic.cpp); release_symbolic_cache() empties the cache.
void analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx,
             const SymbolicOptions& opt, const int64_t* custom_perm, Symbolic& out);
void release_symbolic_cache();

}  // namespace inla
