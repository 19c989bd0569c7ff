// Dense LDL^T factorization, log-determinant and solve that allocate no
// device memory.
//
// Who needs this: a host program that embeds this library but owns every
// device allocation itself (a memory-pool runtime, a framework plugin that
// hands out pre-sized buffers, code that must not trigger cudaMalloc /
// cudaFree because they synchronize the device or are forbidden while other
// work is being captured or scheduled). Those callers pass their own device
// buffers for the inputs and outputs; the intermediate factor lives in the
// fixed-size scratch below, which is part of the loaded module.
//
// Limits and sharing:
//  * n <= kNoAllocMaxN (1024); larger systems are rejected with
//    INLA_ERR_DIM_MISMATCH (use the inla_solver_* / inla_batch_* entry points).
//  * The scratch (8 MiB factor + 8 KiB vector + metadata) is one set of static
//    device arrays per GPU that loads the library, held until process exit.
//  * Every call on a device uses the same scratch and leaves its contents
//    behind; each call overwrites all of the scratch it reads before reading
//    it, so nothing has to start at zero. Calls whose GPU work overlaps (for
//    example on two streams at once) race on the scratch: serialize them.
//  * The first call on a device resolves the scratch addresses with
//    cudaGetSymbolAddress (which also loads the module on that device); make
//    that first call before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include "capi_common.hpp"
#include "inla_b200.h"
#include "snode_kernels.cuh"

namespace inla {
namespace {

constexpr int kNoAllocMaxN = 1024;
constexpr int kMaxDevices = 64;

// factor of one dense front (column-major n x n, leading dimension n)
static __device__ __align__(256) double g_noalloc_front[kNoAllocMaxN * kNoAllocMaxN];
// working vector of the triangular solves
static __device__ __align__(256) double g_noalloc_vec[kNoAllocMaxN];
// one-supernode symbolic description: [0,2) first, [2,4) rowptr, [4,6) child_ptr,
// [6] parent, [7,9) uoff, [9] supernode list {0}, then rows, relx, perm (kNoAllocMaxN each)
static __device__ __align__(256) int g_noalloc_int[16 + 3 * kNoAllocMaxN];
// [0,2) front offsets, [2,4) panel offsets, [8, 8+n) diagonal positions
static __device__ __align__(256) int64_t g_noalloc_i64[8 + kNoAllocMaxN];

struct NoAllocScratch {
  double* front = nullptr;
  double* vec = nullptr;
  int* gi = nullptr;
  int64_t* gl = nullptr;
  std::atomic<bool> ready{false};  // set once, under g_scratch_mu, after the addresses
};
NoAllocScratch g_scratch[kMaxDevices];
std::mutex g_scratch_mu;

// Per-device set-up: host code cannot use the arrays' names as device
// addresses, so resolve them once with the device current.
int scratch_for_current_device(NoAllocScratch** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(INLA_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(INLA_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  NoAllocScratch& s = g_scratch[dev];
  if (!s.ready) {
    void* p = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_front)) != cudaSuccess)
      return fail(INLA_ERR_CUDA, std::string("cudaGetSymbolAddress(front): ") + cudaGetErrorString(e));
    s.front = (double*)p;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_vec)) != cudaSuccess)
      return fail(INLA_ERR_CUDA, std::string("cudaGetSymbolAddress(vec): ") + cudaGetErrorString(e));
    s.vec = (double*)p;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_int)) != cudaSuccess)
      return fail(INLA_ERR_CUDA, std::string("cudaGetSymbolAddress(int): ") + cudaGetErrorString(e));
    s.gi = (int*)p;
    if ((e = cudaGetSymbolAddress(&p, g_noalloc_i64)) != cudaSuccess)
      return fail(INLA_ERR_CUDA, std::string("cudaGetSymbolAddress(i64): ") + cudaGetErrorString(e));
    s.gl = (int64_t*)p;
    s.ready = true;
  }
  *out = &s;
  return INLA_OK;
}

// Write the one-supernode description for size n and copy Q into the front.
__global__ void k_noalloc_setup(int n, const double* __restrict__ q, double* __restrict__ front, int* gi,
                                int64_t* gl) {
  const int64_t nn = (int64_t)n * n;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x)
    front[e] = q[e];
  const int N = kNoAllocMaxN;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    gi[16 + j] = j;          // rows
    gi[16 + N + j] = -1;     // relx (no parent)
    gi[16 + 2 * N + j] = j;  // perm: identity
    gl[8 + j] = (int64_t)j * (n + 1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    gi[0] = 0; gi[1] = n;   // first
    gi[2] = 0; gi[3] = n;   // rowptr
    gi[4] = 0; gi[5] = 0;   // child_ptr
    gi[6] = -1;             // parent
    gi[7] = 0; gi[8] = 0;   // uoff
    gi[9] = 0;              // supernode list
    gl[0] = 0; gl[1] = nn;  // fptr
    gl[2] = 0; gl[3] = nn;  // lptr
  }
}

__global__ void k_noalloc_copy(int n, const double* __restrict__ a, double* __restrict__ b) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) b[j] = a[j];
}

}  // namespace
}  // namespace inla

using namespace inla;

extern "C" int inla_dense_ldlt_solve_noalloc(int n, const double* d_q, const double* d_rhs, double* d_x,
                                             double* d_logdet, int* d_status, void* stream) {
  if (n < 1 || n > kNoAllocMaxN)
    return fail(INLA_ERR_DIM_MISMATCH, "n=" + std::to_string(n) + " is outside the no-allocation limit 1.." +
                                           std::to_string(kNoAllocMaxN) +
                                           "; use inla_solver_* or inla_batch_* for larger systems");
  if (!d_q || !d_logdet || !d_status) return fail(INLA_ERR_INVALID, "null input or output pointer");
  if ((d_rhs == nullptr) != (d_x == nullptr)) return fail(INLA_ERR_INVALID, "rhs and x must both be given or both NULL");
  cudaStream_t st = (cudaStream_t)stream;
  NoAllocScratch* s = nullptr;
  {
    int dev = -1;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < kMaxDevices && !g_scratch[dev].ready) {
      // the one-time set-up may not run inside a stream capture
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      const cudaError_t e = cudaStreamIsCapturing(st, &cs);
      if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return fail(INLA_ERR_INVALID,
                    "the first call on a device resolves the static scratch and cannot run while the stream is "
                    "being captured; make one call on this device before the capture begins");
      }
    }
  }
  int rc = scratch_for_current_device(&s);
  if (rc != INLA_OK) return rc;
  const int N = kNoAllocMaxN;
  DevSym ds;
  ds.n = n;
  ds.ns = 1;
  ds.first = s->gi + 0;
  ds.rowptr = s->gi + 2;
  ds.child_ptr = s->gi + 4;
  ds.parent = s->gi + 6;
  ds.uoff = s->gi + 7;
  ds.child_list = s->gi + 9;  // never read: the single supernode has no children
  ds.rows = s->gi + 16;
  ds.relx = s->gi + 16 + N;
  ds.perm = s->gi + 16 + 2 * N;
  ds.fptr = s->gl + 0;
  ds.lptr = s->gl + 2;
  ds.dpos = s->gl + 8;
  const int* list = s->gi + 9;
  auto cdiv = [](int a, int b) { return (a + b - 1) / b; };

  k_noalloc_setup<<<std::min(cdiv(n * n, 256), 1024), 256, 0, st>>>(n, d_q, s->front, s->gi, s->gl);
  for (int j0 = 0; j0 < n; j0 += kNB) {
    k_diag_large<<<dim3(1, 1), 128, 0, st>>>(ds, list, j0, s->front, 0);
    const int rows = n - j0;
    k_trsm_large<<<dim3(1, 1, cdiv(rows, kTrsmRows)), kTrsmRows, 0, st>>>(ds, list, j0, s->front, 0);
    const int nt = cdiv(rows, kUT);
    k_update_large<<<dim3(1, 1, nt * (nt + 1) / 2), 128, 0, st>>>(ds, list, j0, s->front, 0);
  }
  k_logdet<256><<<1, 256, 0, st>>>(ds, s->front, 0, d_logdet, d_status);
  int launches = 2 + 3 * cdiv(n, kNB);
  if (d_rhs) {
    k_noalloc_copy<<<cdiv(n, 256), 256, 0, st>>>(n, d_rhs, s->vec);
    k_fwd<128><<<dim3(1, 1), 128, n * sizeof(double), st>>>(ds, list, s->front, 0, s->vec, s->vec, 0);
    k_bwd<128><<<dim3(1, 1), 128, n * sizeof(double), st>>>(ds, list, s->front, 0, s->vec);
    k_noalloc_copy<<<cdiv(n, 256), 256, 0, st>>>(n, s->vec, d_x);
    launches += 4;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(INLA_ERR_CUDA, std::string("launch failed: ") + cudaGetErrorString(e));
  g_launches += launches;
  return INLA_OK;
}
