// Allocation-free form of the drop-in CSC solve (mac_csc_solve).
//
// mac_csc_solve keeps the matrix and its five CG work vectors in device memory
// that mac_csc_factorize allocates. This entry point takes the matrix and the
// right-hand side as device pointers the caller already owns and keeps the work
// vectors in one file-scope device array, so it calls no allocator: no
// cudaMalloc/cudaFree, no library call that allocates. The array belongs to the
// library's device code; with CUDA's lazy module loading the driver places it
// in device memory when the first call on a device (or the set-up call with
// n = 0) looks up its address, so that call needs 2.5 MiB of free device
// memory, and no later call needs any. It runs the CG kernels of
// mac_csc_solve (k_csc_diag, k_csc_vec, k_csc_spmv) in the same order, after
// a check that the matrix has the symmetric negative-diagonal form CG needs.
#include <cmath>
#include <mutex>

#include "mac_internal.cuh"

namespace mac {

// Defined with the context-based solve (mac_step.cu).
__global__ void k_csc_spmv(int n, const int* __restrict__ off, const int* __restrict__ ind,
                           const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                           double* partial_dot, const double* __restrict__ pdot);
__global__ void k_csc_diag(int n, const int* __restrict__ off, const int* __restrict__ ind,
                           const double* __restrict__ val, double* dinv);
__global__ void k_csc_vec(int n, int mode, const double* b, double* x, double* r, double* z, double* p,
                          const double* q, const double* dinv, double* scal, double a);

// Scratch: the work vectors r, z, p, q, dinv (MAC_NOALLOC_MAX_N doubles each,
// 2.5 MiB in all) followed by 8 reduction slots. Every vector entry a solve
// reads is written earlier in that solve, so the vectors need no initial
// value; the reduction slots must be zero when each reduction kernel starts,
// and the solve clears them itself before every reduction.
constexpr int kNoAllocVecs = 5;
constexpr size_t kNoAllocSlots = (size_t)kNoAllocVecs * MAC_NOALLOC_MAX_N;
static __device__ __align__(256) double g_csc_scratch[kNoAllocSlots + 8];

constexpr int kMaxDevices = 64;
static std::mutex g_scratch_mu;
static double* g_scratch_addr[kMaxDevices];

// Address of g_csc_scratch on the current device, looked up once per device.
static int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MAC_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return MAC_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_csc_scratch);
    if (e != cudaSuccess || !p) return check(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
    g_scratch_addr[dev] = (double*)p;
  }
  *out = g_scratch_addr[dev];
  return MAC_OK;
}

// Flags (slot 7 = 1) a matrix that is not the symmetric negative-diagonal form
// CG needs: a row index outside [0, n), a diagonal entry that is not negative
// or not present exactly once, or an off-diagonal (i, j) whose mirror (j, i)
// is missing or differs. Column i is scanned linearly for the mirror (the
// reference's columns hold at most 7 entries).
__global__ void k_csc_check(int n, const int* __restrict__ off, const int* __restrict__ ind,
                            const double* __restrict__ val, double* scal) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int k0 = off[j], k1 = off[j + 1];
    bool bad = j == 0 && k0 != 0;
    int ndiag = 0;
    if (k1 < k0) bad = true;
    for (int k = k0; k < k1 && !bad; ++k) {
      const int i = ind[k];
      if (i < 0 || i >= n) {
        bad = true;
      } else if (i == j) {
        ndiag += 1;
        if (!(val[k] < 0)) bad = true;
      } else {
        bool found = false;
        for (int m = off[i]; m < off[i + 1]; ++m)
          if (ind[m] == j) {
            found = val[m] == val[k];
            break;
          }
        if (!found) bad = true;
      }
    }
    if (bad || ndiag != 1) scal[7] = 1.0;
  }
}

static int read_slots(double* hs, const double* scal, cudaStream_t st) {
  int rc = check(cudaMemcpyAsync(hs, scal, 64, cudaMemcpyDeviceToHost, st));
  return rc ? rc : check(cudaStreamSynchronize(st));
}

static int csc_solve_noalloc(cudaStream_t st, int n, const int* off, const int* ind, const double* val,
                             const double* b, double* x, double rtol, int max_iters, int* iterations,
                             double* relres) {
  double* v = nullptr;
  int rc = scratch_address(&v);
  if (rc) return rc;
  double *r = v, *z = v + (size_t)n, *p = v + 2 * (size_t)n, *q = v + 3 * (size_t)n,
         *dinv = v + 4 * (size_t)n, *scal = v + kNoAllocSlots;
  int g = grid_for(n, 256);
  if (g > 1184) g = 1184;
  double hs[8];
  if ((rc = check(cudaMemsetAsync(scal, 0, 64, st)))) return rc;
  k_csc_check<<<g, 256, 0, st>>>(n, off, ind, val, scal);
  if ((rc = check(cudaGetLastError())) || (rc = read_slots(hs, scal, st))) return rc;
  if (hs[7] != 0.0) return MAC_ERR_MATRIX;
  k_csc_diag<<<g, 256, 0, st>>>(n, off, ind, val, dinv);
  if ((rc = check(cudaMemsetAsync(scal, 0, 64, st)))) return rc;
  k_csc_vec<<<g, 256, 0, st>>>(n, 0, b, x, r, z, p, q, dinv, scal, 0);
  if ((rc = check(cudaGetLastError())) || (rc = read_slots(hs, scal, st))) return rc;
  double rz = hs[0], bb = hs[1], rr = bb;
  int it = 0;
  while (bb > 0 && it < max_iters) {
    if ((rc = check(cudaMemsetAsync(scal, 0, 64, st)))) return rc;
    k_csc_spmv<<<g, 256, 0, st>>>(n, off, ind, val, p, q, scal + 3, p);
    if ((rc = check(cudaGetLastError())) || (rc = read_slots(hs, scal, st))) return rc;
    // breakdown (p.q zero or not finite): x keeps the last finite iterate
    if (!(hs[3] != 0.0 && std::isfinite(hs[3]))) break;
    double alpha = rz / hs[3];
    k_csc_vec<<<g, 256, 0, st>>>(n, 1, b, x, r, z, p, q, dinv, scal, alpha);
    k_csc_vec<<<g, 256, 0, st>>>(n, 2, b, x, r, z, p, q, dinv, scal, 0);
    if ((rc = check(cudaGetLastError())) || (rc = read_slots(hs, scal, st))) return rc;
    ++it;
    rr = hs[2];
    if (rr <= rtol * rtol * bb) break;
    double beta = hs[0] / rz;
    rz = hs[0];
    k_csc_vec<<<g, 256, 0, st>>>(n, 3, b, x, r, z, p, q, dinv, scal, beta);
  }
  if ((rc = check(cudaGetLastError()))) return rc;
  if (iterations) *iterations = it;
  if (relres) *relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  return (bb > 0 && !(rr <= rtol * rtol * bb)) ? MAC_ERR_NOT_CONVERGED : MAC_OK;
}

}  // namespace mac

extern "C" int mac_csc_solve_noalloc(void* stream, int n, const int* offset, const int* indice,
                                     const double* value, const double* b, double* x, double rtol,
                                     int max_iters, int* iterations, double* relres) {
  if (n < 0 || max_iters < 0 || !(rtol >= 0)) return MAC_ERR_INVALID;
  if (n > MAC_NOALLOC_MAX_N) return MAC_ERR_CAPACITY;
  if (iterations) *iterations = 0;
  if (relres) *relres = 0.0;
  if (n == 0) {
    // set-up only: resolve the work array's address on the current device
    double* v = nullptr;
    return mac::scratch_address(&v);
  }
  if (!offset || !indice || !value || !b || !x) return MAC_ERR_INVALID;
  return mac::csc_solve_noalloc((cudaStream_t)stream, n, offset, indice, value, b, x, rtol, max_iters,
                                iterations, relres);
}
