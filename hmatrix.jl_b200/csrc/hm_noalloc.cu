// Allocation-free variant of the fully pivoted ACA entry point.
//
// Some callers cannot call cudaMalloc: their device memory is owned by another
// allocator (a framework's caching pool that has already reserved the GPU, so
// a fresh cudaMalloc fails or fragments its budget), or they run latency
// critical loops on a shared GPU where the device-wide synchronisation that
// cudaMalloc/cudaFree imply is not acceptable.  aca_wrapper_noalloc serves
// them: the caller passes device buffers for the input and the outputs, and
// the residual matrix the algorithm needs lives in a fixed, file-scope device
// array that every GPU loading this library holds until the process exits.
//
// Rules that follow from the shared array:
//  * the residual is at most NOALLOC_MAX_ELEMS doubles (m*n + m + n <= the
//    limit, e.g. up to 512 x 510); larger requests are rejected with
//    HM_ERR_ARG before anything is launched;
//  * every call reuses the same array and it keeps the last call's contents;
//    each call overwrites everything it reads (the residual is copied from A,
//    the pivot vectors are written before use, the result slots are written
//    at the end), so no state leaks from one call to the next;
//  * calls that overlap on the GPU (different streams or host threads at the
//    same time) race on the array and must be serialised by the caller;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress while that device is current; make that first call
//    before any stream capture begins.  The address is kept until the process
//    exits, so a cudaDeviceReset on that device ends the use of this entry
//    point;
//  * each call copies the rank back to the host and waits for its stream.
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <mutex>

namespace hm {

constexpr int64_t NOALLOC_RESULT_SLOTS = 32;           // 256 bytes: rank, status
constexpr int64_t NOALLOC_MAX_ELEMS = (1 << 18) - NOALLOC_RESULT_SLOTS;
constexpr int NOALLOC_MAX_DEVICES = 64;

// file-scope scratch; host code must not pass its name to a kernel (on the
// host it is only a stand-in symbol), only the address looked up below
static __device__ __align__(256) double g_aca_scratch[NOALLOC_RESULT_SLOTS + NOALLOC_MAX_ELEMS];

static std::mutex g_scratch_mu;
static double* g_scratch_ptr[NOALLOC_MAX_DEVICES] = {};

// once per device, with that device current
static int scratch_address(int dev, double** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(HM_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_aca_scratch);
    if (e != cudaSuccess)
      return fail(HM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = (double*)p;
  }
  *out = g_scratch_ptr[dev];
  return HM_OK;
}

// Same algorithm and arithmetic as aca_fp_kernel (ACA_FullyPivoted.cpp:9-151,
// the rank == 0 branch with minRank 1); the residual and the current pivot
// column/row live in `scratch`, and the first `keep` columns of U and V are
// written to the caller's buffers, as aca_wrapper copies at most rank+1.
__global__ void __launch_bounds__(512) aca_fp_noalloc_kernel(const double* __restrict__ A, double* __restrict__ U,
                                                             double* __restrict__ V, int m, int n, double eps,
                                                             int keep, double* __restrict__ scratch) {
  __shared__ double red[32];
  __shared__ double s_a[32];
  __shared__ int64_t s_i[32];
  __shared__ double s_v[32];
  __shared__ int64_t s_sel;
  __shared__ double s_max;
  double* res = scratch;                                // [0] rank, [1] status
  double* R = scratch + NOALLOC_RESULT_SLOTS;           // m x n residual
  double* ucur = R + (int64_t)m * n;                    // current pivot column
  double* vcur = ucur + m;                              // current pivot row
  const int64_t mn = (int64_t)m * n;
  const int maxr = min(m, n);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double meps = 2.220446049250313e-16;
  int rank = 0, status = 0;
  bool have_term = false;

  for (int64_t e = threadIdx.x; e < mn; e += blockDim.x) R[e] = A[e];
  __syncthreads();
  for (;;) {
    double best = -1.0, bval = 0.0, ss = 0.0;
    int64_t bidx = INT64_MAX;
    for (int64_t e = threadIdx.x; e < mn; e += blockDim.x) {
      double v = R[e];
      if (have_term) {
        const int i = (int)(e % m), j = (int)(e / m);
        v = v - ucur[i] * vcur[j];
        R[e] = v;
      }
      ss = fma(v, v, ss);
      double a = fabs(v);
      if (a > best) { best = a; bidx = e; bval = v; }
    }
    warp_argmax(best, bidx, bval);
    __syncthreads();
    if (lane == 0) { s_a[w] = best; s_i[w] = bidx; s_v[w] = bval; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = s_a[0]; int64_t bi = s_i[0]; double bv = s_v[0];
      for (int q = 1; q < nw; ++q)
        if (s_a[q] > b || (s_a[q] == b && s_i[q] < bi)) { b = s_a[q]; bi = s_i[q]; bv = s_v[q]; }
      s_sel = bi; s_max = bv;
    }
    const double Rnorm = sqrt(block_sum(ss, red));
    const int64_t sel = s_sel;
    const double Max = s_max;
    if (isnan(Rnorm)) { status = 2; break; }
    if (!((rank < maxr && Rnorm > eps && Rnorm > meps) || rank < 1)) break;
    const int sel_row = (int)(sel % m), sel_col = (int)(sel / m);
    // all threads have read the previous ucur/vcur in the pass above
    __syncthreads();
    if (fabs(Max) > meps && !isnan(Max)) {
      const double gamma = 1.0 / Max;
      for (int i = threadIdx.x; i < m; i += blockDim.x) ucur[i] = gamma * R[i + (int64_t)sel_col * m];
      for (int j = threadIdx.x; j < n; j += blockDim.x) vcur[j] = R[sel_row + (int64_t)j * m];
    } else {
      for (int i = threadIdx.x; i < m; i += blockDim.x) ucur[i] = (i == rank) ? 1.0 : 0.0;
      for (int j = threadIdx.x; j < n; j += blockDim.x) vcur[j] = 0.0;
    }
    __syncthreads();
    if (rank < keep) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) U[i + (int64_t)rank * m] = ucur[i];
      for (int j = threadIdx.x; j < n; j += blockDim.x) V[j + (int64_t)rank * n] = vcur[j];
    }
    have_term = true;
    ++rank;
  }
  if (status == 2) {
    // NaN residual: full-rank fallback of ACA_FullyPivoted.cpp:122-147
    rank = (m < n) ? m : n;
    const int kk = min(rank, keep);
    for (int64_t e = threadIdx.x; e < (int64_t)m * kk; e += blockDim.x) {
      const int i = (int)(e % m), c = (int)(e / m);
      U[e] = (m < n) ? (i == c ? 1.0 : 0.0) : A[e];
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * kk; e += blockDim.x) {
      const int j = (int)(e % n), c = (int)(e / n);
      V[e] = (m < n) ? A[c + (int64_t)j * m] : (j == c ? 1.0 : 0.0);
    }
  }
  if (threadIdx.x == 0) {
    res[0] = (double)rank;
    res[1] = (double)status;
  }
}

}  // namespace hm

using namespace hm;

extern "C" int aca_wrapper_noalloc(const double* A, double* U, double* V, int m, int n, double epsilon, int rank,
                                   void* stream) {
  if (!A || !U || !V || m <= 0 || n <= 0 || rank < 0) {
    fail(HM_ERR_ARG, "aca_wrapper_noalloc: invalid argument");
    return -HM_ERR_ARG;
  }
  const int64_t need = (int64_t)m * n + m + n;
  if (need > NOALLOC_MAX_ELEMS) {
    fail(HM_ERR_ARG, "aca_wrapper_noalloc: m*n + m + n = " + std::to_string(need) +
                         " exceeds the fixed scratch of " + std::to_string(NOALLOC_MAX_ELEMS) +
                         " doubles; use aca_wrapper for larger blocks");
    return -HM_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    fail(HM_ERR_CUDA, "aca_wrapper_noalloc: no current CUDA device");
    return -HM_ERR_CUDA;
  }
  double* scratch = nullptr;
  int s = scratch_address(dev, &scratch);
  if (s != HM_OK) return -s;
  cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamLegacy;
  const int keep = std::min(std::min(m, n), rank + 1);
  aca_fp_noalloc_kernel<<<1, 512, 0, st>>>(A, U, V, m, n, epsilon, keep, scratch);
  cudaError_t e = cudaGetLastError();
  double res[2] = {0.0, 0.0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(res, scratch, sizeof(res), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    fail(HM_ERR_CUDA, std::string("aca_wrapper_noalloc: ") + cudaGetErrorString(e));
    return -HM_ERR_CUDA;
  }
  return (int)res[0];
}
