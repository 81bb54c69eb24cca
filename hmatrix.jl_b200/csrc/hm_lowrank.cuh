// Low-rank building blocks shared by construction and H-LU:
//  * batched partially pivoted ACA ("aca2", src/hlu.jl:59-111)
//  * fully pivoted ACA (deps/src/ACA_FullyPivoted.cpp:9-151)
//  * recompression core: QR of both factors + SVD of the small core +
//    truncation by the relative tolerance eps_trunc (src/harithm.jl:49-56,
//    374-396 with compress of src/hlu.jl:159-190).
#pragma once
#include "hm_internal.h"

#include <map>
#include <vector>

namespace hm {

constexpr int ACA_MAX_EXTENT = 2048;   // largest block side for device aca2
constexpr int RCORE_MAX = 96;          // largest core of the QR+SVD recompression
constexpr int MV_KMAX = 4096;          // largest rank a leaf may carry (bbfmm 2-D: 64^2)

// ---------------------------------------------------------------------------
// warp / block reductions (fixed order: results are reproducible run to run)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// arg-max of |v| with the smallest index on ties; returns the winner in all lanes
__device__ __forceinline__ void warp_argmax(double& a, int64_t& idx, double& val) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double a2 = __shfl_xor_sync(0xffffffffu, a, o);
    int64_t i2 = __shfl_xor_sync(0xffffffffu, idx, o);
    double v2 = __shfl_xor_sync(0xffffffffu, val, o);
    if (a2 > a || (a2 == a && i2 < idx)) { a = a2; idx = i2; val = v2; }
  }
}

// block-wide sum; `red` must hold >= 32 doubles; all threads get the result
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];   // same order in every thread
  return s;
}

// ---------------------------------------------------------------------------
// host-side helpers implemented in hm_lowrank.cu
// ---------------------------------------------------------------------------

// FP64 factors of the "svd"-route low-rank candidates, kept per block-tree node
struct SvdCandidateStore {
  struct F { int m, n, k; std::vector<double> A, B; };
  std::map<int32_t, F> by_node;
  int rank_of(int32_t node) const {
    auto it = by_node.find(node);
    return it == by_node.end() ? 0 : it->second.k;
  }
  int write_pool(hm_handle* h, const std::vector<int64_t>& rk_leaf) const;
};

int svd_compress_candidates(hm_handle* h, const std::vector<int64_t>& r0,
                            const std::vector<int64_t>& c0, const std::vector<int32_t>& m,
                            const std::vector<int32_t>& n, std::vector<int32_t>& ranks,
                            SvdCandidateStore& store, const std::vector<int32_t>& nodes);
int aca2_ranks(hm_handle* h, const std::vector<int64_t>& rk_leaf, std::vector<int32_t>& ranks);
int aca2_write(hm_handle* h, const std::vector<int64_t>& rk_leaf, bool replay = false);
int fill_pools(hm_handle* h, const std::vector<int64_t>& rk_leaf, bool replay, const SvdCandidateStore* svd_store);
// Chebyshev-interpolation ("bbfmm") leaves: the rank of an m x n leaf, and
// the factors of every low-rank leaf written into the pool
int bbfmm_rank(int64_t m, int64_t n, int dim, int max_rank);
int bbfmm_write(hm_handle* h, const std::vector<int64_t>& rk_leaf);

// One recompression problem for the batched QR+SVD core kernel.  A (m x r,
// column stride lda) and B (n x r, stride ldb) are FP64 device buffers that
// are overwritten with their orthonormal Q factors; the truncated result
// A' (m x k) and B' (n x k) goes to outA/outB (column strides ldoa/ldob,
// capacity kcap columns), with H = A' B'.  k is written to *rank.
struct CoreJob {
  double* A; double* B;
  double* outA; double* outB;
  int32_t m, n, r, lda, ldb, ldoa, ldob, kcap;
  int32_t zero_test;       // apply compress()'s sum|W| < 1e-5 test to the core
  int32_t* rank;
  const int32_t* r_dev;    // if set: the core size r is read on the device
  const int32_t* pre_status;  // if set: status of the fully pivoted ACA that made A, B
  int32_t zero_fill;       // zero the output columns [k, kcap)
  int32_t known_zero;      // the output's columns [zero_from, kcap) are zero already:
  int32_t zero_from;       // zero_fill stops there (writes only what changes)
  int32_t ortho_k;         // the first ortho_k columns of A are orthonormal and those of B
                           // mutually orthogonal (a previous core's output): no QR for them
};

// Fully pivoted ACA job (deps/src/ACA_FullyPivoted.cpp:9-151).  rel_mode: the
// "svd"-compress mode -- status 3 for an absolutely tiny block (sum|R| < 1e-5)
// and a stop tolerance derived on the device from |R|_F and eps_trunc.
struct AcaFpJob {
  double* R; double* U; double* V;
  int32_t m, n, cap, min_rank;
  double eps;
  int32_t* rank; int32_t* status;
  int32_t rel_mode;
  double eps_trunc;
};
int launch_aca_fp_one(const AcaFpJob& J, cudaStream_t st);
int launch_aca_fp(const AcaFpJob* d_jobs, int njobs, cudaStream_t st);   // one CTA per job
int launch_core_one(const CoreJob& J, double eps_trunc, int* d_flags, cudaStream_t st);
// launch the batched recompression; status of rank overflow/nonfinite is
// OR-ed into *d_flags (bit 0: rank > kcap, bit 1: non-finite).
// jac8: the Jacobi rounds and ordering of the H-LU's recompressions (core_body_t)
int launch_core_recompress(const CoreJob* d_jobs, int njobs, int rmax, double eps_trunc,
                           int* d_flags, cudaStream_t st, bool jac8 = false);

}  // namespace hm
