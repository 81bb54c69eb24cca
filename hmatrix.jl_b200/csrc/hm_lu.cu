// H-LU and triangular H-solve on the device (src/hlu.jl:227-562, with the
// H-arithmetic of src/harithm.jl:4-420 that the Schur updates use).
//
// The host walks the same recursion as the reference -- lu!, permute_hmat!,
// hmat_trisolve!, mat_full_solve, hmat_sub_mul! = hmul + hmat_add!, and the
// recompressions of rkmat_add!, rkmat_hmat_add and compress -- and issues one
// stream-ordered kernel per primitive.  Nothing is read back during the
// factorisation: ranks live on the device, every low-rank buffer has a fixed
// capacity `cap` and keeps its columns beyond the current rank at zero, so
// every product can run with static shapes.  Temporaries are stream-ordered
// allocations (cudaMallocAsync / cudaFreeAsync).  Pivoting is partial and
// stays inside each diagonal leaf, exactly as in the reference; the global
// permutation is one device array P with H[P,:] = L U.
#include "hm_internal.h"
#include "hm_lowrank.cuh"
#include "hm_core.cuh"


#include <algorithm>
#include <map>
#include <memory>
#include <stdexcept>

namespace hm {

// ---------------------------------------------------------------------------
// strided views: element (i,j) at p[i*rs + j*cs]
// ---------------------------------------------------------------------------
struct View {
  double* p;
  int64_t rs, cs;
  int rows, cols;
};
static inline View vsub(View v, int r0, int c0, int nr, int nc) {
  return View{v.p + (int64_t)r0 * v.rs + (int64_t)c0 * v.cs, v.rs, v.cs, nr, nc};
}
static inline View vtr(View v) { return View{v.p, v.cs, v.rs, v.cols, v.rows}; }
static inline View vrev(View v) {
  return View{v.p + (int64_t)(v.rows - 1) * v.rs + (int64_t)(v.cols - 1) * v.cs, -v.rs, -v.cs, v.rows, v.cols};
}

struct LuError : std::runtime_error {
  int code;
  LuError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HM_LU_CUDA(expr)                                                                    \
  do {                                                                                      \
    cudaError_t _e = (expr);                                                                \
    if (_e != cudaSuccess) throw LuError(HM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)
#define LU_LAUNCH_CHECK()                                                                   \
  do {                                                                                      \
    cudaError_t _e = cudaGetLastError();                                                    \
    if (_e != cudaSuccess) throw LuError(HM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(_e)); \
  } while (0)

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// C = alpha * A * B + beta * C   (A: m x k, B: k x n), FP64, 32x32 tiles
__device__ __forceinline__ void gemm_tile(const View& A, const View& B, const View& C, double alpha, double beta,
                                          int i0, int j0) {
  __shared__ double As[32][33];
  __shared__ double Bs[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int m = C.rows, n = C.cols, kk = A.cols;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < kk; k0 += 32) {
    for (int e = threadIdx.x; e < 1024; e += 256) {
      const int r = e & 31, c = e >> 5;
      As[r][c] = (i0 + r < m && k0 + c < kk) ? A.p[(int64_t)(i0 + r) * A.rs + (int64_t)(k0 + c) * A.cs] : 0.0;
      Bs[r][c] = (k0 + r < kk && j0 + c < n) ? B.p[(int64_t)(k0 + r) * B.rs + (int64_t)(j0 + c) * B.cs] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int q = 0; q < 32; ++q) {
      const double a = As[tx][q];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] = fma(a, Bs[q][ty + 8 * u], acc[u]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int i = i0 + tx, j = j0 + ty + 8 * u;
    if (i < m && j < n) {
      double* c = C.p + (int64_t)i * C.rs + (int64_t)j * C.cs;
      *c = (beta == 0.0) ? alpha * acc[u] : fma(alpha, acc[u], beta * *c);
    }
  }
}

__global__ void __launch_bounds__(256) lu_gemm_kernel(View A, View B, View C, double alpha, double beta) {
  gemm_tile(A, B, C, alpha, beta, blockIdx.y * 32, blockIdx.x * 32);
}

// a batch of independent products, one job per blockIdx.z
struct GemmJob {
  View A, B, C;
  double alpha, beta;
};
__global__ void __launch_bounds__(256) lu_gemm_batch_kernel(const GemmJob* __restrict__ jobs) {
  const GemmJob& J = jobs[blockIdx.z];
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  if (i0 >= J.C.rows || j0 >= J.C.cols) return;
  gemm_tile(J.A, J.B, J.C, J.alpha, J.beta, i0, j0);
}

// Large products (the tile schedule's B_ik' A_kj cores and Q_i = A_ik W): C
// tiles of 128 x 128 per CTA, K in steps of 16 through shared memory, 8 x 8
// outputs per thread (rows tx + 16 u, columns 8 ty + v, so that a warp's
// stores of column-major C are 128-byte runs).  Tiles are read along whichever
// stride of the view is 1, so transposed views stay coalesced.
constexpr int GB_T = 128, GB_K = 16, GB_LD = GB_T + 4;
__device__ __forceinline__ void gemm_big_tile(const View& A, const View& B, const View& C, double alpha,
                                              double beta, int i0, int j0) {
  __shared__ __align__(16) double As[GB_K][GB_LD];
  __shared__ __align__(16) double Bs[GB_K][GB_LD];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m = C.rows, n = C.cols, K = A.cols;
  double acc[8][8];
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[u][v] = 0.0;
  // the next K step's tiles are loaded into registers while this one is
  // multiplied, so the global loads overlap the FMAs
  double ra[8], rb[8];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 256 * q;
      int i, kk;
      if (A.rs == 1) { i = e & 127; kk = e >> 7; } else { kk = e & 15; i = e >> 4; }
      ra[q] = (i0 + i < m && k0 + kk < K) ? A.p[(int64_t)(i0 + i) * A.rs + (int64_t)(k0 + kk) * A.cs] : 0.0;
      int j;
      if (B.rs == 1) { kk = e & 15; j = e >> 4; } else { j = e & 127; kk = e >> 7; }
      rb[q] = (k0 + kk < K && j0 + j < n) ? B.p[(int64_t)(k0 + kk) * B.rs + (int64_t)(j0 + j) * B.cs] : 0.0;
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 256 * q;
      int i, kk;
      if (A.rs == 1) { i = e & 127; kk = e >> 7; } else { kk = e & 15; i = e >> 4; }
      As[kk][i] = ra[q];
      int j;
      if (B.rs == 1) { kk = e & 15; j = e >> 4; } else { j = e & 127; kk = e >> 7; }
      Bs[kk][j] = rb[q];
    }
  };
  load(0);
  for (int k0 = 0; k0 < K; k0 += GB_K) {
    stash();
    __syncthreads();
    if (k0 + GB_K < K) load(k0 + GB_K);
#pragma unroll 4
    for (int kk = 0; kk < GB_K; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] = As[kk][tx + 16 * u];
#pragma unroll
      for (int v = 0; v < 8; v += 2) {
        const double2 t = *reinterpret_cast<const double2*>(&Bs[kk][8 * ty + v]);
        b[v] = t.x;
        b[v + 1] = t.y;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const int j = j0 + 8 * ty + v;
    if (j >= n) continue;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + tx + 16 * u;
      if (i < m) {
        double* c = C.p + (int64_t)i * C.rs + (int64_t)j * C.cs;
        *c = (beta == 0.0) ? alpha * acc[u][v] : fma(alpha, acc[u][v], beta * *c);
      }
    }
  }
}
__global__ void __launch_bounds__(256) lu_gemm_big_kernel(View A, View B, View C, double alpha, double beta) {
  gemm_big_tile(A, B, C, alpha, beta, blockIdx.y * GB_T, blockIdx.x * GB_T);
}
__global__ void __launch_bounds__(256) lu_gemm_big_batch_kernel(const GemmJob* __restrict__ jobs) {
  const GemmJob& J = jobs[blockIdx.z];
  const int i0 = blockIdx.y * GB_T, j0 = blockIdx.x * GB_T;
  if (i0 >= J.C.rows || j0 >= J.C.cols) return;
  gemm_big_tile(J.A, J.B, J.C, J.alpha, J.beta, i0, j0);
}

// Y = alpha * X + beta * Y (beta == 0: Y is not read)
__global__ void lu_axpby_kernel(View Y, View X, double alpha, double beta) {
  const int64_t tot = (int64_t)Y.rows * Y.cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % Y.rows), j = (int)(e / Y.rows);
    double* y = Y.p + (int64_t)i * Y.rs + (int64_t)j * Y.cs;
    const double x = X.p ? X.p[(int64_t)i * X.rs + (int64_t)j * X.cs] : 0.0;
    *y = (beta == 0.0) ? alpha * x : fma(alpha, x, beta * *y);
  }
}

// X <- L^{-1} X, L (m x m) lower triangular (strided: upper/transposed/reversed
// triangles are views of this one), one thread per column of X.
__global__ void __launch_bounds__(128) lu_trsm_lower_kernel(View L, View X, int unit) {
  extern __shared__ double Ls[];
  const int m = L.rows;
  const bool sm = m <= 96;
  if (sm) {
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = e % m, j = e / m;
      Ls[e] = (j <= i) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : 0.0;
    }
    __syncthreads();
  }
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= X.cols) return;
  double* x = X.p + (int64_t)j * X.cs;
  for (int i = 0; i < m; ++i) {
    double s = x[(int64_t)i * X.rs];
    for (int l = 0; l < i; ++l) {
      const double lil = sm ? Ls[i + l * m] : L.p[(int64_t)i * L.rs + (int64_t)l * L.cs];
      s = fma(-lil, x[(int64_t)l * X.rs], s);
    }
    if (!unit) s = s / (sm ? Ls[i + i * m] : L.p[(int64_t)i * L.rs + (int64_t)i * L.cs]);
    x[(int64_t)i * X.rs] = s;
  }
}

// The same solve for triangles of at most MM rows (diagonal leaves): one warp
// per 32 columns of X, each column held in registers, loops fully unrolled.
template <int MM>
__global__ void __launch_bounds__(32) lu_trsm_small_kernel(View L, View X, int unit) {
  __shared__ double Ls[MM * MM];
  const int m = L.rows;
  for (int e = threadIdx.x; e < m * m; e += 32) {
    const int i = e % m, j = e / m;
    Ls[i + j * MM] = (j <= i) ? L.p[(int64_t)i * L.rs + (int64_t)j * L.cs] : 0.0;
  }
  __syncwarp();
  const int j = blockIdx.x * 32 + threadIdx.x;
  if (j >= X.cols) return;
  double* xp = X.p + (int64_t)j * X.cs;
  double x[MM];
#pragma unroll
  for (int i = 0; i < MM; ++i) x[i] = (i < m) ? xp[(int64_t)i * X.rs] : 0.0;
#pragma unroll
  for (int i = 0; i < MM; ++i) {
    if (i < m) {
      double s = x[i];
#pragma unroll
      for (int l = 0; l < i; ++l) s = fma(-Ls[i + l * MM], x[l], s);
      if (!unit) s = s / Ls[i + i * MM];
      x[i] = s;
    }
  }
#pragma unroll
  for (int i = 0; i < MM; ++i)
    if (i < m) xp[(int64_t)i * X.rs] = x[i];
}

// getrf of a leaf of at most 64 rows by one warp (same pivoting and
// arithmetic as lu_getrf_kernel; padded shared tile, warp barriers only)
__global__ void __launch_bounds__(32) lu_getrf_small_kernel(View C, int64_t* __restrict__ P, int64_t goff,
                                                            int* __restrict__ flags) {
  constexpr int LD = 65;
  __shared__ double S[64 * LD];
  __shared__ int perm[64];
  const int m = C.rows, lane = threadIdx.x;
  for (int e = lane; e < m * m; e += 32) {
    const int i = e % m, j = e / m;
    S[i + j * LD] = C.p[(int64_t)i * C.rs + (int64_t)j * C.cs];
  }
  for (int i = lane; i < m; i += 32) perm[i] = i;
  __syncwarp();
  for (int j = 0; j < m; ++j) {
    double best = -1.0, bv = 0.0;
    int64_t bi = INT64_MAX;
    for (int i = j + lane; i < m; i += 32) {
      const double a = fabs(S[i + j * LD]);
      if (a > best) { best = a; bi = i; bv = S[i + j * LD]; }
    }
    warp_argmax(best, bi, bv);
    if (lane == 0 && !(bv != 0.0)) atomicOr(flags, bi == INT64_MAX ? 6 : 4);
    // every candidate NaN: no maximum was found; keep the row (flagged above)
    const int p = bi == INT64_MAX ? j : (int)bi;
    if (p != j) {
      for (int c = lane; c < m; c += 32) {
        const double t = S[j + c * LD];
        S[j + c * LD] = S[p + c * LD];
        S[p + c * LD] = t;
      }
      if (lane == 0) { const int t = perm[j]; perm[j] = perm[p]; perm[p] = t; }
    }
    __syncwarp();
    const double piv = S[j + j * LD];
    if (piv != 0.0)
      for (int i = j + 1 + lane; i < m; i += 32) S[i + j * LD] /= piv;
    __syncwarp();
    for (int c = j + 1 + lane; c < m; c += 32) {
      const double ujc = S[j + c * LD];
      for (int i = j + 1; i < m; ++i) S[i + c * LD] = fma(-S[i + j * LD], ujc, S[i + c * LD]);
    }
    __syncwarp();
  }
  for (int e = lane; e < m * m; e += 32) {
    const int i = e % m, j = e / m;
    C.p[(int64_t)i * C.rs + (int64_t)j * C.cs] = S[i + j * LD];
  }
  for (int i = lane; i < m; i += 32) P[goff + i] = goff + perm[i];
}

// getrf with partial pivoting of an m x m dense leaf (LAPACK semantics: first
// maximum as pivot, full-row swaps); P[goff+i] = goff + p[i] with C[p] = L U.
__global__ void __launch_bounds__(256) lu_getrf_kernel(View C, int64_t* __restrict__ P, int64_t goff,
                                                       int* __restrict__ flags) {
  extern __shared__ double S[];
  const int m = C.rows;
  int* perm = reinterpret_cast<int*>(S + (int64_t)m * m);
  __shared__ int s_piv;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int i = e % m, j = e / m;
    S[e] = C.p[(int64_t)i * C.rs + (int64_t)j * C.cs];
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) perm[i] = i;
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    if (threadIdx.x < 32) {
      double best = -1.0, bv = 0.0;
      int64_t bi = INT64_MAX;
      for (int i = j + threadIdx.x; i < m; i += 32) {
        const double a = fabs(S[i + j * m]);
        if (a > best) { best = a; bi = i; bv = S[i + j * m]; }
      }
      warp_argmax(best, bi, bv);
      if (threadIdx.x == 0) {
        // every candidate NaN: no maximum was found; keep the row
        s_piv = bi == INT64_MAX ? j : (int)bi;
        if (!(bv != 0.0)) atomicOr(flags, bi == INT64_MAX ? 6 : 4);   // exactly zero (or NaN) pivot
      }
    }
    __syncthreads();
    const int p = s_piv;
    if (p != j) {
      for (int c = threadIdx.x; c < m; c += blockDim.x) {
        const double t = S[j + c * m];
        S[j + c * m] = S[p + c * m];
        S[p + c * m] = t;
      }
      if (threadIdx.x == 0) { const int t = perm[j]; perm[j] = perm[p]; perm[p] = t; }
    }
    __syncthreads();
    const double piv = S[j + j * m];
    if (piv != 0.0) {
      for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) S[i + j * m] /= piv;
    }
    __syncthreads();
    const int rem = m - j - 1;
    for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
      const int i = j + 1 + e % rem, c = j + 1 + e / rem;
      S[i + c * m] = fma(-S[i + j * m], S[j + c * m], S[i + c * m]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int i = e % m, j = e / m;
    C.p[(int64_t)i * C.rs + (int64_t)j * C.cs] = S[e];
  }
  for (int i = threadIdx.x; i < m; i += blockDim.x) P[goff + i] = goff + perm[i];
}

// X <- X[p, :] with p[i] = P[goff+i] - goff, columns in chunks through smem
__global__ void lu_laswp_kernel(View X, const int64_t* __restrict__ P, int64_t goff, int chunk) {
  extern __shared__ double T[];
  const int m = X.rows;
  const int c0 = blockIdx.x * chunk;
  const int nc = min(chunk, X.cols - c0);
  for (int e = threadIdx.x; e < m * nc; e += blockDim.x) {
    const int i = e % m, c = e / m;
    const int64_t src = P[goff + i] - goff;
    T[e] = X.p[src * X.rs + (int64_t)(c0 + c) * X.cs];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < m * nc; e += blockDim.x) {
    const int i = e % m, c = e / m;
    X.p[(int64_t)i * X.rs + (int64_t)(c0 + c) * X.cs] = T[e];
  }
}

// y[i, c] = b[P[i], c]
__global__ void lu_gather_rows_kernel(View Y, View Bv, const int64_t* __restrict__ P) {
  const int64_t tot = (int64_t)Y.rows * Y.cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % Y.rows), c = (int)(e / Y.rows);
    Y.p[(int64_t)i * Y.rs + (int64_t)c * Y.cs] = Bv.p[P[i] * Bv.rs + (int64_t)c * Bv.cs];
  }
}

// pieces of a low-rank sum, gathered into contiguous [s_i A_i] / [B_i] with
// their first k_i columns, rows placed at offsets ro_i / co_i (zeros
// elsewhere) -- the concatenations of rkmat_add! and rkmat_hmat_add
struct Piece {
  const double* A; int64_t lda;
  const double* B; int64_t ldb;
  const int32_t* k;
  int m, n, ro, co;
  double s;
};
constexpr int MAX_PIECES = 4;
struct GatherArgs {
  Piece pc[MAX_PIECES];
  int np;
  double* SA; double* SB;     // M x rmax, N x rmax
  int M, N, rmax;
  int32_t* r_out;
  int* flags;
};
__device__ void gather_pieces(const GatherArgs& g);
__global__ void __launch_bounds__(256) lu_gather_pieces_kernel(GatherArgs g) { gather_pieces(g); }
__global__ void __launch_bounds__(256) lu_gather_pieces_batch_kernel(const GatherArgs* __restrict__ jobs) {
  gather_pieces(jobs[blockIdx.x]);
}

__device__ void gather_pieces(const GatherArgs& g) {
  __shared__ int pre[MAX_PIECES + 1];
  if (threadIdx.x == 0) {
    int t = 0;
    for (int q = 0; q < g.np; ++q) { pre[q] = t; t += *g.pc[q].k; }
    pre[g.np] = t;
    if (t > g.rmax) atomicOr(g.flags, 1);
    *g.r_out = t;
  }
  __syncthreads();
  const int r = min(pre[g.np], g.rmax);
  for (int64_t e = threadIdx.x; e < (int64_t)g.M * r; e += blockDim.x) {
    const int i = (int)(e % g.M), c = (int)(e / g.M);
    int q = 0;
    while (q + 1 < g.np && pre[q + 1] <= c) ++q;
    const Piece& P = g.pc[q];
    const int cc = c - pre[q];
    const int ii = i - P.ro;
    g.SA[e] = (ii >= 0 && ii < P.m) ? P.s * P.A[ii + (int64_t)cc * P.lda] : 0.0;
  }
  for (int64_t e = threadIdx.x; e < (int64_t)g.N * r; e += blockDim.x) {
    const int j = (int)(e % g.N), c = (int)(e / g.N);
    int q = 0;
    while (q + 1 < g.np && pre[q + 1] <= c) ++q;
    const Piece& P = g.pc[q];
    const int cc = c - pre[q];
    const int jj = j - P.co;
    g.SB[e] = (jj >= 0 && jj < P.n) ? P.B[jj + (int64_t)cc * P.ldb] : 0.0;
  }
}

__global__ void lu_copy_int_kernel(int32_t* dst, const int32_t* src) { *dst = *src; }

__global__ void lu_max_int_kernel(const int32_t* __restrict__ v, int n, int32_t* __restrict__ out) {
  __shared__ int32_t red[256];
  int32_t m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = max(m, v[i]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}
__global__ void lu_set_int_kernel(int32_t* dst, int v) { *dst = v; }

template <typename T>
__global__ void lu_load_kernel(const T* __restrict__ src, int64_t ld_src, int rows, int cols, double* __restrict__ dst,
                               int64_t ld_dst, int dst_cols) {
  const int64_t tot = (int64_t)rows * dst_cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % rows), c = (int)(e / rows);
    dst[i + (int64_t)c * ld_dst] = c < cols ? from_store<T>(src[i + (int64_t)c * ld_src]) : 0.0;
  }
}

// ---------------------------------------------------------------------------
// host-side block tree of the factorisation and of the temporaries
// ---------------------------------------------------------------------------
struct Blk;
using BP = std::shared_ptr<Blk>;

struct Ctx {
  cudaStream_t st;
  int cap;
  int64_t* P;          // device permutation
  int* flags;          // device error bits: 1 rank overflow, 2 non-finite, 4 singular
  double eps_trunc;
  const hm_handle* h;
  struct Arena* ar = nullptr;      // when set, temporaries come from this fixed buffer
};

// A fixed device buffer handed out front to back; nothing is returned before
// the sequence that uses it ends.  A captured solve takes its temporaries from
// one, so the graph holds no allocation nodes.
struct Arena {
  char* base = nullptr;
  size_t size = 0, used = 0;
};
static inline size_t arena_round(size_t b) { return (std::max<size_t>(b, 8) + 255) & ~(size_t)255; }

struct Blk {
  int8_t type = T_H;
  int m = 0, n = 0;
  int32_t s = -1, t = -1;             // clusters (for the isleaf tests of hmul)
  int64_t row0 = 0;                   // global first row (persistent blocks)
  double* C = nullptr;                // dense, column-major, ld = ldc
  int64_t ldc = 0;
  double* A = nullptr;                // low-rank: A (m x cap), B (n x cap)
  double* B = nullptr;
  int64_t lda = 0, ldb = 0;
  int32_t* k = nullptr;
  int cap = 0;
  BP ch[4];
  std::vector<void*> own;
  cudaStream_t st = nullptr;
  ~Blk() {
    for (void* p : own) cudaFreeAsync(p, st);
  }
  View Cv() const { return View{C, 1, ldc, m, n}; }
  View Av() const { return View{A, 1, lda, m, cap}; }
  View Bv() const { return View{B, 1, ldb, n, cap}; }
};

struct JobTape;
static thread_local JobTape* g_tape = nullptr;
static void tape_note_temporary(size_t bytes);

static void* dmalloc(Ctx& c, Blk& b, size_t bytes) {
  if (c.ar) {
    const size_t r = arena_round(bytes);
    if (c.ar->used + r > c.ar->size) throw LuError(HM_ERR_CUDA, "solve arena exhausted");
    void* q = c.ar->base + c.ar->used;
    c.ar->used += r;
    return q;
  }
  tape_note_temporary(bytes);
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, std::max<size_t>(bytes, 8), c.st);
  if (e != cudaSuccess) throw LuError(HM_ERR_OOM, std::string("H-LU temporary: ") + cudaGetErrorString(e));
  b.own.push_back(p);
  return p;
}

static BP new_dense(Ctx& c, int m, int n, int32_t s, int32_t t) {
  BP b = std::make_shared<Blk>();
  b->st = c.st;
  b->type = T_DENSE; b->m = m; b->n = n; b->s = s; b->t = t;
  b->C = (double*)dmalloc(c, *b, sizeof(double) * (size_t)m * n);
  b->ldc = std::max(m, 1);
  return b;
}

static BP new_rk(Ctx& c, int m, int n, int32_t s, int32_t t, bool alloc_a = true, bool alloc_b = true) {
  BP b = std::make_shared<Blk>();
  b->st = c.st;
  b->type = T_RK; b->m = m; b->n = n; b->s = s; b->t = t; b->cap = c.cap;
  if (alloc_a) { b->A = (double*)dmalloc(c, *b, sizeof(double) * (size_t)m * c.cap); b->lda = std::max(m, 1); }
  if (alloc_b) { b->B = (double*)dmalloc(c, *b, sizeof(double) * (size_t)n * c.cap); b->ldb = std::max(n, 1); }
  b->k = (int32_t*)dmalloc(c, *b, sizeof(int32_t));
  return b;
}

static bool is_leaf_cluster(const Ctx& c, int32_t cl) { return cl >= 0 && c.h->cl_left[cl] < 0; }

// ---- primitive launches --------------------------------------------------

static void gemm(Ctx& c, View C, View A, View B, double alpha, double beta) {
  if (C.rows == 0 || C.cols == 0) return;
  // 128 x 128 tiles once they fill the GPU; medium products keep the 32 x 32
  // tiles (more CTAs)
  const int64_t big_tiles = (int64_t)((C.rows + GB_T - 1) / GB_T) * ((C.cols + GB_T - 1) / GB_T);
  if (A.cols > 0 && (double)C.rows * C.cols * A.cols >= 4.0e6 && big_tiles >= 148) {
    dim3 g((C.cols + GB_T - 1) / GB_T, (C.rows + GB_T - 1) / GB_T);
    lu_gemm_big_kernel<<<g, 256, 0, c.st>>>(A, B, C, alpha, beta);
    LU_LAUNCH_CHECK();
    return;
  }
  if (A.cols == 0) {
    if (beta != 1.0) {
      lu_axpby_kernel<<<64, 256, 0, c.st>>>(C, View{nullptr, 0, 0, C.rows, C.cols}, 0.0, beta);
      LU_LAUNCH_CHECK();
    }
    return;
  }
  dim3 g((C.cols + 31) / 32, (C.rows + 31) / 32);
  lu_gemm_kernel<<<g, 256, 0, c.st>>>(A, B, C, alpha, beta);
  LU_LAUNCH_CHECK();
}

static void axpby(Ctx& c, View Y, View X, double alpha, double beta) {
  const int64_t tot = (int64_t)Y.rows * Y.cols;
  if (tot == 0) return;
  unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, 1024);
  lu_axpby_kernel<<<g, 256, 0, c.st>>>(Y, X, alpha, beta);
  LU_LAUNCH_CHECK();
}

static void trsm_lower(Ctx& c, View L, View X, bool unit) {
  if (X.cols == 0 || L.rows == 0) return;
  if (L.rows <= 32) {
    lu_trsm_small_kernel<32><<<(X.cols + 31) / 32, 32, 0, c.st>>>(L, X, unit ? 1 : 0);
    LU_LAUNCH_CHECK();
    return;
  }
  if (L.rows <= 64) {
    lu_trsm_small_kernel<64><<<(X.cols + 31) / 32, 32, 0, c.st>>>(L, X, unit ? 1 : 0);
    LU_LAUNCH_CHECK();
    return;
  }
  if (smem_attr((const void*)lu_trsm_lower_kernel, 96 * 96 * (int)sizeof(double)) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "trsm smem attribute");
  const size_t smem = L.rows <= 96 ? sizeof(double) * (size_t)L.rows * L.rows : 0;
  lu_trsm_lower_kernel<<<(X.cols + 127) / 128, 128, smem, c.st>>>(L, X, unit ? 1 : 0);
  LU_LAUNCH_CHECK();
}

static void getrf(Ctx& c, View C, int64_t goff) {
  const int m = C.rows;
  if (m != C.cols) throw LuError(HM_ERR_UNSUPPORTED, "non-square diagonal leaf");
  if (m <= 64) {
    lu_getrf_small_kernel<<<1, 32, 0, c.st>>>(C, c.P, goff, c.flags);
    LU_LAUNCH_CHECK();
    return;
  }
  const size_t smem = sizeof(double) * (size_t)m * m + sizeof(int) * m;
  if (smem > 200 * 1024) throw LuError(HM_ERR_UNSUPPORTED, "diagonal leaf above 150 rows (MinBlock too large)");
  if (smem_attr((const void*)lu_getrf_kernel, 200 * 1024) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "getrf smem attribute");
  lu_getrf_kernel<<<1, 256, smem, c.st>>>(C, c.P, goff, c.flags);
  LU_LAUNCH_CHECK();
}

static void laswp(Ctx& c, View X, int64_t goff) {
  if (X.rows == 0 || X.cols == 0) return;
  int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(X.cols, (48 * 1024 / 8) / X.rows));
  const size_t smem = sizeof(double) * (size_t)X.rows * chunk;
  lu_laswp_kernel<<<(X.cols + chunk - 1) / chunk, 256, smem, c.st>>>(X, c.P, goff, chunk);
  LU_LAUNCH_CHECK();
}

static void copy_int(Ctx& c, int32_t* dst, const int32_t* src) {
  lu_copy_int_kernel<<<1, 1, 0, c.st>>>(dst, src);
  LU_LAUNCH_CHECK();
}

// ---- recompression --------------------------------------------------------
// target (low-rank) = truncated sum of pieces: QR of both concatenations and
// compress() of the core (src/harithm.jl:374-396, 49-56, src/hlu.jl:159-190)
static void recompress(Ctx& c, Blk& target, const std::vector<Piece>& pcs) {
  if (pcs.size() > (size_t)MAX_PIECES) throw LuError(HM_ERR_UNSUPPORTED, "too many pieces");
  Blk tmp;
  tmp.st = c.st;
  const int M = target.m, N = target.n;
  double* SA = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)M * RCORE_MAX);
  double* SB = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)N * RCORE_MAX);
  int32_t* r = (int32_t*)dmalloc(c, tmp, sizeof(int32_t));
  GatherArgs g{};
  for (size_t q = 0; q < pcs.size(); ++q) g.pc[q] = pcs[q];
  g.np = (int)pcs.size();
  g.SA = SA; g.SB = SB; g.M = M; g.N = N; g.rmax = RCORE_MAX; g.r_out = r; g.flags = c.flags;
  lu_gather_pieces_kernel<<<1, 256, 0, c.st>>>(g);
  LU_LAUNCH_CHECK();
  CoreJob J{};
  J.A = SA; J.B = SB; J.outA = target.A; J.outB = target.B;
  J.m = M; J.n = N; J.r = 0; J.lda = std::max(M, 1); J.ldb = std::max(N, 1);
  J.ldoa = (int32_t)target.lda; J.ldob = (int32_t)target.ldb; J.kcap = target.cap;
  J.zero_test = 1; J.rank = target.k; J.r_dev = r; J.pre_status = nullptr; J.zero_fill = 1;
  int s = launch_core_one(J, c.eps_trunc, c.flags, c.st);
  if (s != HM_OK) throw LuError(s, "recompression launch");
}

// target (low-rank) = compress(D) for a dense D (src/hlu.jl:159-190): fully
// pivoted ACA far below eps_trunc * s_1, then the exact SVD of its core
static void compress_dense_into(Ctx& c, Blk& target, View D) {
  Blk tmp;
  tmp.st = c.st;
  const int m = D.rows, n = D.cols;
  double* R = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)m * n);
  double* U = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)m * RCORE_MAX);
  double* V = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)n * RCORE_MAX);
  int32_t* rk = (int32_t*)dmalloc(c, tmp, sizeof(int32_t) * 2);
  axpby(c, View{R, 1, std::max(m, 1), m, n}, D, 1.0, 0.0);
  AcaFpJob J{};
  J.R = R; J.U = U; J.V = V; J.m = m; J.n = n; J.cap = RCORE_MAX; J.min_rank = 1; J.eps = 0.0;
  J.rank = rk; J.status = rk + 1; J.rel_mode = 1; J.eps_trunc = c.eps_trunc;
  int s = launch_aca_fp_one(J, c.st);
  if (s != HM_OK) throw LuError(s, "compress launch");
  CoreJob K{};
  K.A = U; K.B = V; K.outA = target.A; K.outB = target.B; K.m = m; K.n = n; K.r = 0;
  K.lda = std::max(m, 1); K.ldb = std::max(n, 1); K.ldoa = (int32_t)target.lda; K.ldob = (int32_t)target.ldb;
  K.kcap = target.cap; K.zero_test = 0; K.rank = target.k; K.r_dev = rk; K.pre_status = rk + 1; K.zero_fill = 1;
  s = launch_core_one(K, c.eps_trunc, c.flags, c.st);
  if (s != HM_OK) throw LuError(s, "compress core launch");
}

// ---- H-matrix products with dense blocks ----------------------------------
// Y += s H X   (hmat_matvec! with a matrix, src/harithm.jl:340-354)
static void hmm(Ctx& c, View Y, double s, const Blk& H, View X) {
  if (H.type == T_DENSE) {
    gemm(c, Y, H.Cv(), X, s, 1.0);
  } else if (H.type == T_RK) {
    Blk tmp;
    tmp.st = c.st;
    double* T = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)H.cap * X.cols);
    View Tv{T, 1, H.cap, H.cap, X.cols};
    gemm(c, Tv, vtr(H.Bv()), X, 1.0, 0.0);
    gemm(c, Y, H.Av(), Tv, s, 1.0);
  } else {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    hmm(c, vsub(Y, 0, 0, m, Y.cols), s, *H.ch[0], vsub(X, 0, 0, n, X.cols));
    hmm(c, vsub(Y, 0, 0, m, Y.cols), s, *H.ch[1], vsub(X, n, 0, H.n - n, X.cols));
    hmm(c, vsub(Y, m, 0, H.m - m, Y.cols), s, *H.ch[2], vsub(X, 0, 0, n, X.cols));
    hmm(c, vsub(Y, m, 0, H.m - m, Y.cols), s, *H.ch[3], vsub(X, n, 0, H.n - n, X.cols));
  }
}

// Y += s H' X   (transpose_hmat_mat_mul, src/harithm.jl:243-260)
static void hmm_t(Ctx& c, View Y, double s, const Blk& H, View X) {
  if (H.type == T_DENSE) {
    gemm(c, Y, vtr(H.Cv()), X, s, 1.0);
  } else if (H.type == T_RK) {
    Blk tmp;
    tmp.st = c.st;
    double* T = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)H.cap * X.cols);
    View Tv{T, 1, H.cap, H.cap, X.cols};
    gemm(c, Tv, vtr(H.Av()), X, 1.0, 0.0);
    gemm(c, Y, H.Bv(), Tv, s, 1.0);
  } else {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    hmm_t(c, vsub(Y, 0, 0, n, Y.cols), s, *H.ch[0], vsub(X, 0, 0, m, X.cols));
    hmm_t(c, vsub(Y, 0, 0, n, Y.cols), s, *H.ch[2], vsub(X, m, 0, H.m - m, X.cols));
    hmm_t(c, vsub(Y, n, 0, H.n - n, Y.cols), s, *H.ch[1], vsub(X, 0, 0, m, X.cols));
    hmm_t(c, vsub(Y, n, 0, H.n - n, Y.cols), s, *H.ch[3], vsub(X, m, 0, H.m - m, X.cols));
  }
}

// Y += s X H   (v*H of src/harithm.jl:331-371 for a matrix v)
static void xh(Ctx& c, View Y, double s, View X, const Blk& H) {
  hmm_t(c, vtr(Y), s, H, vtr(X));
}

// dense copy of H (to_fmat, src/utils.jl:162-192)
static void densify_into(Ctx& c, View D, const Blk& H) {
  if (H.type == T_DENSE) {
    axpby(c, D, H.Cv(), 1.0, 0.0);
  } else if (H.type == T_RK) {
    gemm(c, D, H.Av(), vtr(H.Bv()), 1.0, 0.0);
  } else {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    densify_into(c, vsub(D, 0, 0, m, n), *H.ch[0]);
    densify_into(c, vsub(D, 0, n, m, H.n - n), *H.ch[1]);
    densify_into(c, vsub(D, m, 0, H.m - m, n), *H.ch[2]);
    densify_into(c, vsub(D, m, n, H.m - m, H.n - n), *H.ch[3]);
  }
}

static BP dense_of(Ctx& c, const Blk& H) {
  BP d = new_dense(c, H.m, H.n, H.s, H.t);
  densify_into(c, d->Cv(), H);
  return d;
}

static BP copy_blk(Ctx& c, const Blk& a) {
  if (a.type == T_DENSE) {
    BP d = new_dense(c, a.m, a.n, a.s, a.t);
    d->row0 = a.row0;
    axpby(c, d->Cv(), a.Cv(), 1.0, 0.0);
    return d;
  }
  if (a.type == T_RK) {
    BP r = new_rk(c, a.m, a.n, a.s, a.t);
    r->row0 = a.row0;
    axpby(c, r->Av(), a.Av(), 1.0, 0.0);
    axpby(c, r->Bv(), a.Bv(), 1.0, 0.0);
    copy_int(c, r->k, a.k);
    return r;
  }
  BP h = std::make_shared<Blk>();
  h->st = c.st;
  h->type = T_H; h->m = a.m; h->n = a.n; h->s = a.s; h->t = a.t; h->row0 = a.row0;
  for (int q = 0; q < 4; ++q) h->ch[q] = copy_blk(c, *a.ch[q]);
  return h;
}

// ---- H-add (src/harithm.jl:4-151, 374-420) ---------------------------------
static void hmat_full_add(Ctx& c, Blk& a, View D, double s);
static void hmat_add(Ctx& c, Blk& a, const Blk& b, double s);

static void hmat_full_add(Ctx& c, Blk& a, View D, double s) {
  if (a.type == T_DENSE) {
    axpby(c, a.Cv(), D, s, 1.0);
  } else if (a.type == T_RK) {
    // C = A B' + s b; a.A, a.B = compress(C)   (src/harithm.jl:12-15)
    Blk tmp;
    tmp.st = c.st;
    double* T = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)a.m * a.n);
    View Tv{T, 1, std::max(a.m, 1), a.m, a.n};
    axpby(c, Tv, D, s, 0.0);
    gemm(c, Tv, a.Av(), vtr(a.Bv()), 1.0, 1.0);
    compress_dense_into(c, a, Tv);
  } else {
    const int m = a.ch[0]->m, n = a.ch[0]->n;
    hmat_full_add(c, *a.ch[0], vsub(D, 0, 0, m, n), s);
    hmat_full_add(c, *a.ch[1], vsub(D, 0, n, m, a.n - n), s);
    hmat_full_add(c, *a.ch[2], vsub(D, m, 0, a.m - m, n), s);
    hmat_full_add(c, *a.ch[3], vsub(D, m, n, a.m - m, a.n - n), s);
  }
}

// A B' + s H as a new low-rank block (src/harithm.jl:58-91)
static BP rkmat_hmat_add(Ctx& c, View A, View B, const int32_t* k, double s, const Blk& H) {
  BP out = new_rk(c, A.rows, B.rows, H.s, H.t);
  if (H.type == T_DENSE) {
    Blk tmp;
    tmp.st = c.st;
    double* T = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)H.m * H.n);
    View Tv{T, 1, std::max(H.m, 1), H.m, H.n};
    axpby(c, Tv, H.Cv(), s, 0.0);
    gemm(c, Tv, A, vtr(B), 1.0, 1.0);
    compress_dense_into(c, *out, Tv);
  } else if (H.type == T_RK) {
    std::vector<Piece> pcs = {
        Piece{A.p, A.cs, B.p, B.cs, k, A.rows, B.rows, 0, 0, 1.0},
        Piece{H.A, H.lda, H.B, H.ldb, H.k, H.m, H.n, 0, 0, s}};
    recompress(c, *out, pcs);
  } else {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    BP r11 = rkmat_hmat_add(c, vsub(A, 0, 0, m, A.cols), vsub(B, 0, 0, n, B.cols), k, s, *H.ch[0]);
    BP r12 = rkmat_hmat_add(c, vsub(A, 0, 0, m, A.cols), vsub(B, n, 0, H.n - n, B.cols), k, s, *H.ch[1]);
    BP r21 = rkmat_hmat_add(c, vsub(A, m, 0, H.m - m, A.cols), vsub(B, 0, 0, n, B.cols), k, s, *H.ch[2]);
    BP r22 = rkmat_hmat_add(c, vsub(A, m, 0, H.m - m, A.cols), vsub(B, n, 0, H.n - n, B.cols), k, s, *H.ch[3]);
    // A0 = [A11 A12 0 0; 0 0 A21 A22], B0 = [B11 0 B21 0; 0 B12 0 B22]  (src/harithm.jl:82-86)
    std::vector<Piece> pcs = {
        Piece{r11->A, r11->lda, r11->B, r11->ldb, r11->k, m, n, 0, 0, 1.0},
        Piece{r12->A, r12->lda, r12->B, r12->ldb, r12->k, m, H.n - n, 0, n, 1.0},
        Piece{r21->A, r21->lda, r21->B, r21->ldb, r21->k, H.m - m, n, m, 0, 1.0},
        Piece{r22->A, r22->lda, r22->B, r22->ldb, r22->k, H.m - m, H.n - n, m, n, 1.0}};
    recompress(c, *out, pcs);
  }
  return out;
}

static void hmat_add(Ctx& c, Blk& a, const Blk& b, double s) {
  if (b.type == T_DENSE) {
    hmat_full_add(c, a, b.Cv(), s);
  } else if (a.type == T_DENSE && b.type == T_RK) {
    gemm(c, a.Cv(), b.Av(), vtr(b.Bv()), s, 1.0);
  } else if (a.type == T_DENSE && b.type == T_H) {
    // a.C += s * (a.C + dense(b))  as written in src/harithm.jl:112; not
    // reached from lu! (a dense target has a leaf cluster, so b is never H)
    BP d = dense_of(c, b);
    axpby(c, d->Cv(), a.Cv(), 1.0, 1.0);
    axpby(c, a.Cv(), d->Cv(), s, 1.0);
  } else if (a.type == T_RK && b.type == T_RK) {
    std::vector<Piece> pcs = {
        Piece{a.A, a.lda, a.B, a.ldb, a.k, a.m, a.n, 0, 0, 1.0},
        Piece{b.A, b.lda, b.B, b.ldb, b.k, b.m, b.n, 0, 0, s}};
    recompress(c, a, pcs);
  } else if (a.type == T_RK && b.type == T_H) {
    BP r = rkmat_hmat_add(c, a.Av(), a.Bv(), a.k, s, b);
    axpby(c, a.Av(), r->Av(), 1.0, 0.0);
    axpby(c, a.Bv(), r->Bv(), 1.0, 0.0);
    copy_int(c, a.k, r->k);
  } else if (a.type == T_H && b.type == T_RK) {
    const int m = a.ch[0]->m, n = a.ch[0]->n;
    auto part = [&](int r0, int mr, int c0, int nc) {
      Blk v;
      v.st = c.st;
      v.type = T_RK; v.m = mr; v.n = nc; v.cap = b.cap; v.k = b.k;
      v.A = b.A + r0; v.lda = b.lda; v.B = b.B + c0; v.ldb = b.ldb;
      return v;
    };
    Blk c11 = part(0, m, 0, n), c21 = part(m, a.m - m, 0, n);
    Blk c12 = part(0, m, n, a.n - n), c22 = part(m, a.m - m, n, a.n - n);
    hmat_add(c, *a.ch[0], c11, s);
    hmat_add(c, *a.ch[2], c21, s);
    hmat_add(c, *a.ch[1], c12, s);
    hmat_add(c, *a.ch[3], c22, s);
  } else if (a.type == T_H && b.type == T_H) {
    for (int q = 0; q < 4; ++q) hmat_add(c, *a.ch[q], *b.ch[q], s);
  }
}

static BP hadd(Ctx& c, const Blk& a, const Blk& b) {
  BP r = copy_blk(c, a);
  hmat_add(c, *r, b, 1.0);
  return r;
}

// ---- H x H (src/harithm.jl:162-314) -----------------------------------------
static BP hmul(Ctx& c, const Blk& a, const Blk& b) {
  BP M;
  if (a.type == T_DENSE) {
    if (b.type == T_H && !is_leaf_cluster(c, a.s) && !is_leaf_cluster(c, a.t))
      throw LuError(HM_ERR_UNSUPPORTED, "full_mat_mul branch that has no method in the reference");
    if (b.type == T_H) {
      BP db = dense_of(c, b);
      M = new_dense(c, a.m, b.n, a.s, b.t);
      gemm(c, M->Cv(), a.Cv(), db->Cv(), 1.0, 0.0);
    } else if (b.type == T_DENSE) {
      M = new_dense(c, a.m, b.n, a.s, b.t);
      gemm(c, M->Cv(), a.Cv(), b.Cv(), 1.0, 0.0);
    } else {
      M = new_rk(c, a.m, b.n, a.s, b.t, true, false);
      M->B = b.B; M->ldb = b.ldb;
      gemm(c, M->Av(), a.Cv(), b.Av(), 1.0, 0.0);
      copy_int(c, M->k, b.k);
    }
  } else if (b.type == T_DENSE) {
    if (a.type == T_H && !is_leaf_cluster(c, b.s) && !is_leaf_cluster(c, b.t))
      throw LuError(HM_ERR_UNSUPPORTED, "mat_full_mul branch that has no method in the reference");
    if (a.type == T_H) {
      M = new_dense(c, a.m, b.n, a.s, b.t);
      axpby(c, M->Cv(), View{nullptr, 0, 0, a.m, b.n}, 0.0, 0.0);
      hmm(c, M->Cv(), 1.0, a, b.Cv());
    } else {
      M = new_rk(c, a.m, b.n, a.s, b.t, false, true);
      M->A = a.A; M->lda = a.lda;
      gemm(c, M->Bv(), vtr(b.Cv()), a.Bv(), 1.0, 0.0);
      copy_int(c, M->k, a.k);
    }
  } else if (a.type == T_RK && b.type == T_RK) {
    M = new_rk(c, a.m, b.n, a.s, b.t, false, true);
    M->A = a.A; M->lda = a.lda;
    Blk tmp;
    tmp.st = c.st;
    double* W = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)b.cap * a.cap);
    View Wv{W, 1, b.cap, b.cap, a.cap};
    gemm(c, Wv, vtr(b.Av()), a.Bv(), 1.0, 0.0);
    gemm(c, M->Bv(), b.Bv(), Wv, 1.0, 0.0);
    copy_int(c, M->k, a.k);
  } else if (a.type == T_RK && b.type == T_H) {
    M = new_rk(c, a.m, b.n, a.s, b.t, false, true);
    M->A = a.A; M->lda = a.lda;
    axpby(c, M->Bv(), View{nullptr, 0, 0, b.n, M->cap}, 0.0, 0.0);
    hmm_t(c, M->Bv(), 1.0, b, a.Bv());
    copy_int(c, M->k, a.k);
  } else if (a.type == T_H && b.type == T_RK) {
    M = new_rk(c, a.m, b.n, a.s, b.t, true, false);
    M->B = b.B; M->ldb = b.ldb;
    axpby(c, M->Av(), View{nullptr, 0, 0, a.m, M->cap}, 0.0, 0.0);
    hmm(c, M->Av(), 1.0, a, b.Av());
    copy_int(c, M->k, b.k);
  } else {
    M = std::make_shared<Blk>();
    M->st = c.st;
    M->type = T_H; M->m = a.m; M->n = b.n; M->s = a.s; M->t = b.t;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        BP H1 = hmul(c, *a.ch[2 * i + 0], *b.ch[0 + j]);
        BP H2 = hmul(c, *a.ch[2 * i + 1], *b.ch[2 + j]);
        M->ch[2 * i + j] = hadd(c, *H1, *H2);
      }
  }
  M->s = a.s;
  M->t = b.t;
  return M;
}

static void sub_mul(Ctx& c, Blk& cc, const Blk& a, const Blk& b) {
  BP M = hmul(c, a, b);
  hmat_add(c, cc, *M, -1.0);
}

// ---- triangular solves (src/hlu.jl:236-442) ----------------------------------
static void mfs(Ctx& c, const Blk& a, View X, bool unit, bool lower) {
  if (a.type == T_RK) throw LuError(HM_ERR_UNSUPPORTED, "A should not be a low-rank matrix");
  if (lower) {
    if (a.type == T_DENSE) {
      trsm_lower(c, a.Cv(), X, unit);
    } else {
      const int n = a.ch[0]->m;
      View X1 = vsub(X, 0, 0, n, X.cols), X2 = vsub(X, n, 0, X.rows - n, X.cols);
      mfs(c, *a.ch[0], X1, unit, true);
      hmm(c, X2, -1.0, *a.ch[2], X1);
      mfs(c, *a.ch[3], X2, unit, true);
    }
  } else {
    if (a.type == T_DENSE) {
      // X <- X U^{-1}  ==  X' <- U'^{-1} X'
      trsm_lower(c, vtr(a.Cv()), vtr(X), unit);
    } else {
      const int n = a.ch[0]->m;
      View X1 = vsub(X, 0, 0, X.rows, n), X2 = vsub(X, 0, n, X.rows, X.cols - n);
      mfs(c, *a.ch[0], X1, unit, false);
      xh(c, X2, -1.0, X1, *a.ch[1]);
      mfs(c, *a.ch[3], X2, unit, false);
    }
  }
}

static void trisolve(Ctx& c, const Blk& a, Blk& b, bool lower, bool unit) {
  if (a.type == T_RK) throw LuError(HM_ERR_UNSUPPORTED, "A should not be a low-rank matrix");
  if (lower) {
    if (a.type == T_DENSE && b.type == T_DENSE) trsm_lower(c, a.Cv(), b.Cv(), unit);
    else if (a.type == T_DENSE && b.type == T_RK) trsm_lower(c, a.Cv(), b.Av(), unit);
    else if (a.type == T_DENSE && b.type == T_H) throw LuError(HM_ERR_UNSUPPORTED, "This is never used");
    else if (a.type == T_H && b.type == T_H) {
      trisolve(c, *a.ch[0], *b.ch[0], lower, unit);
      trisolve(c, *a.ch[0], *b.ch[1], lower, unit);
      sub_mul(c, *b.ch[2], *a.ch[2], *b.ch[0]);
      sub_mul(c, *b.ch[3], *a.ch[2], *b.ch[1]);
      trisolve(c, *a.ch[3], *b.ch[2], lower, unit);
      trisolve(c, *a.ch[3], *b.ch[3], lower, unit);
    } else if (a.type == T_H && b.type == T_DENSE) mfs(c, a, b.Cv(), unit, true);
    else if (a.type == T_H && b.type == T_RK) mfs(c, a, b.Av(), unit, true);
  } else {
    if (a.type == T_DENSE && b.type == T_DENSE) trsm_lower(c, vtr(a.Cv()), vtr(b.Cv()), unit);
    else if (a.type == T_DENSE && b.type == T_RK) trsm_lower(c, vtr(a.Cv()), b.Bv(), unit);
    else if (a.type == T_H && b.type == T_DENSE) mfs(c, a, b.Cv(), unit, false);
    else if (a.type == T_H && b.type == T_RK) mfs(c, a, vtr(b.Bv()), unit, false);
    else if (a.type == T_H && b.type == T_H) {
      trisolve(c, *a.ch[0], *b.ch[0], lower, unit);
      trisolve(c, *a.ch[0], *b.ch[2], lower, unit);
      sub_mul(c, *b.ch[1], *b.ch[0], *a.ch[1]);
      sub_mul(c, *b.ch[3], *b.ch[2], *a.ch[1]);
      trisolve(c, *a.ch[3], *b.ch[1], lower, unit);
      trisolve(c, *a.ch[3], *b.ch[3], lower, unit);
    } else throw LuError(HM_ERR_UNSUPPORTED, "Invalid");
  }
}

// ---- LU (src/hlu.jl:446-515) --------------------------------------------------
static void permute(Ctx& c, Blk& H) {
  if (H.type == T_DENSE) laswp(c, H.Cv(), H.row0);
  else if (H.type == T_RK) laswp(c, H.Av(), H.row0);
  else
    for (int q = 0; q < 4; ++q) permute(c, *H.ch[q]);
}

static void lu_rec(Ctx& c, Blk& H) {
  if (H.type == T_RK) throw LuError(HM_ERR_UNSUPPORTED, "H should not be a low-rank matrix");
  if (H.type == T_DENSE) {
    getrf(c, H.Cv(), H.row0);
    return;
  }
  lu_rec(c, *H.ch[0]);
  permute(c, *H.ch[1]);
  trisolve(c, *H.ch[0], *H.ch[1], true, true);
  trisolve(c, *H.ch[0], *H.ch[2], false, false);
  sub_mul(c, *H.ch[3], *H.ch[2], *H.ch[1]);
  lu_rec(c, *H.ch[3]);
  permute(c, *H.ch[2]);
}

// ---- solve (src/hlu.jl:524-562) -----------------------------------------------
static void solve_rec(Ctx& c, const Blk& a, View y, bool lower) {
  if (a.type == T_RK) throw LuError(HM_ERR_UNSUPPORTED, "a cannot be a low-rank matrix");
  const int m = a.type == T_H ? a.ch[0]->m : a.m;
  if (lower) {
    if (a.type == T_DENSE) {
      trsm_lower(c, a.Cv(), y, true);
    } else {
      solve_rec(c, *a.ch[0], vsub(y, 0, 0, m, y.cols), true);
      hmm(c, vsub(y, m, 0, y.rows - m, y.cols), -1.0, *a.ch[2], vsub(y, 0, 0, m, y.cols));
      solve_rec(c, *a.ch[3], vsub(y, m, 0, y.rows - m, y.cols), true);
    }
  } else {
    if (a.type == T_DENSE) {
      trsm_lower(c, vrev(a.Cv()), vrev(y), false);       // U^{-1} y as a reversed lower solve
    } else {
      solve_rec(c, *a.ch[3], vsub(y, m, 0, y.rows - m, y.cols), false);
      hmm(c, vsub(y, 0, 0, m, y.cols), -1.0, *a.ch[1], vsub(y, m, 0, y.rows - m, y.cols));
      solve_rec(c, *a.ch[0], vsub(y, 0, 0, m, y.cols), false);
    }
  }
}

// transposed solve H' x = b with H[P,:] = L U: U' z = b (lower, non-unit),
// L' w = z (upper, unit), x[P] = w.  No counterpart in the reference (the
// adjoint of H\y); the same leaf kernels run on transposed/reversed views.
static void solve_t_rec(Ctx& c, const Blk& a, View y, bool upper_t) {
  if (a.type == T_RK) throw LuError(HM_ERR_UNSUPPORTED, "a cannot be a low-rank matrix");
  const int m = a.type == T_H ? a.ch[0]->m : a.m;
  if (upper_t) {                       // U' is lower triangular
    if (a.type == T_DENSE) {
      trsm_lower(c, vtr(a.Cv()), y, false);
    } else {
      solve_t_rec(c, *a.ch[0], vsub(y, 0, 0, m, y.cols), true);
      hmm_t(c, vsub(y, m, 0, y.rows - m, y.cols), -1.0, *a.ch[1], vsub(y, 0, 0, m, y.cols));
      solve_t_rec(c, *a.ch[3], vsub(y, m, 0, y.rows - m, y.cols), true);
    }
  } else {                             // L' is unit upper triangular
    if (a.type == T_DENSE) {
      trsm_lower(c, vrev(vtr(a.Cv())), vrev(y), true);
    } else {
      solve_t_rec(c, *a.ch[3], vsub(y, m, 0, y.rows - m, y.cols), false);
      hmm_t(c, vsub(y, 0, 0, m, y.cols), -1.0, *a.ch[2], vsub(y, m, 0, y.rows - m, y.cols));
      solve_t_rec(c, *a.ch[0], vsub(y, 0, 0, m, y.cols), false);
    }
  }
}

// x[P[i], c] = w[i, c]
__global__ void lu_scatter_rows_kernel(View Xv, View W, const int64_t* __restrict__ P) {
  const int64_t tot = (int64_t)W.rows * W.cols;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % W.rows), c = (int)(e / W.rows);
    Xv.p[P[i] * Xv.rs + (int64_t)c * Xv.cs] = W.p[(int64_t)i * W.rs + (int64_t)c * W.cs];
  }
}

// ---------------------------------------------------------------------------
// batched helpers
// ---------------------------------------------------------------------------
// Job arrays of a sequence that is later captured into a CUDA graph: the first
// (recording) run keeps every uploaded array alive in order; the capture run
// takes the same arrays back instead of uploading (a host-to-device copy of
// pageable memory cannot be captured).  The job contents are identical since
// the capture replays the recorded sequence on the same buffers.
struct JobTape {
  bool record = false, replay = false;
  std::vector<void*> bufs;
  std::vector<size_t> bytes;
  size_t pos = 0;
  size_t temp_bytes = 0;   // arena size that holds every temporary of the recorded run
  ~JobTape() {             // the owner has synchronised the device
    for (void* p : bufs) cudaFreeAsync(p, cudaStreamLegacy);
  }
};
static void tape_note_temporary(size_t bytes) {
  if (g_tape && g_tape->record) g_tape->temp_bytes += arena_round(bytes);
}

template <typename J>
static J* upload_jobs(Ctx& c, Blk& owner, const std::vector<J>& v) {
  if (g_tape && g_tape->replay) {
    if (g_tape->pos >= g_tape->bufs.size() || g_tape->bytes[g_tape->pos] != sizeof(J) * v.size())
      throw LuError(HM_ERR_CUDA, "job tape does not match the recorded sequence");
    return (J*)g_tape->bufs[g_tape->pos++];
  }
  J* d = nullptr;
  if (g_tape && g_tape->record) {
    if (cudaMallocAsync(&d, sizeof(J) * v.size(), c.st) != cudaSuccess) throw LuError(HM_ERR_OOM, "job tape");
    g_tape->bufs.push_back(d);
    g_tape->bytes.push_back(sizeof(J) * v.size());
  } else {
    d = (J*)dmalloc(c, owner, sizeof(J) * v.size());
  }
  if (cudaMemcpyAsync(d, v.data(), sizeof(J) * v.size(), cudaMemcpyHostToDevice, c.st) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "job upload");
  return d;
}

// copies of stored leaves into the FP64 working buffers of the factorisation,
// collected and launched as one kernel (one CTA per block)
struct LoadJob {
  const void* src;
  int64_t ld_src;
  int rows, cols;          // valid source columns; columns [cols, dst_cols) become zero
  int type;                // HM_F64 / HM_F32 / HM_BF16 element type of src
  double* dst;
  int64_t ld_dst;
  int dst_cols;
  int32_t* kdst;           // if set: *kdst = kval
  int kval;
};
__global__ void lu_load_batch_kernel(const LoadJob* __restrict__ jobs) {
  const LoadJob J = jobs[blockIdx.x];
  const int64_t tot = (int64_t)J.rows * J.dst_cols;
  for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
    const int i = (int)(e % J.rows), c = (int)(e / J.rows);
    double v = 0.0;
    if (c < J.cols) {
      const int64_t s = i + (int64_t)c * J.ld_src;
      if (J.type == HM_F64) v = ((const double*)J.src)[s];
      else if (J.type == HM_F32) v = (double)((const float*)J.src)[s];
      else v = (double)__bfloat162float(((const __nv_bfloat16*)J.src)[s]);
    }
    J.dst[i + (int64_t)c * J.ld_dst] = v;
  }
  if (threadIdx.x == 0 && J.kdst) *J.kdst = J.kval;
}

struct Loader {
  std::vector<LoadJob> jobs;
  void flush(Ctx& c) {
    for (size_t b = 0; b < jobs.size(); b += 65535) {
      const size_t nb = std::min<size_t>(65535, jobs.size() - b);
      Blk tmp;
      tmp.st = c.st;
      std::vector<LoadJob> part(jobs.begin() + b, jobs.begin() + b + nb);
      LoadJob* d = upload_jobs(c, tmp, part);
      lu_load_batch_kernel<<<(unsigned)nb, 256, 0, c.st>>>(d);
      LU_LAUNCH_CHECK();
    }
    jobs.clear();
  }
};

static BP build_tree(Ctx& c, const hm_handle* h, int32_t node, Loader& ld);
static BP build_from_handle(Ctx& c, const hm_handle* h, int32_t node);

// independent products in one launch; big = true: 128 x 128 tiles
static void gemm_batch(Ctx& c, const std::vector<GemmJob>& jobs, bool big = false) {
  if (jobs.empty()) return;
  const int t = big ? GB_T : 32;
  int gx = 1, gy = 1;
  for (auto& j : jobs) {
    gx = std::max(gx, (j.C.cols + t - 1) / t);
    gy = std::max(gy, (j.C.rows + t - 1) / t);
  }
  for (size_t b = 0; b < jobs.size(); b += 65535) {
    const size_t nb = std::min<size_t>(65535, jobs.size() - b);
    Blk tmp;
    tmp.st = c.st;
    std::vector<GemmJob> part(jobs.begin() + b, jobs.begin() + b + nb);
    GemmJob* d = upload_jobs(c, tmp, part);
    if (big) lu_gemm_big_batch_kernel<<<dim3(gx, gy, (unsigned)nb), 256, 0, c.st>>>(d);
    else lu_gemm_batch_kernel<<<dim3(gx, gy, (unsigned)nb), 256, 0, c.st>>>(d);
    LU_LAUNCH_CHECK();
  }
}

// one low-rank target = truncated sum of its pieces
struct RcReq {
  Piece pc[2];
  int np;
  double* outA; int64_t ldoa;
  double* outB; int64_t ldob;
  int32_t* k;
  int m, n, kcap;
};

// size_to_batch: read the largest core size back and launch for it (one host
// synchronisation); otherwise launch for rmax.
static void recompress_batch(Ctx& c, const std::vector<RcReq>& reqs, int rmax, bool size_to_batch = true) {
  if (reqs.empty()) return;
  rmax = std::min(std::max(rmax, 1), RCORE_MAX);
  size_t b = 0;
  while (b < reqs.size()) {
    size_t e = b, elems = 0;
    while (e < reqs.size() && (e == b || elems + (size_t)(reqs[e].m + reqs[e].n) * rmax < (size_t)1 << 27)) {
      elems += (size_t)(reqs[e].m + reqs[e].n) * rmax;
      ++e;
    }
    Blk tmp;
    tmp.st = c.st;
    double* scratch = (double*)dmalloc(c, tmp, sizeof(double) * elems);
    int32_t* rr = (int32_t*)dmalloc(c, tmp, sizeof(int32_t) * (e - b));
    std::vector<GatherArgs> ga(e - b);
    std::vector<CoreJob> cj(e - b);
    size_t off = 0;
    for (size_t q = b; q < e; ++q) {
      const RcReq& R = reqs[q];
      GatherArgs& g = ga[q - b];
      g = GatherArgs{};
      for (int p = 0; p < R.np; ++p) g.pc[p] = R.pc[p];
      g.np = R.np;
      g.SA = scratch + off;
      g.SB = scratch + off + (size_t)R.m * rmax;
      g.M = R.m; g.N = R.n; g.rmax = rmax; g.r_out = rr + (q - b); g.flags = c.flags;
      CoreJob& J = cj[q - b];
      J = CoreJob{};
      J.A = g.SA; J.B = g.SB; J.outA = R.outA; J.outB = R.outB;
      J.m = R.m; J.n = R.n; J.lda = std::max(R.m, 1); J.ldb = std::max(R.n, 1);
      J.ldoa = (int32_t)R.ldoa; J.ldob = (int32_t)R.ldob; J.kcap = R.kcap;
      J.zero_test = 1; J.rank = R.k; J.r_dev = g.r_out; J.zero_fill = 1;
      off += (size_t)(R.m + R.n) * rmax;
    }
    GatherArgs* dg = upload_jobs(c, tmp, ga);
    CoreJob* dc = upload_jobs(c, tmp, cj);
    lu_gather_pieces_batch_kernel<<<(unsigned)(e - b), 256, 0, c.st>>>(dg);
    LU_LAUNCH_CHECK();
    // size the core launch to the largest core of this batch (ranks are on
    // the device: one small read-back per batch)
    int rlaunch = rmax;
    if (size_to_batch) {
      int32_t* dmax = (int32_t*)dmalloc(c, tmp, sizeof(int32_t));
      lu_max_int_kernel<<<1, 256, 0, c.st>>>(rr, (int)(e - b), dmax);
      LU_LAUNCH_CHECK();
      int32_t hmax = 0;
      if (cudaMemcpyAsync(&hmax, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, c.st) != cudaSuccess ||
          cudaStreamSynchronize(c.st) != cudaSuccess)
        throw LuError(HM_ERR_CUDA, "core size read-back");
      rlaunch = std::min(rmax, std::max(8, (hmax + 7) / 8 * 8));
    }
    int s = launch_core_recompress(dc, (int)(e - b), rlaunch, c.eps_trunc, c.flags, c.st, true);
    if (s != HM_OK) throw LuError(s, "batched recompression launch");
    b = e;
  }
}

// The off-diagonal part of step k's trailing update, generated on the device:
// for every pair i != j of trailing tiles, A_ij B_ij' - Q_ij B_kj' is gathered
// into one [A | -Q] [B | B_kj] pair and recompressed (Q_ij = A_ik W_kj, the
// panel product of step k).  Job q of the batch is pair (ii, jj) of the
// trailing tiles with the diagonal skipped; its scratch is a fixed stride.
// Pair q of the trailing update of step k: mode 0 every pair i != j of the
// tiles (k, T); mode 1 the pairs of tile row and tile column k+1; mode 2 the
// pairs among the tiles (k+1, T).
__device__ __forceinline__ void tile_pair(int T, int k, int mode, int64_t gq, int& i, int& j) {
  if (mode == 1) {
    const int n1 = T - k - 2;
    if (gq < n1) { i = k + 1; j = k + 2 + (int)gq; }
    else { i = k + 2 + (int)(gq - n1); j = k + 1; }
    return;
  }
  const int base = mode == 2 ? k + 2 : k + 1;
  const int Tr = T - base;
  const int ii = (int)(gq / (Tr - 1));
  int jj = (int)(gq % (Tr - 1));
  if (jj >= ii) ++jj;
  i = base + ii;
  j = base + jj;
}
static int64_t tile_pair_count(int T, int k, int mode) {
  const int64_t Tr = T - k - 1;
  if (mode == 0) return Tr * (Tr - 1);
  if (mode == 1) return Tr >= 2 ? 2 * (Tr - 1) : 0;
  return Tr >= 2 ? (Tr - 1) * (Tr - 2) : 0;
}

// truncation tolerance from which the tile recompressions run in FP32
constexpr double MIXED_CORE_EPS = 1e-6;

struct TileJobArgs {
  const double* const* Ap;
  const double* const* Bp;
  const int64_t* start;
  const int32_t* size;
  int32_t* kmat;
  int T, cap, k, rmax;
  int64_t R;                 // (T-k-1) cap: columns of a Q panel row
  const double* qbase;       // Q_i = qbase + (start[i] - start[k+1]) R
  double* scratch;
  int64_t stride;            // scratch doubles per job
  int32_t* rr;               // gathered rank per job
  int* flags;
  CoreJob* cj;
  int64_t q0;                // first job of this batch
  int mode;                  // which pairs (tile_pair)
};
__global__ void __launch_bounds__(256) lu_tile_gather_kernel(TileJobArgs a) {
  const int64_t q = blockIdx.x;
  const int64_t gq = a.q0 + q;
  int i, j;
  tile_pair(a.T, a.k, a.mode, gq, i, j);
  const int mi = a.size[i], nj = a.size[j];
  const double* Qi = a.qbase + (a.start[i] - a.start[a.k + 1]) * a.R;
  double* Aij = const_cast<double*>(a.Ap[i]) + (int64_t)j * a.cap * mi;
  double* Bij = const_cast<double*>(a.Bp[j]) + (int64_t)i * a.cap * nj;
  GatherArgs g{};
  g.pc[0] = Piece{Aij, mi, Bij, nj, a.kmat + i * a.T + j, mi, nj, 0, 0, 1.0};
  g.pc[1] = Piece{Qi + (int64_t)(j - a.k - 1) * a.cap * mi, mi, a.Bp[j] + (int64_t)a.k * a.cap * nj, nj,
                  a.kmat + a.k * a.T + j, mi, nj, 0, 0, -1.0};
  g.np = 2;
  g.SA = a.scratch + q * a.stride;
  g.SB = g.SA + (int64_t)mi * a.rmax;
  g.M = mi; g.N = nj; g.rmax = a.rmax;
  g.r_out = a.rr + q;
  g.flags = a.flags;
  if (threadIdx.x == 0) {
    CoreJob J{};
    J.A = g.SA; J.B = g.SB; J.outA = Aij; J.outB = Bij;
    J.m = mi; J.n = nj; J.lda = max(mi, 1); J.ldb = max(nj, 1);
    J.ldoa = mi; J.ldob = nj; J.kcap = a.cap;
    J.zero_test = 1; J.rank = a.kmat + i * a.T + j; J.r_dev = g.r_out; J.zero_fill = 1;
    a.cj[q] = J;
  }
  gather_pieces(g);
}

// H_tile += s * A B' for an H-structured diagonal tile, as jobs: dense leaves
// get a product, low-rank leaves a recompression (hmat_add! of H += Rk splits
// the low-rank term over the children, src/harithm.jl:129-142)
static void tile_add_lowrank(const Blk& H, int r0, int c0, const double* A, int64_t lda, const double* B,
                             int64_t ldb, const int32_t* k, int cap, double s, std::vector<GemmJob>& gj,
                             std::vector<RcReq>& rj) {
  if (H.type == T_DENSE) {
    GemmJob g{};
    g.A = View{const_cast<double*>(A) + r0, 1, lda, H.m, cap};
    g.B = vtr(View{const_cast<double*>(B) + c0, 1, ldb, H.n, cap});
    g.C = H.Cv();
    g.alpha = s;
    g.beta = 1.0;
    gj.push_back(g);
  } else if (H.type == T_RK) {
    RcReq R{};
    R.pc[0] = Piece{H.A, H.lda, H.B, H.ldb, H.k, H.m, H.n, 0, 0, 1.0};
    R.pc[1] = Piece{A + r0, lda, B + c0, ldb, k, H.m, H.n, 0, 0, s};
    R.np = 2;
    R.outA = H.A; R.ldoa = H.lda; R.outB = H.B; R.ldob = H.ldb; R.k = H.k;
    R.m = H.m; R.n = H.n; R.kcap = H.cap;
    rj.push_back(R);
  } else {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    tile_add_lowrank(*H.ch[0], r0, c0, A, lda, B, ldb, k, cap, s, gj, rj);
    tile_add_lowrank(*H.ch[1], r0, c0 + n, A, lda, B, ldb, k, cap, s, gj, rj);
    tile_add_lowrank(*H.ch[2], r0 + m, c0, A, lda, B, ldb, k, cap, s, gj, rj);
    tile_add_lowrank(*H.ch[3], r0 + m, c0 + n, A, lda, B, ldb, k, cap, s, gj, rj);
  }
}

// ---------------------------------------------------------------------------
// tile LU.  When every leaf outside the diagonal tiles (row group x column
// group blocks) is one low-rank block covering its whole tile -- the
// partition of the aca2 route with the identity adjacency -- the recursion of
// lu! is carried out tile by tile (right-looking), which performs the same
// operations with leaf-local pivoting but batches them: per step k the
// diagonal tile is factorised by the recursion above, the whole row panel
// (A factors of tiles (k, j>k)) and column panel (B factors of tiles (i>k, k))
// are solved as one wide triangular solve each, every core B_ik' A_kj comes
// out of one GEMM, and all updates of the trailing tiles run as one batched
// product + one batched recompression.  Updates are truncated per step (the
// recursion sums some products before truncating); both stay within
// eps_trunc of the exact Schur complement.
// ---------------------------------------------------------------------------
struct TileLU {
  int T = 0;
  std::vector<int64_t> start, size;      // tile ranges
  std::vector<BP> diag;                  // diagonal tiles (H or dense)
  std::vector<double*> Ap, Bp;           // row panels (m_i x T*cap), column panels (n_j x T*cap)
  int32_t* kmat = nullptr;               // ranks of the off-diagonal tiles, T x T
  BP hold;                               // owns the panel memory
  double* Ai(int i, int j, int cap) const { return Ap[i] + (int64_t)j * cap * size[i]; }
  double* Bj(int i, int j, int cap) const { return Bp[j] + (int64_t)i * cap * size[j]; }
  // for the sweep solve (built on the first solve): the inverses of the
  // diagonal tiles' unit-lower L and upper U, each stored column-major and
  // row-major, and device tables of the panels
  BP sweep_hold;
  const double** d_Ap = nullptr;
  const double** d_Bp = nullptr;
  const double** d_inv[4] = {nullptr, nullptr, nullptr, nullptr};   // see sweep_finish
  int64_t* d_start = nullptr;
  int32_t* d_size = nullptr;
};

// tile structure of the handle, or false when the partition has no such level
// A tiling of [0, n) by clusters gcl (sorted by start) can run the tile
// schedule when every leaf off the tile diagonal is a low-rank leaf whose rows
// and columns are unions of whole tiles (a leaf spanning several tiles is
// loaded as its tile parts, which keep its rank) and every diagonal tile is a
// node of the block tree (leaves inside it stay in its recursive tree).
static bool tile_check(const hm_handle* h, const std::vector<int32_t>& gcl, std::vector<int32_t>& diag_node) {
  const int T = (int)gcl.size();
  if (T < 2) return false;
  if (h->cl_s[gcl[0]] != 0 || h->cl_e[gcl[T - 1]] != h->n) return false;
  for (int i = 1; i < T; ++i)
    if (h->cl_s[gcl[i]] != h->cl_e[gcl[i - 1]]) return false;
  std::vector<int64_t> st(T);
  for (int i = 0; i < T; ++i) st[i] = h->cl_s[gcl[i]];
  auto tile_of = [&](int64_t r) { return (int)(std::upper_bound(st.begin(), st.end(), r) - st.begin()) - 1; };
  auto aligned = [&](int64_t a, int64_t len, int t0, int t1) { return a == st[t0] && a + len == h->cl_e[gcl[t1]]; };
  for (auto& L : h->leaves) {
    const int i0 = tile_of(L.row0), i1 = tile_of(L.row0 + L.m - 1);
    const int j0 = tile_of(L.col0), j1 = tile_of(L.col0 + L.n - 1);
    if (i0 == i1 && j0 == j1 && i0 == j0) continue;            // inside a diagonal tile
    const bool overlap = !(i1 < j0 || j1 < i0);                 // would cover part of a diagonal tile
    if (overlap || L.type != T_RK || !aligned(L.row0, L.m, i0, i1) || !aligned(L.col0, L.n, j0, j1))
      return false;
  }
  const int64_t ncl = (int64_t)h->cl_s.size();
  diag_node.assign(T, -1);
  std::vector<int32_t> tile_of_cluster(ncl, -1);
  for (int i = 0; i < T; ++i) tile_of_cluster[gcl[i]] = i;
  for (int32_t id = 0; id < (int32_t)h->nodes.size(); ++id) {
    const Node& nd = h->nodes[id];
    if (nd.s == nd.t && tile_of_cluster[nd.s] >= 0) diag_node[tile_of_cluster[nd.s]] = id;
  }
  for (int i = 0; i < T; ++i)
    if (diag_node[i] < 0) return false;
  return true;
}

// The tile level.  First candidate: the highest clusters that are the row
// cluster of some leaf (for a balanced partition, the clusters of the first
// admissible level; for a KMeans tree the tiles may sit at several depths).
// Otherwise the shallowest depth whose clusters form a valid tiling (a median
// bisection of an n that is not a power of two mixes cluster sizes on both
// sides of MaxBlock on one level, so the admissible blocks start one level
// lower on part of it).
static bool tile_structure(const hm_handle* h, std::vector<int32_t>& gcl, std::vector<int32_t>& diag_node) {
  const int64_t ncl = (int64_t)h->cl_s.size();
  auto by_start = [&](int32_t a, int32_t b) { return h->cl_s[a] < h->cl_s[b]; };
  {
    std::vector<char> is_row(ncl, 0), covered(ncl, 0);
    for (auto& L : h->leaves) is_row[L.s] = 1;
    gcl.clear();
    for (int64_t c = 0; c < ncl; ++c) {
      if (!covered[c] && is_row[c]) gcl.push_back((int32_t)c);
      if (h->cl_left[c] >= 0) {
        const char cv = covered[c] || is_row[c];
        covered[h->cl_left[c]] = cv;
        covered[h->cl_right[c]] = cv;
      }
    }
    std::sort(gcl.begin(), gcl.end(), by_start);
    if (tile_check(h, gcl, diag_node)) return true;
  }
  int maxd = 0;
  for (int64_t c = 0; c < ncl; ++c) maxd = std::max(maxd, (int)h->cl_depth[c]);
  for (int d = 1; d <= maxd; ++d) {
    gcl.clear();
    int64_t cover = 0;
    for (int64_t c = 0; c < ncl; ++c)
      if (h->cl_depth[c] == d) {
        gcl.push_back((int32_t)c);
        cover += h->cl_e[c] - h->cl_s[c];
      }
    if (cover != h->n) return false;            // a cluster leaf above depth d: no deeper level covers
    std::sort(gcl.begin(), gcl.end(), by_start);
    if (tile_check(h, gcl, diag_node)) return true;
  }
  return false;
}

// The same update with the gather fused into the recompression: the CTA
// loads [A_ij | -Q_ij] and [B_ij | B_kj] into shared memory (rl columns at
// most, smax rows) and runs the QR + SVD core there.
// TS: the precision of the staged factors and of the QR + SVD core (FP32 when
// the truncation tolerance is loose: the mixed-precision factorisation)
template <typename TS>
__global__ void __launch_bounds__(128) lu_tile_core_kernel(TileJobArgs a, int rl, int smax, double eps_trunc) {
  extern __shared__ double sm_raw[];
  TS* sm = reinterpret_cast<TS*>(sm_raw);
  const int64_t gq = a.q0 + blockIdx.x;
  int i, j;
  tile_pair(a.T, a.k, a.mode, gq, i, j);
  const int mi = a.size[i], nj = a.size[j];
  const double* Qij = a.qbase + (a.start[i] - a.start[a.k + 1]) * a.R + (int64_t)(j - a.k - 1) * a.cap * mi;
  double* Aij = const_cast<double*>(a.Ap[i]) + (int64_t)j * a.cap * mi;
  double* Bij = const_cast<double*>(a.Bp[j]) + (int64_t)i * a.cap * nj;
  const double* Bkj = a.Bp[j] + (int64_t)a.k * a.cap * nj;
  int32_t* kij = a.kmat + i * a.T + j;
  const int k1 = *kij, k2 = a.kmat[a.k * a.T + j];
  int r = k1 + k2;
  if (r > rl) {                      // cannot happen: rl bounds every pair of the step
    if (threadIdx.x == 0) atomicOr(a.flags, 1);
    r = rl;
  }
  TS* XA = sm + 3 * rl * rl;
  TS* XB = XA + (int64_t)smax * rl;
  for (int q = 0; q < r; ++q)
    for (int t = threadIdx.x; t < mi; t += blockDim.x)
      XA[t + q * mi] = (TS)(q < k1 ? Aij[t + (int64_t)q * mi] : -Qij[t + (int64_t)(q - k1) * mi]);
  for (int q = 0; q < r; ++q)
    for (int t = threadIdx.x; t < nj; t += blockDim.x)
      XB[t + q * nj] = (TS)(q < k1 ? Bij[t + (int64_t)q * nj] : Bkj[t + (int64_t)(q - k1) * nj]);
  __syncthreads();
  CoreJob J{};
  J.outA = Aij; J.outB = Bij;
  J.m = mi; J.n = nj; J.r = r; J.lda = max(mi, 1); J.ldb = max(nj, 1);
  J.ldoa = mi; J.ldob = nj; J.kcap = a.cap;
  J.zero_test = 1; J.rank = kij; J.zero_fill = 1;
  // the tile's columns at and beyond its previous rank k1 are zero: only the
  // columns [k, k1) a smaller new rank frees need zeros
  J.known_zero = 1; J.zero_from = k1;
  // from step 1 on, every trailing tile (and tile (k, j)) is a previous step's
  // core output: A_ij orthonormal, B_ij and B_kj with orthogonal columns
  J.ortho_k = a.k >= 1 ? k1 : 0;
  core_body_t<TS, true>(J, XA, XB, rl, eps_trunc, a.flags);
}

// an upper bound of rank(A_ij) + rank(B_kj) over the trailing pairs of step k
__global__ void lu_tile_rank_bound_kernel(const int32_t* __restrict__ kmat, int T, int k, int32_t* out) {
  __shared__ int32_t red[256];
  int32_t m1 = 0, m2 = 0;
  const int Tr = T - k - 1;
  for (int e = threadIdx.x; e < Tr * Tr; e += blockDim.x) {
    const int i = k + 1 + e / Tr, j = k + 1 + e % Tr;
    if (i != j) m1 = max(m1, kmat[i * T + j]);
  }
  for (int j = k + 1 + threadIdx.x; j < T; j += blockDim.x) m2 = max(m2, kmat[k * T + j]);
  red[threadIdx.x] = m1;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const int32_t a1 = red[0];
  __syncthreads();
  red[threadIdx.x] = m2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = a1 + red[0];
}

// the launch size of step k's recompression cores: a bound of rank(A_ij) +
// rank(B_kj) over its pairs, read back once per step
static int tile_rank_bound(Ctx& c, const TileLU& TL, int k, int rmax) {
  Blk tmp;
  tmp.st = c.st;
  int32_t* dmax = (int32_t*)dmalloc(c, tmp, sizeof(int32_t));
  lu_tile_rank_bound_kernel<<<1, 256, 0, c.st>>>(TL.kmat, TL.T, k, dmax);
  LU_LAUNCH_CHECK();
  int32_t hb = 0;
  if (cudaMemcpyAsync(&hb, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, c.st) != cudaSuccess ||
      cudaStreamSynchronize(c.st) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "rank bound read-back");
  return std::min(std::min(std::max(rmax, 1), RCORE_MAX), std::max(8, (hb + 7) / 8 * 8));
}

static void recompress_tile_pairs(Ctx& c, const TileLU& TL, int k, int64_t R, const double* qbase, int rmax,
                                  int mode, int rl) {
  const int T = TL.T;
  const int64_t njobs = tile_pair_count(T, k, mode);
  if (njobs <= 0) return;
  rmax = std::min(std::max(rmax, 1), RCORE_MAX);
  int64_t smax = 1;
  for (int i = k + 1; i < T; ++i) smax = std::max<int64_t>(smax, TL.size[i]);
  Blk tmp;
  tmp.st = c.st;
  {
    // fused path: the pairs' factors staged in shared memory, in FP32 when the
    // truncation tolerance is loose (>= 1e-6, the mixed-precision scheme)
    const bool f32 = c.eps_trunc >= MIXED_CORE_EPS;
    const size_t smem = (f32 ? sizeof(float) : sizeof(double)) * ((size_t)3 * rl * rl + (size_t)2 * smax * rl);
    if (smem <= 200 * 1024) {
      const void* kfn = f32 ? (const void*)lu_tile_core_kernel<float> : (const void*)lu_tile_core_kernel<double>;
      if (smem_attr(kfn, 200 * 1024) != cudaSuccess) throw LuError(HM_ERR_CUDA, "tile core smem");
      for (int64_t q0 = 0; q0 < njobs; q0 += INT32_MAX) {
        const int64_t nb = std::min<int64_t>(INT32_MAX, njobs - q0);
        TileJobArgs a{TL.d_Ap, TL.d_Bp, TL.d_start, TL.d_size, TL.kmat, T, c.cap, k, rmax, R, qbase, nullptr, 0,
                      nullptr, c.flags, nullptr, q0, mode};
        if (f32) lu_tile_core_kernel<float><<<(unsigned)nb, 128, smem, c.st>>>(a, rl, (int)smax, c.eps_trunc);
        else lu_tile_core_kernel<double><<<(unsigned)nb, 128, smem, c.st>>>(a, rl, (int)smax, c.eps_trunc);
        LU_LAUNCH_CHECK();
      }
      return;
    }
  }
  const int64_t stride = 2 * smax * rmax;
  const int64_t per = std::max<int64_t>(1, std::min<int64_t>(((int64_t)1 << 28) / stride, 65535));
  const int64_t nb0 = std::min(per, njobs);
  double* scratch = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)(nb0 * stride));
  int32_t* rr = (int32_t*)dmalloc(c, tmp, sizeof(int32_t) * (size_t)nb0);
  CoreJob* cj = (CoreJob*)dmalloc(c, tmp, sizeof(CoreJob) * (size_t)nb0);
  int32_t* dmax = (int32_t*)dmalloc(c, tmp, sizeof(int32_t));
  for (int64_t q0 = 0; q0 < njobs; q0 += per) {
    const int64_t nb = std::min(per, njobs - q0);
    TileJobArgs a{TL.d_Ap, TL.d_Bp, TL.d_start, TL.d_size, TL.kmat, T, c.cap, k, rmax, R, qbase, scratch, stride,
                  rr, c.flags, cj, q0, mode};
    lu_tile_gather_kernel<<<(unsigned)nb, 256, 0, c.st>>>(a);
    LU_LAUNCH_CHECK();
    lu_max_int_kernel<<<1, 256, 0, c.st>>>(rr, (int)nb, dmax);
    LU_LAUNCH_CHECK();
    int32_t hmax = 0;
    if (cudaMemcpyAsync(&hmax, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, c.st) != cudaSuccess ||
        cudaStreamSynchronize(c.st) != cudaSuccess)
      throw LuError(HM_ERR_CUDA, "core size read-back");
    const int rlaunch = std::min(rmax, std::max(8, (hmax + 7) / 8 * 8));
    int st = launch_core_recompress(cj, (int)nb, rlaunch, c.eps_trunc, c.flags, c.st, true);
    if (st != HM_OK) throw LuError(st, "batched recompression launch");
  }
}

// Step k's products for the trailing update, kept until the update has run:
// W = B_ik' A_kj for the whole panels and Q_i = A_ik W for every trailing tile
// row (freed on the main stream).
struct StepQ {
  std::shared_ptr<Blk> hold;
  double* qbase = nullptr;
  std::vector<double*> Q;
};

static void tile_factor(Ctx& c, const hm_handle* h, TileLU& TL, const std::vector<int32_t>& gcl,
                        const std::vector<int32_t>& dnode, cudaStream_t look) {
  const int T = (int)gcl.size(), cap = c.cap;
  TL.T = T;
  TL.start.resize(T);
  TL.size.resize(T);
  for (int i = 0; i < T; ++i) {
    TL.start[i] = h->cl_s[gcl[i]];
    TL.size[i] = h->cl_e[gcl[i]] - h->cl_s[gcl[i]];
  }
  TL.hold = std::make_shared<Blk>();
  TL.hold->st = c.st;
  TL.Ap.resize(T);
  TL.Bp.resize(T);
  for (int i = 0; i < T; ++i) {
    TL.Ap[i] = (double*)dmalloc(c, *TL.hold, sizeof(double) * TL.size[i] * T * cap);
    TL.Bp[i] = (double*)dmalloc(c, *TL.hold, sizeof(double) * TL.size[i] * T * cap);
  }
  TL.kmat = (int32_t*)dmalloc(c, *TL.hold, sizeof(int32_t) * T * T);
  {
    std::vector<const double*> ap(TL.Ap.begin(), TL.Ap.end()), bp(TL.Bp.begin(), TL.Bp.end());
    std::vector<int32_t> sz(TL.size.begin(), TL.size.end());
    TL.d_Ap = (const double**)dmalloc(c, *TL.hold, sizeof(void*) * T);
    TL.d_Bp = (const double**)dmalloc(c, *TL.hold, sizeof(void*) * T);
    TL.d_start = (int64_t*)dmalloc(c, *TL.hold, sizeof(int64_t) * T);
    TL.d_size = (int32_t*)dmalloc(c, *TL.hold, sizeof(int32_t) * T);
    if (cudaMemcpyAsync(TL.d_Ap, ap.data(), sizeof(void*) * T, cudaMemcpyHostToDevice, c.st) != cudaSuccess ||
        cudaMemcpyAsync(TL.d_Bp, bp.data(), sizeof(void*) * T, cudaMemcpyHostToDevice, c.st) != cudaSuccess ||
        cudaMemcpyAsync(TL.d_start, TL.start.data(), sizeof(int64_t) * T, cudaMemcpyHostToDevice, c.st) !=
            cudaSuccess ||
        cudaMemcpyAsync(TL.d_size, sz.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice, c.st) != cudaSuccess ||
        cudaStreamSynchronize(c.st) != cudaSuccess)
      throw LuError(HM_ERR_CUDA, "tile tables");
  }
  if (cudaMemsetAsync(TL.kmat, 0, sizeof(int32_t) * T * T, c.st) != cudaSuccess) throw LuError(HM_ERR_CUDA, "memset");
  // load the off-diagonal tiles into the panels and the diagonal tiles as trees
  const int eb = elem_bytes(h->storage);
  std::vector<int32_t> kh(T * T, 0);
  auto tile_of = [&](int64_t r) {
    return (int)(std::upper_bound(TL.start.begin(), TL.start.end(), r) - TL.start.begin()) - 1;
  };
  Loader ld;
  const char* base = (const char*)h->d_rk;
  for (auto& L : h->leaves) {
    const int i0 = tile_of(L.row0), i1 = tile_of(L.row0 + L.m - 1);
    const int j0 = tile_of(L.col0), j1 = tile_of(L.col0 + L.n - 1);
    if (i0 == i1 && j0 == j1 && i0 == j0) continue;            // part of a diagonal tile's tree
    if (L.k > cap) throw LuError(HM_ERR_RANK, "leaf rank above the H-LU rank capacity");
    const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
    // a leaf spanning several tiles: tile (i, j) holds rows of A and of B
    for (int i = i0; i <= i1; ++i)
      for (int j = j0; j <= j1; ++j) {
        kh[i * T + j] = L.k;
        const int64_t ro = TL.start[i] - L.row0, co = TL.start[j] - L.col0;
        ld.jobs.push_back(LoadJob{base + (L.off + co) * eb, npad, (int)TL.size[j], L.k, h->storage,
                                  TL.Bj(i, j, cap), TL.size[j], cap, nullptr, 0});
        ld.jobs.push_back(LoadJob{base + (L.off + npad * L.k + ro) * eb, mpad, (int)TL.size[i], L.k, h->storage,
                                  TL.Ai(i, j, cap), TL.size[i], cap, nullptr, 0});
      }
  }
  if (cudaMemcpyAsync(TL.kmat, kh.data(), sizeof(int32_t) * T * T, cudaMemcpyHostToDevice, c.st) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "rank upload");
  cudaStreamSynchronize(c.st);       // kh leaves scope before the async copy otherwise
  TL.diag.resize(T);
  for (int i = 0; i < T; ++i) TL.diag[i] = build_tree(c, h, dnode[i], ld);
  ld.flush(c);

  // Step k: the diagonal tile's LU and the panels (x: the stream they run on),
  // then the trailing update.  With a look-ahead stream, the LU and panels of
  // tile k+1 run there as soon as step k has updated tile row and column k+1,
  // overlapping the rest of step k's update on the main stream.
  auto panels = [&](Ctx& x, int k, StepQ& out) {
    const int mk = (int)TL.size[k];
    const int R = (T - k - 1) * cap;
    lu_rec(x, *TL.diag[k]);
    if (k > 0) laswp(x, View{TL.Ap[k], 1, mk, mk, k * cap}, TL.start[k]);
    if (R == 0) return;
    View Ua{TL.Ai(k, k + 1, cap), 1, mk, mk, R};          // A factors of tiles (k, j>k)
    View Lb{TL.Bj(k + 1, k, cap), 1, mk, mk, R};          // B factors of tiles (i>k, k)
    laswp(x, Ua, TL.start[k]);
    mfs(x, *TL.diag[k], Ua, true, true);                  // L_kk^{-1} P_k A_kj
    mfs(x, *TL.diag[k], vtr(Lb), false, false);           // B_ik' U_kk^{-1}
    out.hold = std::make_shared<Blk>();
    out.hold->st = c.st;                                  // freed after the main stream used it
    Blk& hold = *out.hold;
    double* W = (double*)dmalloc(x, hold, sizeof(double) * (size_t)R * R);
    View Wv{W, 1, R, R, R};
    gemm(x, Wv, vtr(Lb), Ua, 1.0, 0.0);                   // W_ij = B_ik' A_kj
    // Q_i = A_ik W_i,:   (m_i x R) for every trailing tile row i
    std::vector<double*>& Q = out.Q;
    Q.assign(T, nullptr);
    int64_t qtot = 0;
    for (int i = k + 1; i < T; ++i) qtot += TL.size[i] * (int64_t)R;
    out.qbase = (double*)dmalloc(x, hold, sizeof(double) * (size_t)qtot);
    int64_t qo = 0;
    for (int i = k + 1; i < T; ++i) { Q[i] = out.qbase + qo; qo += TL.size[i] * (int64_t)R; }
    // Q_i = A_ik W_i,: for every trailing tile row: one batched launch, with
    // 128 x 128 tiles once the products are large
    std::vector<GemmJob> gq;
    double macs = 0.0;
    for (int i = k + 1; i < T; ++i) {
      const int mi = (int)TL.size[i];
      GemmJob g{};
      g.A = View{TL.Ai(i, k, cap), 1, mi, mi, cap};
      g.B = vsub(Wv, (i - k - 1) * cap, 0, cap, R);
      g.C = View{Q[i], 1, mi, mi, R};
      g.alpha = 1.0; g.beta = 0.0;
      gq.push_back(g);
      macs += (double)mi * R * cap;
    }
    // 128 x 128 tiles when the batch fills the GPU with them
    int64_t big_tiles = 0;
    for (auto& g : gq) big_tiles += (int64_t)((g.C.rows + GB_T - 1) / GB_T) * ((g.C.cols + GB_T - 1) / GB_T);
    gemm_batch(x, gq, macs >= 4.0e6 && big_tiles >= 148);
  };
  // updates of the trailing diagonal tiles i in [i0, i1) (H-structured targets)
  auto diag_updates = [&](int k, const StepQ& sq, int i0, int i1) {
    std::vector<RcReq> rj;
    std::vector<GemmJob> gd;
    for (int i = i0; i < i1; ++i) {
      const int mi = (int)TL.size[i];
      const double* Qii = sq.Q[i] + (int64_t)(i - k - 1) * cap * mi;
      tile_add_lowrank(*TL.diag[i], 0, 0, Qii, mi, TL.Bj(k, i, cap), mi, TL.kmat + k * T + i, cap, -1.0, gd, rj);
    }
    gemm_batch(c, gd);
    recompress_batch(c, rj, 2 * cap, false);              // no read-back: keeps the host ahead
  };
  Ctx cl = c;
  cl.st = look;
  cudaEvent_t ev_up = nullptr, ev_dn = nullptr;
  if (look && (cudaEventCreateWithFlags(&ev_up, cudaEventDisableTiming) != cudaSuccess ||
               cudaEventCreateWithFlags(&ev_dn, cudaEventDisableTiming) != cudaSuccess))
    throw LuError(HM_ERR_CUDA, "look-ahead events");
  struct EvGuard {
    cudaEvent_t a, b;
    cudaStream_t s;
    ~EvGuard() {
      if (s) cudaStreamSynchronize(s);
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } evg{ev_up, ev_dn, look};
  StepQ cur;
  panels(c, 0, cur);
  for (int k = 0; k < T; ++k) {
    const int R = (T - k - 1) * cap;
    if (R == 0) break;
    const int rl = tile_rank_bound(c, TL, k, 2 * cap);
    StepQ next;
    if (look) {
      diag_updates(k, cur, k + 1, k + 2);
      recompress_tile_pairs(c, TL, k, R, cur.qbase, 2 * cap, 1, rl);   // tile row and column k+1
      if (cudaEventRecord(ev_up, c.st) != cudaSuccess || cudaStreamWaitEvent(look, ev_up, 0) != cudaSuccess)
        throw LuError(HM_ERR_CUDA, "look-ahead wait");
      panels(cl, k + 1, next);
      if (cudaEventRecord(ev_dn, look) != cudaSuccess) throw LuError(HM_ERR_CUDA, "look-ahead record");
      recompress_tile_pairs(c, TL, k, R, cur.qbase, 2 * cap, 2, rl);   // the rest
      diag_updates(k, cur, k + 2, T);
      if (cudaStreamWaitEvent(c.st, ev_dn, 0) != cudaSuccess) throw LuError(HM_ERR_CUDA, "look-ahead join");
    } else {
      diag_updates(k, cur, k + 1, T);
      recompress_tile_pairs(c, TL, k, R, cur.qbase, 2 * cap, 0, rl);
      panels(c, k + 1, next);
    }
    cur = std::move(next);
  }
}

// ---- sweep solve ---------------------------------------------------------
// The triangular solves over the tile level as one kernel per tile: step k of
// a sweep finishes tile k (the update from the tile finished at step k-1, then
// the diagonal tile's triangular solve) in a few finisher CTAs, while the
// other CTAs apply the same finished tile's update to every later tile: 2T
// launches a solve.  The diagonal solves multiply by the inverses of the
// diagonal tiles' L and U factors (computed once from the factored tiles), so
// a step has no row-by-row dependency chain.
constexpr int SW_THREADS = 256;

struct SweepTab {
  const double* const* Ap;
  const double* const* Bp;
  // per tile, the inverse factor sweep_finish applies for which = 0, 1, 2, 3
  const double* const* Inv0;
  const double* const* Inv1;
  const double* const* Inv2;
  const double* const* Inv3;
  const int64_t* start;
  const int32_t* size;
  const int32_t* kmat;
  int T, cap;
};

// The low-rank factors of tile (i, s) as used by a sweep step: y_i -= P (Q' y_s)
// with, non-transposed, P = A_is and Q = B_is (tile (i,s) = A B') and,
// transposed, P = B_si and Q = A_si (tile (s,i)' = B A'); r is the rank.
__device__ __forceinline__ void sweep_factors(const SweepTab& t, int i, int s, bool trans, const double*& P,
                                              const double*& Q, int& r) {  // inlined: no addresses taken
  const int Si = t.size[i], Ss = t.size[s];
  if (!trans) {
    P = t.Ap[i] + (int64_t)s * t.cap * Si;
    Q = t.Bp[s] + (int64_t)i * t.cap * Ss;
    r = t.kmat[i * t.T + s];
  } else {
    P = t.Bp[i] + (int64_t)s * t.cap * Si;
    Q = t.Ap[s] + (int64_t)i * t.cap * Ss;
    r = t.kmat[s * t.T + i];
  }
}

// zsh[q + c r] = (Q' y_s)[q, c], y_s = the finished tile s in F
__device__ void sweep_z(const SweepTab& t, const double* F, int64_t ldy, int nc, int s, const double* Q, int r,
                        double* zsh) {
  const int Ss = t.size[s];
  const double* ys = F + t.start[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int qc = warp; qc < r * nc; qc += SW_THREADS / 32) {
    const int q = qc % r, cc = qc / r;
    double acc = 0.0;
#pragma unroll 8
    for (int row = lane; row < Ss; row += 32)
      acc = fma(__ldg(Q + row + (int64_t)q * Ss), __ldg(ys + row + cc * ldy), acc);
    acc = warp_sum(acc);
    if (lane == 0) zsh[q + cc * r] = acc;
  }
  __syncthreads();
}

// A_i -= P (Q' y_s): the finished tile s applied to the pending tile i
__device__ void sweep_update(const SweepTab& t, double* A, const double* F, int64_t ldy, int nc, int i, int s,
                             bool trans, double* zsh) {
  const double* P;
  const double* Q;
  int r;
  sweep_factors(t, i, s, trans, P, Q, r);
  if (r <= 0) return;
  sweep_z(t, F, ldy, nc, s, Q, r, zsh);
  const int Si = t.size[i];
  double* yi = A + t.start[i];
  for (int e = threadIdx.x; e < Si * nc; e += SW_THREADS) {
    const int row = e % Si, cc = e / Si;
    double acc = 0.0;
#pragma unroll 8
    for (int q = 0; q < r; ++q) acc = fma(__ldg(P + row + (int64_t)q * Si), zsh[q + cc * r], acc);
    yi[row + cc * ldy] -= acc;
  }
}

// Finisher f of tile k: rows [f rpf, f rpf + rpf) (rpf <= 32) of
// M (A_k - P (Q' y_s)) written to F, where M = Inv[which][k] (M[q*S + r] =
// M(r, q); which 0 and 2 lower, 1 and 3 upper).  Lane = row, warp = segment
// of the columns q the rows need: each thread loads its part of M into
// registers first (those loads wait for nothing), then the update of tile k
// from the finished tile s (if any) is recomputed for the rows q needed, and
// the 8 segment sums of a row are added in shared memory.
constexpr int SW_MREG = 32;
__device__ void sweep_finish(const SweepTab& t, const double* A, double* F, int64_t ldy, int nc, int k, int s,
                             bool has_src, bool trans, int which, int f, int rpf, int chunk, double* sh) {
  constexpr int NW = SW_THREADS / 32;
  const int S = t.size[k];
  const int r0 = f * rpf, r1 = min(S, r0 + rpf), nr = r1 - r0;
  if (nr <= 0) return;
  const bool lower = which == 0 || which == 2;
  const int qa = lower ? 0 : r0, qb = lower ? r1 : S, span = qb - qa;
  const int segl = (span + NW - 1) / NW;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool row_ok = lane < nr;
  const int qs = qa + warp * segl;                    // this thread's columns [qs, qs + segl)
  const double* const* inv = which == 0 ? t.Inv0 : which == 1 ? t.Inv1 : which == 2 ? t.Inv2 : t.Inv3;
  const double* M = inv[k] + r0 + lane;               // M(r0 + lane, q) = M[q*S]
  double mreg[SW_MREG];
  const bool in_reg = segl <= SW_MREG;
  if (in_reg) {
#pragma unroll
    for (int j = 0; j < SW_MREG; ++j)
      mreg[j] = (row_ok && j < segl && qs + j < qb) ? __ldg(M + (int64_t)(qs + j) * S) : 0.0;
  }
  double* ysh = sh;                                   // span x chunk
  double* part = ysh + (size_t)S * chunk;             // NW x 32 x chunk
  double* zsh = part + (size_t)NW * 32 * chunk;       // cap x nc
  const double* P = nullptr;
  const double* Q = nullptr;
  int r = 0;
  if (has_src) sweep_factors(t, k, s, trans, P, Q, r);
  if (r > 0) sweep_z(t, F, ldy, nc, s, Q, r, zsh);
  const double* yk = A + t.start[k];
  double* out = F + t.start[k];
  for (int c0 = 0; c0 < nc; c0 += chunk) {
    const int ncc = min(chunk, nc - c0);
    __syncthreads();                                  // ysh and part free
    for (int e = threadIdx.x; e < span * ncc; e += SW_THREADS) {
      const int q = e % span, cc = e / span;
      double v = yk[qa + q + (int64_t)(c0 + cc) * ldy];
#pragma unroll 8
      for (int j = 0; j < r; ++j) v = fma(-__ldg(P + qa + q + (int64_t)j * S), zsh[j + (c0 + cc) * r], v);
      ysh[q + cc * span] = v;
    }
    __syncthreads();
    for (int cc = 0; cc < ncc; ++cc) {
      const double* yv = ysh + cc * span - qa;        // yv[q], q in [qa, qb)
      double acc = 0.0;
      if (in_reg) {
#pragma unroll
        for (int j = 0; j < SW_MREG; ++j)
          if (j < segl && qs + j < qb) acc = fma(mreg[j], yv[qs + j], acc);
      } else if (row_ok) {
        for (int q = qs; q < min(qs + segl, qb); ++q) acc = fma(__ldg(M + (int64_t)q * S), yv[q], acc);
      }
      part[(cc * NW + warp) * 32 + lane] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * ncc; e += SW_THREADS) {
      const int ii = e % nr, cc = e / nr;
      double acc = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) acc += part[(cc * NW + w) * 32 + ii];
      out[r0 + ii + (int64_t)(c0 + cc) * ldy] = acc;
    }
  }
}

// Step k of a sweep (dir +1 forward, -1 backward; which: 0 L, 1 U, 2 U', 3 L').
// A holds the pending right-hand sides, F receives the finished tiles; the
// finished tile s = k - dir is applied to tile k by the nf finisher CTAs and
// to every later tile of the sweep by one CTA each.
__global__ void __launch_bounds__(SW_THREADS, 2) lu_sweep_kernel(SweepTab t, double* A, double* F, int64_t ldy,
                                                              int nc, int k, int dir, int which, int nf, int rpf,
                                                              int chunk) {
  extern __shared__ double sh[];
  const bool trans = which >= 2;
  const int s = k - dir;
  const bool has_src = s >= 0 && s < t.T;
  if ((int)blockIdx.x < nf) {
    sweep_finish(t, A, F, ldy, nc, k, s, has_src, trans, which, blockIdx.x, rpf, chunk, sh);
  } else if (has_src) {
    sweep_update(t, A, F, ldy, nc, k + dir * ((int)blockIdx.x - nf + 1), s, trans, sh);
  }
}

// dense copy of the factored diagonal tiles' leaves (dense or low-rank)
struct DensJob {
  double* dst;
  int64_t ldd;
  const double* C;
  int64_t ldc;
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  const int32_t* k;
  int m, n, type;
};
__global__ void lu_densify_batch_kernel(const DensJob* __restrict__ jobs) {
  const DensJob J = jobs[blockIdx.x];
  const int k = J.type == T_RK ? *J.k : 0;
  for (int64_t e = threadIdx.x; e < (int64_t)J.m * J.n; e += blockDim.x) {
    const int i = (int)(e % J.m), j = (int)(e / J.m);
    double v;
    if (J.type == T_DENSE) {
      v = J.C[i + (int64_t)j * J.ldc];
    } else {
      v = 0.0;
      for (int q = 0; q < k; ++q) v = fma(J.A[i + (int64_t)q * J.lda], J.B[j + (int64_t)q * J.ldb], v);
    }
    J.dst[i + (int64_t)j * J.ldd] = v;
  }
}

static void densify_jobs(const Blk& H, double* dst, int64_t ldd, std::vector<DensJob>& out) {
  if (H.type == T_H) {
    const int m = H.ch[0]->m, n = H.ch[0]->n;
    densify_jobs(*H.ch[0], dst, ldd, out);
    densify_jobs(*H.ch[1], dst + (int64_t)n * ldd, ldd, out);
    densify_jobs(*H.ch[2], dst + m, ldd, out);
    densify_jobs(*H.ch[3], dst + m + (int64_t)n * ldd, ldd, out);
    return;
  }
  out.push_back(DensJob{dst, ldd, H.C, H.ldc, H.A, H.lda, H.B, H.ldb, H.k, H.m, H.n, H.type});
}

// Inverses of the unit-lower L (upper = 0) or the upper U (upper = 1) of the
// packed S x S tiles D (column-major), one thread per column of the inverse,
// written row-major to W (W[i*S + j] = inverse(i, j)) and column-major to Wc.
// All threads of a tile run the same substitution, so the reads of D are
// broadcasts and the reads and writes of W are coalesced.
__global__ void lu_tri_inverse_kernel(const double* const* __restrict__ D, double* const* __restrict__ W,
                                      double* const* __restrict__ Wc, const int32_t* __restrict__ size, int upper) {
  const int tile = blockIdx.y;
  const int S = size[tile];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.x * blockDim.x >= S) return;
  const double* d = D[tile];
  double* w = W[tile];
  double* wc = Wc[tile];
  const bool act = j < S;
  if (!upper) {
    for (int i = 0; i < S; ++i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int l = 0; l < i; ++l) s = fma(-d[i + (int64_t)l * S], act ? w[(int64_t)l * S + j] : 0.0, s);
      if (act) {
        const double v = (i < j) ? 0.0 : s;
        w[(int64_t)i * S + j] = v;
        wc[i + (int64_t)j * S] = v;
      }
    }
  } else {
    for (int i = S - 1; i >= 0; --i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int l = i + 1; l < S; ++l) s = fma(-d[i + (int64_t)l * S], act ? w[(int64_t)l * S + j] : 0.0, s);
      if (act) {
        const double v = (i > j) ? 0.0 : s / d[i + (int64_t)i * S];
        w[(int64_t)i * S + j] = v;
        wc[i + (int64_t)j * S] = v;
      }
    }
  }
}

// inverse factors and device tables, once per factorisation
static void ensure_sweep(Ctx& c, TileLU& TL) {
  if (TL.d_inv[0]) return;
  const int T = TL.T;
  auto hold = std::make_shared<Blk>();
  hold->st = c.st;
  Blk tmp;
  tmp.st = c.st;
  int smax = 0;
  std::vector<double*> D(T);
  std::vector<const double*> inv[4];         // Lc, Uc, Ur, Lr: the matrices of which = 0..3
  std::vector<DensJob> jobs;
  for (int k = 0; k < T; ++k) {
    const int S = (int)TL.size[k];
    smax = std::max(smax, S);
    D[k] = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)S * S);
    for (int w = 0; w < 4; ++w) inv[w].push_back((double*)dmalloc(c, *hold, sizeof(double) * (size_t)S * S));
    densify_jobs(*TL.diag[k], D[k], S, jobs);
  }
  for (size_t b = 0; b < jobs.size(); b += 65535) {
    const size_t nb = std::min<size_t>(65535, jobs.size() - b);
    std::vector<DensJob> part(jobs.begin() + b, jobs.begin() + b + nb);
    DensJob* dj = upload_jobs(c, tmp, part);
    lu_densify_batch_kernel<<<(unsigned)nb, 256, 0, c.st>>>(dj);
    LU_LAUNCH_CHECK();
  }
  std::vector<int32_t> sz(T);
  for (int k = 0; k < T; ++k) sz[k] = (int32_t)TL.size[k];
  std::vector<const double*> Ap(TL.Ap.begin(), TL.Ap.end()), Bp(TL.Bp.begin(), TL.Bp.end());
  auto up = [&](const void* src, size_t bytes) {
    void* d = dmalloc(c, *hold, bytes);
    if (cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, c.st) != cudaSuccess)
      throw LuError(HM_ERR_CUDA, "sweep tables");
    return d;
  };
  double** dD = (double**)dmalloc(c, tmp, sizeof(void*) * T);
  if (cudaMemcpyAsync(dD, D.data(), sizeof(void*) * T, cudaMemcpyHostToDevice, c.st) != cudaSuccess)
    throw LuError(HM_ERR_CUDA, "sweep tables");
  if (!TL.d_Ap) {                            // a copied factorisation has no tables yet
    TL.d_Ap = (const double**)up(Ap.data(), sizeof(void*) * T);
    TL.d_Bp = (const double**)up(Bp.data(), sizeof(void*) * T);
    TL.d_start = (int64_t*)up(TL.start.data(), sizeof(int64_t) * T);
    TL.d_size = (int32_t*)up(sz.data(), sizeof(int32_t) * T);
  }
  for (int w = 0; w < 4; ++w) TL.d_inv[w] = (const double**)up(inv[w].data(), sizeof(void*) * T);
  const dim3 g((smax + 127) / 128, T);
  // L^-1: row-major (which 3) and column-major (which 0); U^-1: row-major (2), column-major (1)
  lu_tri_inverse_kernel<<<g, 128, 0, c.st>>>(dD, (double* const*)TL.d_inv[3], (double* const*)TL.d_inv[0],
                                             TL.d_size, 0);
  LU_LAUNCH_CHECK();
  lu_tri_inverse_kernel<<<g, 128, 0, c.st>>>(dD, (double* const*)TL.d_inv[2], (double* const*)TL.d_inv[1],
                                             TL.d_size, 1);
  LU_LAUNCH_CHECK();
  if (cudaStreamSynchronize(c.st) != cudaSuccess) throw LuError(HM_ERR_CUDA, "sweep set-up");
  TL.sweep_hold = hold;
}

static void tile_solve(Ctx& c, const TileLU& TL, View X, bool trans, double* Zext);

// the two sweeps of a\y (trans 0) or a'\y (trans 1) on X in place (X already
// permuted for a\y; permuted afterwards by the caller for a'\y).  The
// forward sweep finishes tiles into a second array W, the backward sweep
// takes W as its right-hand sides and finishes into X.
static void tile_sweeps(Ctx& c, const TileLU& TL, View X, bool trans) {
  const int T = TL.T, nc = X.cols;
  int smax = 1;
  for (int k = 0; k < T; ++k) smax = std::max<int>(smax, (int)TL.size[k]);
  const int rpf = 32;                                              // rows of a finisher (a lane each)
  const int chunk = std::min(nc, 8);                               // columns staged per pass
  const size_t smem = sizeof(double) * ((size_t)smax * chunk + (size_t)SW_THREADS * chunk + (size_t)c.cap * nc);
  if (smem > 200 * 1024 || X.rs != 1) {
    tile_solve(c, TL, X, trans, nullptr);
    return;
  }
  if (smem_attr((const void*)lu_sweep_kernel, 200 * 1024) != cudaSuccess) throw LuError(HM_ERR_CUDA, "sweep smem");
  Blk tmp;
  tmp.st = c.st;
  double* W = (double*)dmalloc(c, tmp, sizeof(double) * (size_t)X.cs * nc);
  SweepTab t{TL.d_Ap, TL.d_Bp, TL.d_inv[0], TL.d_inv[1], TL.d_inv[2], TL.d_inv[3], TL.d_start, TL.d_size,
             TL.kmat, T, c.cap};
  for (int k = 0; k < T; ++k) {
    const int nf = ((int)TL.size[k] + rpf - 1) / rpf;
    const int nu = k > 0 ? T - 1 - k : 0;
    lu_sweep_kernel<<<nf + nu, SW_THREADS, smem, c.st>>>(t, X.p, W, X.cs, nc, k, 1, trans ? 2 : 0, nf, rpf, chunk);
    LU_LAUNCH_CHECK();
  }
  for (int k = T - 1; k >= 0; --k) {
    const int nf = ((int)TL.size[k] + rpf - 1) / rpf;
    const int nu = k < T - 1 ? k : 0;
    lu_sweep_kernel<<<nf + nu, SW_THREADS, smem, c.st>>>(t, W, X.p, X.cs, nc, k, -1, trans ? 3 : 1, nf, rpf, chunk);
    LU_LAUNCH_CHECK();
  }
}

// y = P b, forward (unit L), backward (U) tile by tile; trans: U' then L'
// (the launch-per-operation form, used beyond SWEEP_MAX_COLS right-hand sides)
static void tile_solve(Ctx& c, const TileLU& TL, View X, bool trans, double* Zext) {
  const int T = TL.T, cap = c.cap, nc = X.cols;
  auto yv = [&](int i) { return vsub(X, (int)TL.start[i], 0, (int)TL.size[i], nc); };
  Blk tmp;
  tmp.st = c.st;
  double* Z = Zext ? Zext : (double*)dmalloc(c, tmp, sizeof(double) * (size_t)T * cap * nc);
  if (!trans) {
    for (int k = 0; k < T; ++k) {                       // L y = b
      solve_rec(c, *TL.diag[k], yv(k), true);
      const int R = (T - k - 1) * cap;
      if (R == 0) break;
      View Zv{Z, 1, R, R, nc};
      gemm(c, Zv, vtr(View{TL.Bj(k + 1, k, cap), 1, TL.size[k], (int)TL.size[k], R}), yv(k), 1.0, 0.0);
      std::vector<GemmJob> g;
      for (int i = k + 1; i < T; ++i)
        g.push_back(GemmJob{View{TL.Ai(i, k, cap), 1, TL.size[i], (int)TL.size[i], cap},
                            vsub(Zv, (i - k - 1) * cap, 0, cap, nc), yv(i), -1.0, 1.0});
      gemm_batch(c, g);
    }
    for (int k = T - 1; k >= 0; --k) {                  // U x = y
      const int R = (T - k - 1) * cap;
      if (R > 0) {
        View Zv{Z, 1, R, R, nc};
        std::vector<GemmJob> g;
        for (int j = k + 1; j < T; ++j)
          g.push_back(GemmJob{vtr(View{TL.Bj(k, j, cap), 1, TL.size[j], (int)TL.size[j], cap}), yv(j),
                              vsub(Zv, (j - k - 1) * cap, 0, cap, nc), 1.0, 0.0});
        gemm_batch(c, g);
        gemm(c, yv(k), View{TL.Ai(k, k + 1, cap), 1, TL.size[k], (int)TL.size[k], R}, Zv, -1.0, 1.0);
      }
      solve_rec(c, *TL.diag[k], yv(k), false);
    }
  } else {
    for (int k = 0; k < T; ++k) {                       // U' z = b
      solve_t_rec(c, *TL.diag[k], yv(k), true);
      const int R = (T - k - 1) * cap;
      if (R == 0) break;
      View Zv{Z, 1, R, R, nc};
      gemm(c, Zv, vtr(View{TL.Ai(k, k + 1, cap), 1, TL.size[k], (int)TL.size[k], R}), yv(k), 1.0, 0.0);
      std::vector<GemmJob> g;
      for (int j = k + 1; j < T; ++j)
        g.push_back(GemmJob{View{TL.Bj(k, j, cap), 1, TL.size[j], (int)TL.size[j], cap},
                            vsub(Zv, (j - k - 1) * cap, 0, cap, nc), yv(j), -1.0, 1.0});
      gemm_batch(c, g);
    }
    for (int k = T - 1; k >= 0; --k) {                  // L' w = z
      const int R = (T - k - 1) * cap;
      if (R > 0) {
        View Zv{Z, 1, R, R, nc};
        std::vector<GemmJob> g;
        for (int i = k + 1; i < T; ++i)
          g.push_back(GemmJob{vtr(View{TL.Ai(i, k, cap), 1, TL.size[i], (int)TL.size[i], cap}), yv(i),
                              vsub(Zv, (i - k - 1) * cap, 0, cap, nc), 1.0, 0.0});
        gemm_batch(c, g);
        gemm(c, yv(k), View{TL.Bj(k + 1, k, cap), 1, TL.size[k], (int)TL.size[k], R}, Zv, -1.0, 1.0);
      }
      solve_t_rec(c, *TL.diag[k], yv(k), false);
    }
  }
}

static void tile_densify(Ctx& c, const TileLU& TL, View D) {
  const int T = TL.T, cap = c.cap;
  std::vector<GemmJob> g;
  for (int i = 0; i < T; ++i)
    for (int j = 0; j < T; ++j) {
      View blk = vsub(D, (int)TL.start[i], (int)TL.start[j], (int)TL.size[i], (int)TL.size[j]);
      if (i == j) densify_into(c, blk, *TL.diag[i]);
      else
        g.push_back(GemmJob{View{TL.Ai(i, j, cap), 1, TL.size[i], (int)TL.size[i], cap},
                            vtr(View{TL.Bj(i, j, cap), 1, TL.size[j], (int)TL.size[j], cap}), blk, 1.0, 0.0});
    }
  gemm_batch(c, g);
}

// ---------------------------------------------------------------------------
// state, entry points
// ---------------------------------------------------------------------------
// One captured solve: the launch sequence of a\y (or a'\y) for a fixed number
// of right-hand sides, recorded into a CUDA graph that works on the plan's own
// input/output buffers.  A call copies b in, launches the graph, copies x out.
struct SolvePlan {
  int64_t ncols = 0;
  int trans = 0;
  double* xin = nullptr;   // n x ncols, right-hand sides (the transposed solve works in place here)
  double* xout = nullptr;  // n x ncols, solution
  double* Z = nullptr;     // tile-solve product scratch
  Arena arena;             // temporaries of the captured sequence
  JobTape tape;
  cudaGraphExec_t exec = nullptr;
  bool no_graph = false;   // capture failed: the plan runs its sequence directly
  ~SolvePlan() {           // the owner has synchronised the device
    if (exec) cudaGraphExecDestroy(exec);
    for (void* p : {(void*)xin, (void*)xout, (void*)Z, (void*)arena.base})
      if (p) cudaFreeAsync(p, cudaStreamLegacy);
  }
};

struct LuState {
  BP root;                       // recursive format
  std::unique_ptr<TileLU> tile;  // tile format
  int64_t* P = nullptr;
  int* flags = nullptr;
  int cap = 0;
  cudaStream_t st = nullptr;
  // look-ahead stream of the tile schedule (blocks made there keep it as
  // their stream, so it lives as long as the factors)
  cudaStream_t look = nullptr;
  std::vector<std::unique_ptr<SolvePlan>> plans;
  ~LuState() {
    if (!plans.empty()) cudaDeviceSynchronize();
    plans.clear();
    if (look) cudaStreamSynchronize(look);
    root.reset();
    tile.reset();
    if (P) cudaFreeAsync(P, st);
    if (flags) cudaFreeAsync(flags, st);
    if (st) cudaStreamSynchronize(st);
    if (look) {
      cudaStreamSynchronize(look);
      cudaStreamDestroy(look);
    }
  }
  // a second stream (nullptr if it cannot be made: the schedule then runs on
  // one stream)
  void make_look() {
    if (look) return;
    // high priority: its small kernels are scheduled between the blocks of the
    // main stream's large recompression launches instead of after them
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&look, cudaStreamNonBlocking, greatest) != cudaSuccess) {
      cudaGetLastError();
      look = nullptr;
    }
  }
};

static BP build_tree(Ctx& c, const hm_handle* h, int32_t node, Loader& ld) {
  const Node& nd = h->nodes[node];
  const int m = (int)(h->cl_e[nd.s] - h->cl_s[nd.s]), n = (int)(h->cl_e[nd.t] - h->cl_s[nd.t]);
  if (nd.type == T_H) {
    BP b = std::make_shared<Blk>();
    b->st = c.st;
    b->type = T_H; b->m = m; b->n = n; b->s = nd.s; b->t = nd.t; b->row0 = h->cl_s[nd.s];
    for (int q = 0; q < 4; ++q) b->ch[q] = build_tree(c, h, nd.child[q], ld);
    return b;
  }
  const Leaf& L = h->leaves[nd.leaf];
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  if (nd.type == T_DENSE) {
    BP d = new_dense(c, m, n, nd.s, nd.t);
    d->row0 = L.row0;
    const int dt = h->storage == HM_F64 ? HM_F64 : HM_F32;
    ld.jobs.push_back(LoadJob{(const char*)h->d_dense + L.off * deb, col_pad(m, deb), m, n, dt, d->C, d->ldc, n,
                              nullptr, 0});
    return d;
  }
  if (L.k > c.cap) throw LuError(HM_ERR_RANK, "leaf rank above the H-LU rank capacity");
  BP r = new_rk(c, m, n, nd.s, nd.t);
  r->row0 = L.row0;
  const int64_t npad = col_pad(n, eb), mpad = col_pad(m, eb);
  const char* base = (const char*)h->d_rk;
  ld.jobs.push_back(LoadJob{base + L.off * eb, npad, n, L.k, h->storage, r->B, r->ldb, c.cap, nullptr, 0});
  ld.jobs.push_back(LoadJob{base + (L.off + npad * L.k) * eb, mpad, m, L.k, h->storage, r->A, r->lda, c.cap,
                            r->k, L.k});
  return r;
}

static BP build_from_handle(Ctx& c, const hm_handle* h, int32_t node) {
  Loader ld;
  BP b = build_tree(c, h, node, ld);
  ld.flush(c);
  return b;
}

static int finish(Ctx& c, const char* what) {
  int flags = 0;
  HM_CUDA_TRY(cudaMemcpyAsync(&flags, c.flags, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  HM_CUDA_TRY(cudaStreamSynchronize(c.st));
  if (flags & 4) return fail(HM_ERR_SINGULAR, std::string(what) + ": exactly zero pivot in a diagonal leaf");
  if (flags & 2) return fail(HM_ERR_NONFINITE, std::string(what) + ": non-finite values");
  if (flags & 1) return fail(HM_ERR_RANK, std::string(what) + ": a rank exceeded the capacity " + std::to_string(c.cap));
  return HM_OK;
}

int lu_factor(hm_handle* h) {
  // the factorisation allocates and frees many stream-ordered temporaries:
  // keep freed memory in the device's pool instead of returning it to the
  // driver at every synchronisation
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, h->device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  LuState* S = new LuState();
  S->st = h->stream;
  // capacity of low-rank blocks: twice the largest leaf rank (updated blocks
  // are truncated back after every addition), at least 12; HM_ERR_RANK if a
  // truncated rank ever exceeds it (raise rank_cap then)
  S->cap = h->prm.rank_cap > 0 ? h->prm.rank_cap : std::max(12, 2 * std::max(h->kmax, 1));
  S->cap = std::min(S->cap, RCORE_MAX / 2);
  HM_CUDA_TRY(cudaMallocAsync((void**)&S->P, sizeof(int64_t) * h->n, h->stream));
  HM_CUDA_TRY(cudaMallocAsync((void**)&S->flags, sizeof(int), h->stream));
  HM_CUDA_TRY(cudaMemsetAsync(S->flags, 0, sizeof(int), h->stream));
  const double eps_lu = h->prm.eps_trunc_lu > 0.0 ? h->prm.eps_trunc_lu : h->prm.eps_trunc;
  Ctx c{h->stream, S->cap, S->P, S->flags, eps_lu, h};
  const int mode = h->prm.lu_mode;     // 0 auto, 1 recursion, 2 tiles
  try {
    if (h->kmax > S->cap) throw LuError(HM_ERR_RANK, "a leaf rank exceeds the H-LU rank capacity");
    std::vector<int32_t> gcl, dnode;
    const bool tiled = mode != 1 && tile_structure(h, gcl, dnode);
    if (mode == 2 && !tiled) throw LuError(HM_ERR_UNSUPPORTED, "the partition has no tile level");
    if (tiled) {
      S->tile.reset(new TileLU());
      S->make_look();
      tile_factor(c, h, *S->tile, gcl, dnode, S->look);
    } else {
      S->root = build_from_handle(c, h, 0);
      lu_rec(c, *S->root);
    }
  } catch (const LuError& e) {
    cudaStreamSynchronize(h->stream);
    delete S;
    return fail(e.code, std::string("lu!: ") + e.what());
  }
  int s = finish(c, "lu!");
  if (s != HM_OK) {
    delete S;
    return s;
  }
  h->lu = S;
  h->factorized = true;
  return HM_OK;
}

// right-hand sides per sweep solve (the update's z values sit in shared memory)
static constexpr int SWEEP_MAX_COLS = 64;

// The launch sequence of a\y (trans = 0) or a'\y (trans = 1) from d_b into d_x.
// W, when given, is the working copy of b for the transposed solve; it may be
// d_b itself (the solve then overwrites b).
static void issue_solve(Ctx& c, LuState* S, const hm_handle* h, const double* d_b, double* d_x, int nc,
                        int trans, double* Z, double* W) {
  View B{const_cast<double*>(d_b), 1, h->n, (int)h->n, nc};
  View X{d_x, 1, h->n, (int)h->n, nc};
  const int64_t tot = h->n * nc;
  const unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, 4096);
  if (!trans) {
    // a\y (src/hlu.jl:553-562): permute!(w, P), unit-L forward, U backward
    lu_gather_rows_kernel<<<g, 256, 0, c.st>>>(X, B, S->P);
    LU_LAUNCH_CHECK();
    if (S->tile && S->tile->d_inv[0] && nc <= SWEEP_MAX_COLS) {
      tile_sweeps(c, *S->tile, X, false);
    } else if (S->tile) {
      tile_solve(c, *S->tile, X, false, Z);
    } else {
      solve_rec(c, *S->root, X, true);
      solve_rec(c, *S->root, X, false);
    }
  } else {
    Blk tmp;
    tmp.st = c.st;
    double* w = W ? W : (double*)dmalloc(c, tmp, sizeof(double) * (size_t)tot);
    View Wv{w, 1, h->n, (int)h->n, nc};
    if (w != d_b) axpby(c, Wv, B, 1.0, 0.0);
    if (S->tile && S->tile->d_inv[0] && nc <= SWEEP_MAX_COLS) {
      tile_sweeps(c, *S->tile, Wv, true);
    } else if (S->tile) {
      tile_solve(c, *S->tile, Wv, true, Z);
    } else {
      solve_t_rec(c, *S->root, Wv, true);
      solve_t_rec(c, *S->root, Wv, false);
    }
    lu_scatter_rows_kernel<<<g, 256, 0, c.st>>>(X, Wv, S->P);
    LU_LAUNCH_CHECK();
  }
}

// Solves with at most this many right-hand sides are captured into a graph.
static constexpr int64_t SOLVE_GRAPH_MAX_COLS = 64;
static constexpr size_t SOLVE_MAX_PLANS = 8;

static SolvePlan* new_plan(LuState* S, const hm_handle* h, int64_t nc, int trans, cudaStream_t st) {
  auto pl = std::make_unique<SolvePlan>();
  pl->ncols = nc;
  pl->trans = trans;
  const size_t xb = sizeof(double) * (size_t)h->n * nc;
  const size_t zb = S->tile ? sizeof(double) * (size_t)S->tile->T * S->cap * nc : 8;
  if (cudaMallocAsync(&pl->xin, xb, st) != cudaSuccess || cudaMallocAsync(&pl->xout, xb, st) != cudaSuccess ||
      cudaMallocAsync(&pl->Z, zb, st) != cudaSuccess) {
    cudaGetLastError();
    throw LuError(HM_ERR_OOM, "solve plan buffers");
  }
  if (S->plans.size() >= SOLVE_MAX_PLANS) {
    cudaDeviceSynchronize();
    S->plans.erase(S->plans.begin());
  }
  S->plans.push_back(std::move(pl));
  return S->plans.back().get();
}

// Records the plan's sequence into a graph on a private stream.  Nothing runs
// during capture; a failure leaves the plan without a graph.
static void capture_plan(LuState* S, hm_handle* h, SolvePlan* pl, cudaStream_t caller) {
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    pl->no_graph = true;
    return;
  }
  if (pl->tape.temp_bytes > 0 &&
      cudaMallocAsync((void**)&pl->arena.base, pl->tape.temp_bytes, caller) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(cs);
    pl->no_graph = true;
    return;
  }
  pl->arena.size = pl->tape.temp_bytes;
  pl->arena.used = 0;
  Ctx c{cs, S->cap, S->P, S->flags, h->prm.eps_trunc, h, &pl->arena};
  pl->tape.record = false;
  pl->tape.replay = true;
  pl->tape.pos = 0;
  bool ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    g_tape = &pl->tape;
    try {
      issue_solve(c, S, h, pl->xin, pl->xout, (int)pl->ncols, pl->trans, pl->Z, pl->xin);
    } catch (const LuError&) {
      ok = false;
    }
    g_tape = nullptr;
    cudaGraph_t graph = nullptr;
    if (cudaStreamEndCapture(cs, &graph) != cudaSuccess) ok = false;
    if (ok && pl->tape.pos != pl->tape.bufs.size()) ok = false;
    if (ok && cudaGraphInstantiate(&pl->exec, graph, 0) != cudaSuccess) {
      pl->exec = nullptr;
      ok = false;
    }
    if (graph) cudaGraphDestroy(graph);
  }
  cudaGetLastError();                  // capture errors are not sticky; clear them
  pl->tape.replay = false;
  pl->no_graph = !ok;
  cudaStreamDestroy(cs);
  // the plan's buffers were allocated in the caller's stream order; later
  // calls may come on other streams
  cudaStreamSynchronize(caller);
}

int lu_solve_device(hm_handle* h, const double* d_b, double* d_x, int64_t ncols, int trans, cudaStream_t st) {
  LuState* S = h->lu;
  if (!S) return fail(HM_ERR_STATE, "a has not been factorized");
  if (ncols <= 0) return HM_OK;
  Ctx c{st, S->cap, S->P, S->flags, h->prm.eps_trunc, h};
  try {
    if (S->tile) ensure_sweep(c, *S->tile);
    if (ncols > SOLVE_GRAPH_MAX_COLS) {
      issue_solve(c, S, h, d_b, d_x, (int)ncols, trans, nullptr, nullptr);
    } else {
      SolvePlan* pl = nullptr;
      for (auto& q : S->plans)
        if (q->ncols == ncols && q->trans == trans) pl = q.get();
      const size_t xb = sizeof(double) * (size_t)h->n * ncols;
      if (pl && pl->exec) {
        HM_LU_CUDA(cudaMemcpyAsync(pl->xin, d_b, xb, cudaMemcpyDeviceToDevice, st));
        HM_LU_CUDA(cudaGraphLaunch(pl->exec, st));
        HM_LU_CUDA(cudaMemcpyAsync(d_x, pl->xout, xb, cudaMemcpyDeviceToDevice, st));
      } else if (pl) {                 // capture failed earlier: direct run on the plan's buffers
        HM_LU_CUDA(cudaMemcpyAsync(pl->xin, d_b, xb, cudaMemcpyDeviceToDevice, st));
        issue_solve(c, S, h, pl->xin, pl->xout, (int)ncols, trans, pl->Z, pl->xin);
        HM_LU_CUDA(cudaMemcpyAsync(d_x, pl->xout, xb, cudaMemcpyDeviceToDevice, st));
      } else {                         // first solve of this shape: run it recording, then capture
        pl = new_plan(S, h, ncols, trans, st);
        HM_LU_CUDA(cudaMemcpyAsync(pl->xin, d_b, xb, cudaMemcpyDeviceToDevice, st));
        pl->tape.record = true;
        g_tape = &pl->tape;
        try {
          issue_solve(c, S, h, pl->xin, pl->xout, (int)ncols, trans, pl->Z, pl->xin);
        } catch (...) {
          g_tape = nullptr;
          pl->tape.record = false;
          throw;
        }
        g_tape = nullptr;
        pl->tape.record = false;
        HM_LU_CUDA(cudaMemcpyAsync(d_x, pl->xout, xb, cudaMemcpyDeviceToDevice, st));
        capture_plan(S, h, pl, st);
      }
    }
  } catch (const LuError& e) {
    return fail(e.code, std::string("H\\y: ") + e.what());
  }
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

__global__ void lu_colnorm2_kernel(View X, double* __restrict__ out) {
  __shared__ double red[32];
  const int c = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < X.rows; i += blockDim.x) {
    const double v = X.p[(int64_t)i * X.rs + (int64_t)c * X.cs];
    s = fma(v, v, s);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[c] = s;
}

// Iterative refinement: x = (LU)^{-1} b, then r = b - H x with the FP64
// H-matvec of the unfactorised matrix (the matvec pools stay intact after
// lu!), x += (LU)^{-1} r, until max_c |r_c|/|b_c| <= tol or max_iter steps.
int lu_solve_refined(hm_handle* h, const double* d_b, double* d_x, int64_t ncols, int trans, double tol,
                     int max_iter, cudaStream_t st, int* iters, double* relres) {
  if (!h->lu) return fail(HM_ERR_STATE, "a has not been factorized");
  const int64_t n = h->n, tot = n * ncols;
  double *r = nullptr, *d = nullptr, *nrm = nullptr;
  HM_CUDA_TRY(cudaMallocAsync(&r, sizeof(double) * tot, st));
  HM_CUDA_TRY(cudaMallocAsync(&d, sizeof(double) * tot, st));
  HM_CUDA_TRY(cudaMallocAsync(&nrm, sizeof(double) * 2 * ncols, st));
  std::vector<double> hb(ncols), hr(ncols);
  int status = HM_OK, it = 0;
  double worst = 0.0;
  View Bv{const_cast<double*>(d_b), 1, n, (int)n, (int)ncols};
  View Rv{r, 1, n, (int)n, (int)ncols};
  Ctx c{st, h->lu->cap, h->lu->P, h->lu->flags, h->prm.eps_trunc, h};
  auto norms = [&](View V, double* dst, std::vector<double>& host) -> int {
    lu_colnorm2_kernel<<<(unsigned)ncols, 256, 0, st>>>(V, dst);
    HM_CUDA_TRY(cudaGetLastError());
    HM_CUDA_TRY(cudaMemcpyAsync(host.data(), dst, sizeof(double) * ncols, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
    return HM_OK;
  };
  status = norms(Bv, nrm, hb);
  if (status == HM_OK) status = lu_solve_device(h, d_b, d_x, ncols, trans, st);
  for (; status == HM_OK; ++it) {
    // r = b - H x, summed in twice the FP64 precision
    for (int64_t q = 0; q < ncols && status == HM_OK; ++q)
      status = residual_device(h, d_x + q * n, d_b + q * n, r + q * n, trans, st);
    if (status != HM_OK) break;
    status = norms(Rv, nrm + ncols, hr);
    if (status != HM_OK) break;
    worst = 0.0;
    bool finite = true;
    for (int64_t q = 0; q < ncols; ++q) {
      const double v = hb[q] > 0 ? std::sqrt(hr[q] / hb[q]) : std::sqrt(hr[q]);
      if (!std::isfinite(v) || !std::isfinite(hb[q])) finite = false;   // std::max would drop a NaN
      worst = std::max(worst, v);
    }
    if (!finite) { status = fail(HM_ERR_NONFINITE, "refinement: non-finite residual"); break; }
    if (worst <= tol || it >= max_iter) break;
    status = lu_solve_device(h, r, d, ncols, trans, st);
    if (status != HM_OK) break;
    try {
      axpby(c, View{d_x, 1, n, (int)n, (int)ncols}, View{d, 1, n, (int)n, (int)ncols}, 1.0, 1.0);
    } catch (const LuError& e) {
      status = fail(e.code, e.what());
      break;
    }
  }
  cudaFreeAsync(r, st);
  cudaFreeAsync(d, st);
  cudaFreeAsync(nrm, st);
  cudaStreamSynchronize(st);
  if (iters) *iters = it;
  if (relres) *relres = worst;
  return status;
}

void lu_describe(const hm_handle* h, int64_t* tiles, int64_t* cap) {
  *tiles = h->lu && h->lu->tile ? h->lu->tile->T : 0;
  *cap = h->lu ? h->lu->cap : 0;
}

int lu_perm(const hm_handle* h, int64_t* P) {
  if (!h->lu) return fail(HM_ERR_STATE, "a has not been factorized");
  HM_CUDA_TRY(cudaMemcpyAsync(P, h->lu->P, sizeof(int64_t) * h->n, cudaMemcpyDeviceToHost, h->stream));
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HM_OK;
}

int lu_to_dense(const hm_handle* h, double* d_out) {
  if (!h->lu) return fail(HM_ERR_STATE, "a has not been factorized");
  Ctx c{h->stream, h->lu->cap, h->lu->P, h->lu->flags, h->prm.eps_trunc, h};
  try {
    View D{d_out, 1, h->n, (int)h->n, (int)h->n};
    if (h->lu->tile) tile_densify(c, *h->lu->tile, D);
    else densify_into(c, D, *h->lu->root);
  } catch (const LuError& e) {
    return fail(e.code, e.what());
  }
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HM_OK;
}

void lu_free(hm_handle* h) {
  delete h->lu;
  h->lu = nullptr;
}

int lu_copy(const hm_handle* src, hm_handle* dst) {
  if (!src->lu) return HM_OK;
  LuState* S = new LuState();
  S->st = dst->stream;
  S->cap = src->lu->cap;
  HM_CUDA_TRY(cudaStreamSynchronize(src->stream));
  HM_CUDA_TRY(cudaMallocAsync((void**)&S->P, sizeof(int64_t) * src->n, dst->stream));
  HM_CUDA_TRY(cudaMallocAsync((void**)&S->flags, sizeof(int), dst->stream));
  HM_CUDA_TRY(cudaMemcpyAsync(S->P, src->lu->P, sizeof(int64_t) * src->n, cudaMemcpyDeviceToDevice, dst->stream));
  HM_CUDA_TRY(cudaMemsetAsync(S->flags, 0, sizeof(int), dst->stream));
  Ctx c{dst->stream, S->cap, S->P, S->flags, src->prm.eps_trunc, src};
  try {
    if (src->lu->tile) {
      const TileLU& A = *src->lu->tile;
      TileLU* B = new TileLU();
      S->tile.reset(B);
      B->T = A.T;
      B->start = A.start;
      B->size = A.size;
      B->hold = std::make_shared<Blk>();
      B->hold->st = c.st;
      B->Ap.resize(A.T);
      B->Bp.resize(A.T);
      for (int i = 0; i < A.T; ++i) {
        const size_t bytes = sizeof(double) * A.size[i] * A.T * S->cap;
        B->Ap[i] = (double*)dmalloc(c, *B->hold, bytes);
        B->Bp[i] = (double*)dmalloc(c, *B->hold, bytes);
        if (cudaMemcpyAsync(B->Ap[i], A.Ap[i], bytes, cudaMemcpyDeviceToDevice, c.st) != cudaSuccess ||
            cudaMemcpyAsync(B->Bp[i], A.Bp[i], bytes, cudaMemcpyDeviceToDevice, c.st) != cudaSuccess)
          throw LuError(HM_ERR_CUDA, "panel copy");
      }
      B->kmat = (int32_t*)dmalloc(c, *B->hold, sizeof(int32_t) * A.T * A.T);
      if (cudaMemcpyAsync(B->kmat, A.kmat, sizeof(int32_t) * A.T * A.T, cudaMemcpyDeviceToDevice, c.st) !=
          cudaSuccess)
        throw LuError(HM_ERR_CUDA, "rank copy");
      B->diag.resize(A.T);
      for (int i = 0; i < A.T; ++i) B->diag[i] = copy_blk(c, *A.diag[i]);
    } else {
      S->root = copy_blk(c, *src->lu->root);
    }
  } catch (const LuError& e) {
    delete S;
    return fail(e.code, e.what());
  }
  HM_CUDA_TRY(cudaStreamSynchronize(dst->stream));
  dst->lu = S;
  return HM_OK;
}

}  // namespace hm
