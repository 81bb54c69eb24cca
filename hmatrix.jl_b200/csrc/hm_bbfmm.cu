// Chebyshev-interpolation construction of the low-rank leaves ("bbfmm",
// the reference's default ConsMethod: src/cluster.jl:68-75, src/hlu.jl:20-29,
// 113-132, deps/src/lowrank.cpp:24-222), for sm_100a.
//
// For a leaf with row points X (m) and column points Y (n):
//   nodes    c_i = u_i (b - a) / 2 + (a + b) / 2, u_i = cos(pi (2i + 1) / (2r)),
//            [a, b] the bounding interval of the points in each coordinate;
//   Lagrange L(x)_j = prod_{k != j} (x - c_k) / (c_j - c_k), products in k order;
//   1-D: U = L_X S, V = L_Y, S_ij = K(cX_i, cY_j), rank r = MaxRank;
//   2-D: node (i, j) = (cx_i, cy_j) at index i r + j, P(x)_(i r + j) =
//        Lx(x)_i Ly(x)_j, U = P_X S, V = P_Y, rank r^2, with r lowered to
//        floor(sqrt(max(m, n))) when r^2 > max(m, n) (src/hlu.jl:24-26).
// H_leaf = U V' is stored as A = U, B = V.  V and the interpolation tables
// use the reference's operation order with no FMA contraction (bit-identical
// to a CPU restatement with the same unit nodes); U = P_X S is an FP64
// product whose summation order differs from Eigen's GEMM.
//
// Two kernels per chunk of leaves: bbfmm_tables_kernel (one CTA per leaf:
// bounding boxes, nodes, the 1-D Lagrange tables of both sides and S into an
// FP64 scratch, then V into the pool) and bbfmm_u_kernel (64 x 64 tiles of
// U = P_X S, P_X formed from the tables while it is staged in shared memory).
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace hm {

namespace {

constexpr double kPi = 3.14159265358979323846;   // M_PI
constexpr int BB_RMAX = 64;          // r <= MaxRank <= 64
constexpr int BB_THREADS = 256;
constexpr int BB_TILE = 64;          // U tile: 64 rows x 64 columns
constexpr int BB_KC = 16;            // inner-dimension chunk of the U product

struct BbJob {
  int64_t row0, col0;   // first row / column point of the leaf
  int64_t off;          // element offset of the leaf in the low-rank pool
  int64_t scr;          // double offset of the leaf's tables in the scratch
  int32_t m, n, r, R;   // R = r (1-D) or r^2 (2-D)
};

struct BbTile {
  int32_t job, rt, ct;  // leaf (index into the chunk), row tile, column tile
};

__device__ __forceinline__ void bb_minmax(double& lo, double& hi, double* red) {
  // block-wide min / max (exact, order-free); red holds 2 * 32 doubles
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { red[w] = lo; red[32 + w] = hi; }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  lo = red[0];
  hi = red[32];
  for (int q = 1; q < nw; ++q) { lo = fmin(lo, red[q]); hi = fmax(hi, red[32 + q]); }
}

// Lagrange basis j at x on the nodes c[0..r) (Interpolation::ComputeMatrix).
__device__ __forceinline__ double bb_lagrange(double x, const double* c, int r, int j) {
  double L = 1.0;
  for (int k = 0; k < r; ++k)
    if (k != j) L = __dmul_rn(L, __ddiv_rn(__dsub_rn(x, c[k]), __dsub_rn(c[j], c[k])));
  return L;
}

// Tables of one leaf in the scratch (doubles from J.scr): LX (d blocks of
// m x r, column-major), LY (d blocks of n x r), S (R x R, column-major).
template <typename T>
__global__ void __launch_bounds__(BB_THREADS) bbfmm_tables_kernel(KernelDesc kd, const double* __restrict__ geom,
                                                                  int64_t ng, const BbJob* __restrict__ jobs,
                                                                  const double* __restrict__ unit,
                                                                  double* __restrict__ scratch,
                                                                  T* __restrict__ pool, int eb) {
  __shared__ double red[64];
  __shared__ double cn[2][2][BB_RMAX];   // side (0 rows, 1 columns), coordinate, node
  const BbJob J = jobs[blockIdx.x];
  const int d = kd.dim, r = J.r, R = J.R, m = J.m, n = J.n;
  // bounding intervals (minimum/maximum of each coordinate, lowrank.cpp:152-155, hlu.jl:119)
  for (int side = 0; side < 2; ++side) {
    const int64_t p0 = side ? J.col0 : J.row0;
    const int cnt = side ? n : m;
    for (int q = 0; q < d; ++q) {
      double lo = INFINITY, hi = -INFINITY;
      for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const double v = geom[p0 + k + (int64_t)q * ng];
        lo = fmin(lo, v);
        hi = fmax(hi, v);
      }
      bb_minmax(lo, hi, red);
      // nodes: u * (b - a) / 2 + (a + b) / 2 (lowrank.cpp:33-35, 40-41)
      const double* u = unit + (int64_t)r * BB_RMAX;
      for (int i = threadIdx.x; i < r; i += blockDim.x)
        cn[side][q][i] = __dadd_rn(__ddiv_rn(__dmul_rn(u[i], __dsub_rn(hi, lo)), 2.0),
                                   __ddiv_rn(__dadd_rn(lo, hi), 2.0));
      __syncthreads();
    }
  }
  double* LX = scratch + J.scr;
  double* LY = LX + (int64_t)d * m * r;
  double* S = LY + (int64_t)d * n * r;
  for (int side = 0; side < 2; ++side) {
    const int64_t p0 = side ? J.col0 : J.row0;
    const int cnt = side ? n : m;
    double* L = side ? LY : LX;
    const int64_t tot = (int64_t)d * cnt * r;
    for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
      const int q = (int)(e / ((int64_t)cnt * r));
      const int rem = (int)(e - (int64_t)q * cnt * r);
      const int j = rem / cnt, k = rem - j * cnt;
      L[e] = bb_lagrange(geom[p0 + k + (int64_t)q * ng], cn[side][q], r, j);
    }
  }
  // S(a, b) = K(node a of the rows, node b of the columns) (lowrank.cpp:92-94, 176-178)
  for (int64_t e = threadIdx.x; e < (int64_t)R * R; e += blockDim.x) {
    const int b = (int)(e / R), a = (int)(e - (int64_t)b * R);
    double xa[2], xb[2];
    if (d == 1) {
      xa[0] = cn[0][0][a];
      xb[0] = cn[1][0][b];
    } else {
      xa[0] = cn[0][0][a / r]; xa[1] = cn[0][1][a % r];
      xb[0] = cn[1][0][b / r]; xb[1] = cn[1][1][b % r];
    }
    S[e] = kernel_eval_xy(kd, xa, 1, xb, 1);
  }
  __syncthreads();   // the Y tables are read by other threads below
  // V = P_Y into the B slot (n x R, column stride npad, padding rows zero)
  const int64_t npad = col_pad_dev(n, eb);
  T* Bout = pool + J.off;
  for (int64_t e = threadIdx.x; e < npad * R; e += blockDim.x) {
    const int b = (int)(e / npad), k = (int)(e - (int64_t)b * npad);
    double v = 0.0;
    if (k < n) v = d == 1 ? LY[(int64_t)b * n + k]
                          : __dmul_rn(LY[(int64_t)(b / r) * n + k], LY[(int64_t)n * r + (int64_t)(b % r) * n + k]);
    Bout[e] = to_store<T>(v);
  }
}

// U = P_X S for one 64 x 64 tile, written to the A slot (m x R, column
// stride mpad, padding rows zero).
template <typename T>
__global__ void __launch_bounds__(BB_THREADS) bbfmm_u_kernel(int dim, const BbJob* __restrict__ jobs,
                                                             const BbTile* __restrict__ tiles,
                                                             const double* __restrict__ scratch,
                                                             T* __restrict__ pool, int eb) {
  __shared__ double Ps[BB_KC][BB_TILE + 1];
  __shared__ double Ss[BB_KC][BB_TILE + 1];
  const BbTile tl = tiles[blockIdx.x];
  const BbJob J = jobs[tl.job];
  const int r = J.r, R = J.R, m = J.m, n = J.n;
  const double* LX = scratch + J.scr;
  const double* S = LX + (int64_t)dim * m * r + (int64_t)dim * n * r;
  const int row0 = tl.rt * BB_TILE, col0 = tl.ct * BB_TILE;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;    // 4 x 4 outputs a thread
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int a0 = 0; a0 < R; a0 += BB_KC) {
    __syncthreads();
    for (int e = threadIdx.x; e < BB_KC * BB_TILE; e += blockDim.x) {
      const int kk = e / BB_TILE, i = e - kk * BB_TILE;
      const int a = a0 + kk, row = row0 + i, col = col0 + i;
      double p = 0.0, s = 0.0;
      if (a < R && row < m)
        p = dim == 1 ? LX[(int64_t)a * m + row]
                     : __dmul_rn(LX[(int64_t)(a / r) * m + row], LX[(int64_t)m * r + (int64_t)(a % r) * m + row]);
      if (a < R && col < R) s = S[(int64_t)col * R + a];
      Ps[kk][i] = p;
      Ss[kk][i] = s;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BB_KC; ++kk) {
      double pv[4], sv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) pv[i] = Ps[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) sv[j] = Ss[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(pv[i], sv[j], acc[i][j]);
    }
  }
  const int64_t npad = col_pad_dev(n, eb), mpad = col_pad_dev(m, eb);
  T* Aout = pool + J.off + npad * R;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int col = col0 + tx + 16 * j;
    if (col >= R) continue;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = row0 + ty + 16 * i;
      if (row < mpad) Aout[(int64_t)col * mpad + row] = to_store<T>(row < m ? acc[i][j] : 0.0);
    }
  }
}

template <typename T>
int bbfmm_chunk(hm_handle* h, const std::vector<BbJob>& jobs, const double* d_unit, double* d_scr,
                cudaStream_t st) {
  std::vector<BbTile> tiles;
  for (int32_t j = 0; j < (int32_t)jobs.size(); ++j) {
    const int eb = (int)sizeof(T);
    const int64_t mpad = col_pad(jobs[j].m, eb);
    const int nrt = (int)((mpad + BB_TILE - 1) / BB_TILE), nct = (jobs[j].R + BB_TILE - 1) / BB_TILE;
    for (int rt = 0; rt < nrt; ++rt)
      for (int ct = 0; ct < nct; ++ct) tiles.push_back(BbTile{j, rt, ct});
  }
  BbJob* dj = nullptr;
  BbTile* dt = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void**)&dj, sizeof(BbJob) * jobs.size(), st));
  HM_CUDA_TRY(cudaMallocAsync((void**)&dt, sizeof(BbTile) * tiles.size(), st));
  HM_CUDA_TRY(cudaMemcpyAsync(dj, jobs.data(), sizeof(BbJob) * jobs.size(), cudaMemcpyHostToDevice, st));
  HM_CUDA_TRY(cudaMemcpyAsync(dt, tiles.data(), sizeof(BbTile) * tiles.size(), cudaMemcpyHostToDevice, st));
  bbfmm_tables_kernel<T><<<(unsigned)jobs.size(), BB_THREADS, 0, st>>>(h->kd, h->d_geom, h->n, dj, d_unit, d_scr,
                                                                      (T*)h->d_rk, (int)sizeof(T));
  HM_CUDA_TRY(cudaGetLastError());
  bbfmm_u_kernel<T><<<(unsigned)tiles.size(), BB_THREADS, 0, st>>>(h->kd.dim, dj, dt, d_scr, (T*)h->d_rk,
                                                                  (int)sizeof(T));
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaFreeAsync(dj, st));
  HM_CUDA_TRY(cudaFreeAsync(dt, st));
  return HM_OK;
}

}  // namespace

int bbfmm_rank(int64_t m, int64_t n, int dim, int max_rank) {
  int r = max_rank;
  if (dim >= 2) {
    const int64_t mx = std::max(m, n);
    if ((int64_t)r * r > mx) r = (int)std::floor(std::sqrt((double)mx));
    return r * r;
  }
  return r;
}

int bbfmm_write(hm_handle* h, const std::vector<int64_t>& rk_leaf) {
  if (rk_leaf.empty()) return HM_OK;
  const int d = h->kd.dim;
  if (d > 2) return fail(HM_ERR_UNSUPPORTED, "bbfmm construction takes 1-D or 2-D geometry");
  // unit Chebyshev nodes cos(pi (2i + 1) / (2r)) for every r <= 64, on the host
  // (lowrank.cpp:26-31): the same libm cos as a CPU restatement
  std::vector<double> unit((size_t)(BB_RMAX + 1) * BB_RMAX, 0.0);
  for (int r = 1; r <= BB_RMAX; ++r)
    for (int i = 0; i < r; ++i) unit[(size_t)r * BB_RMAX + i] = std::cos(kPi * (2.0 * i + 1.0) / (2.0 * r));
  cudaStream_t st = h->stream;
  double* d_unit = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void**)&d_unit, sizeof(double) * unit.size(), st));
  HM_CUDA_TRY(cudaMemcpyAsync(d_unit, unit.data(), sizeof(double) * unit.size(), cudaMemcpyHostToDevice, st));
  // leaves in chunks whose tables fit a 512 MB scratch (at least one leaf a chunk)
  const int64_t budget = (int64_t)64 << 20;   // doubles
  std::vector<std::vector<BbJob>> chunks(1);
  int64_t used = 0, maxscr = 0;
  for (int64_t li : rk_leaf) {
    const Leaf& L = h->leaves[li];
    const int R = L.k;
    const int r = d == 1 ? R : (int)std::lround(std::sqrt((double)R));
    if (r < 1 || r > BB_RMAX || (d == 2 && r * r != R)) return fail(HM_ERR_CUDA, "bbfmm: invalid leaf rank");
    const int64_t need = (int64_t)d * (L.m + L.n) * r + (int64_t)R * R;
    if (!chunks.back().empty() && used + need > budget) {
      chunks.emplace_back();
      used = 0;
    }
    chunks.back().push_back(BbJob{L.row0, L.col0, L.off, used, L.m, L.n, r, R});
    used += need;
    maxscr = std::max(maxscr, used);
  }
  double* d_scr = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void**)&d_scr, sizeof(double) * std::max<int64_t>(maxscr, 1), st));
  for (auto& c : chunks) {
    int s;
    switch (h->storage) {
      case HM_F64: s = bbfmm_chunk<double>(h, c, d_unit, d_scr, st); break;
      case HM_F32: s = bbfmm_chunk<float>(h, c, d_unit, d_scr, st); break;
      default: s = bbfmm_chunk<__nv_bfloat16>(h, c, d_unit, d_scr, st);
    }
    if (s != HM_OK) return s;
  }
  HM_CUDA_TRY(cudaFreeAsync(d_scr, st));
  HM_CUDA_TRY(cudaFreeAsync(d_unit, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  return HM_OK;
}

}  // namespace hm
