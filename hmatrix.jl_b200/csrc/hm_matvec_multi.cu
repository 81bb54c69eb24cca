// Multi-RHS H-matvec (K5) on the CUDA cores: Y = H X and Y = H' X for an
// n x c block of right-hand sides, the device form of *(Hmat, Matrix)
// (src/harithm.jl:323-329), which the reference evaluates one column at a
// time.  Every factor is streamed from HBM once per block of CB columns
// instead of once per column, in FP64 arithmetic.  This is the path of FP64
// factors (tcgen05 has no FP64 kind) and of the dense leaves of FP32/BF16
// handles, whose low-rank part runs on the tensor cores (hm_matvec_tc.cu).
//
// Layout: the input is first transposed into XR, n+2 rows of LD = c rounded up
// to CB doubles (row i holds x[i, 0..c), zero padded), so that a leaf row's CB
// values are contiguous 16-byte loads.  Phase 1 writes ZR, one row of LD
// values per low-rank term; phase 2 writes Y column-major directly.
//
// Phase 1: one warp per low-rank leaf and column block; a lane owns pairs of
//          segment rows, accumulates two ranks x CB columns, and the warp
//          reduces the 2*CB sums with a butterfly reduce-scatter.
// Phase 2: one CTA per (window half of 512 rows, column block); a thread owns
//          2 consecutive rows x CB columns; the (leaf, column) entries of the
//          window are expanded in shared memory with their CB z values.
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <algorithm>
#include <type_traits>
#include <vector>

namespace hm {

namespace {

__device__ __forceinline__ float mbf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float mbf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

// two consecutive elements of a factor column as FP64 (the pair starts on an
// even element; columns are padded to 4 elements and 16 bytes)
template <typename T> struct Pair;
template <> struct Pair<double> {
  __device__ static double2 ld(const double* p) { return __ldcs(reinterpret_cast<const double2*>(p)); }
  __device__ static double one(const double* p) { return __ldcs(p); }
};
template <> struct Pair<float> {
  __device__ static double2 ld(const float* p) {
    const float2 v = __ldcs(reinterpret_cast<const float2*>(p));
    return make_double2(v.x, v.y);
  }
  __device__ static double one(const float* p) { return (double)__ldcs(p); }
};
template <> struct Pair<__nv_bfloat16> {
  __device__ static double2 ld(const __nv_bfloat16* p) {
    const uint32_t w = __ldcs(reinterpret_cast<const unsigned int*>(p));
    return make_double2(mbf_lo(w), mbf_hi(w));
  }
  __device__ static double one(const __nv_bfloat16* p) {
    const unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
    return (double)__uint_as_float((uint32_t)u << 16);
  }
};

// Sums NV values over the warp.  Each round halves the values a lane keeps
// (it sends the other half to the partner lane), so 2*CB sums cost NV-1
// shuffles instead of 5*NV.  On return the lane holds the total of value idx;
// the lanes that agree in their low log2(32/NV) bits hold the same total.
template <int NV>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[NV], int lane, int& idx) {
  idx = 0;
#pragma unroll
  for (int h = NV / 2, o = 16; h >= 1; h >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const double send = up ? v[i] : v[i + h];
      const double keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
    if (up) idx += h;
  }
  double s = v[0];
#pragma unroll
  for (int o = 16 / NV; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// XR[i, j] = X[i + j * ldx] (j < ncols, i < n), zero elsewhere, for n + 2 rows
__global__ void mvm_xr_kernel(const double* __restrict__ X, int64_t n, int64_t ldx, int ncols,
                              double* __restrict__ xr, int ld) {
  const int64_t tot = (n + 2) * ld;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / ld;
    const int j = (int)(e % ld);
    xr[e] = (i < n && j < ncols) ? X[i + (int64_t)j * ldx] : 0.0;
  }
}

// Phase 1 works on groups of up to G1 leaves that share an input segment
// (descriptors ordered by segment): one x load then feeds G1 leaves x 2 ranks.
// Lane = (row sub-index rs, column pair cp): a 32-row chunk of the segment is
// read as RS x IT rows by CP column pairs, so each warp-wide x load is 512
// contiguous bytes; the factor values of the chunk are loaded once (lane l
// holds row l) and handed to the lanes that need them by shuffles.
constexpr int G1 = 4;

template <typename T, int CB>
__global__ void __launch_bounds__(256) mvm_phase1_kernel(const P1Desc* __restrict__ d, const uint32_t* __restrict__ grp,
                                                         int64_t ngrp, const T* __restrict__ pool,
                                                         const double* __restrict__ xr, int ld, int ncb,
                                                         double* __restrict__ zr) {
  constexpr int CP = CB / 2, RS = 32 / CP, IT = 32 / RS;
  const int lane = threadIdx.x & 31;
  const int cp = lane % CP, rs = lane / CP;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = gw; w < ngrp * ncb; w += nw) {
    const int64_t g = w / ncb;
    const int cb = (int)(w % ncb);
    const uint32_t b0 = grp[g], nb = grp[g + 1] - b0;
    P1Desc D[G1];
    int kmax = 0;
#pragma unroll
    for (int q = 0; q < G1; ++q) {
      if (q < (int)nb) {
        D[q] = d[b0 + q];
        kmax = max(kmax, (int)D[q].k);
      } else {
        D[q].k = 0;
      }
    }
    const uint32_t seg0 = D[0].seg0, len = D[0].len;
    const double* xb = xr + (int64_t)seg0 * ld + cb * CB + 2 * cp;
    for (int r = 0; r < kmax; r += 2) {
      double acc[G1][2][2];
#pragma unroll
      for (int q = 0; q < G1; ++q)
#pragma unroll
        for (int a = 0; a < 2; ++a) acc[q][a][0] = acc[q][a][1] = 0.0;
      for (uint32_t r0 = 0; r0 < len; r0 += 32) {
        double2 xv[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
          const uint32_t row = r0 + RS * it + rs;
          xv[it] = row < len ? __ldg(reinterpret_cast<const double2*>(xb + (int64_t)row * ld)) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int q = 0; q < G1; ++q) {
          if (r < (int)D[q].k) {             // uniform over the warp
            const T* f0 = pool + D[q].off + (int64_t)r * D[q].stride;
            const bool two = r + 1 < (int)D[q].k;
            const uint32_t row = r0 + lane;
            const double a0 = row < len ? (double)from_store<T>(f0[row]) : 0.0;
            const double a1 = (two && row < len) ? (double)from_store<T>(f0[D[q].stride + row]) : 0.0;
#pragma unroll
            for (int it = 0; it < IT; ++it) {
              const double u = __shfl_sync(0xffffffffu, a0, RS * it + rs);
              const double v = __shfl_sync(0xffffffffu, a1, RS * it + rs);
              acc[q][0][0] = fma(u, xv[it].x, acc[q][0][0]);
              acc[q][0][1] = fma(u, xv[it].y, acc[q][0][1]);
              acc[q][1][0] = fma(v, xv[it].x, acc[q][1][0]);
              acc[q][1][1] = fma(v, xv[it].y, acc[q][1][1]);
            }
          }
        }
      }
      // sum over the RS lanes that share a column pair
#pragma unroll
      for (int o = CP; o < 32; o <<= 1)
#pragma unroll
        for (int q = 0; q < G1; ++q)
#pragma unroll
          for (int a = 0; a < 2; ++a) {
            acc[q][a][0] += __shfl_xor_sync(0xffffffffu, acc[q][a][0], o);
            acc[q][a][1] += __shfl_xor_sync(0xffffffffu, acc[q][a][1], o);
          }
      if (rs == 0) {
#pragma unroll
        for (int q = 0; q < G1; ++q)
#pragma unroll
          for (int a = 0; a < 2; ++a)
            if (r + a < (int)D[q].k) {
              double* zp = zr + (int64_t)(D[q].zoff + r + a) * ld + cb * CB + 2 * cp;
              *reinterpret_cast<double2*>(zp) = make_double2(acc[q][a][0], acc[q][a][1]);
            }
      }
    }
  }
}

// Phase 1, segment tasks: a CTA takes up to S1_LEAVES leaves that share one
// input segment (descriptors ordered by segment) and stages the segment's rows
// of X (its CB columns) in shared memory once, rows padded by two doubles so
// that the 32 rows a warp reads at a time fall in distinct banks.  Each warp
// runs one leaf at a time, lane = row: its factor values come from its own
// coalesced loads (a block of S1_ROWS rows prefetched at once), its x row from
// shared memory, and the 2 x CB sums are reduced over the warp at the end.
constexpr int S1_LEAVES = 64;
constexpr int S1_ROWS = 256;                // factor rows prefetched per pass

template <typename T, int CB>
__global__ void __launch_bounds__(256) mvm_phase1_seg_kernel(const P1Desc* __restrict__ d,
                                                             const uint32_t* __restrict__ task, int64_t ntask,
                                                             const T* __restrict__ pool,
                                                             const double* __restrict__ xr, int ld, int ncb,
                                                             double* __restrict__ zr) {
  constexpr int XS = CB + 2;                          // padded row of the staged X
  constexpr int NV = 2 * CB;
  extern __shared__ double xs[];                     // len x XS
  const int64_t tk = blockIdx.x / ncb;
  const int cb = (int)(blockIdx.x % ncb);
  const uint32_t b0 = task[tk], b1 = task[tk + 1];
  const uint32_t seg0 = d[b0].seg0, len = d[b0].len;
  const double* xb = xr + (int64_t)seg0 * ld + cb * CB;
  for (uint32_t e = threadIdx.x; e < len * (CB / 2); e += blockDim.x) {
    const uint32_t row = e / (CB / 2), c2 = e % (CB / 2);
    *reinterpret_cast<double2*>(xs + row * XS + 2 * c2) =
        __ldg(reinterpret_cast<const double2*>(xb + (int64_t)row * ld) + c2);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t b = b0 + warp; b < b1; b += blockDim.x / 32) {
    const P1Desc D = d[b];
    const T* F = pool + D.off;
    for (int r = 0; r < D.k; r += 2) {
      const bool two = r + 1 < D.k;
      const T* f0 = F + (int64_t)r * D.stride;
      double v[NV];
#pragma unroll
      for (int c = 0; c < NV; ++c) v[c] = 0.0;
      for (uint32_t base = 0; base < len; base += S1_ROWS) {
        double u0[S1_ROWS / 32], u1[S1_ROWS / 32];
#pragma unroll
        for (int q = 0; q < S1_ROWS / 32; ++q) {
          const uint32_t row = base + 32 * q + lane;
          u0[q] = row < len ? (double)from_store<T>(f0[row]) : 0.0;
          u1[q] = (two && row < len) ? (double)from_store<T>(f0[D.stride + row]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < S1_ROWS / 32; ++q) {
          const uint32_t row = base + 32 * q + lane;
          if (base + 32 * q >= len) break;
          if (row < len) {
            const double* xrow = xs + row * XS;
#pragma unroll
            for (int c = 0; c < CB; c += 2) {
              const double2 xv = *reinterpret_cast<const double2*>(xrow + c);
              v[c] = fma(u0[q], xv.x, v[c]);
              v[c + 1] = fma(u0[q], xv.y, v[c + 1]);
              v[CB + c] = fma(u1[q], xv.x, v[CB + c]);
              v[CB + c + 1] = fma(u1[q], xv.y, v[CB + c + 1]);
            }
          }
        }
      }
      int idx;
      const double sum = warp_reduce_scatter<NV>(v, lane, idx);
      if ((lane & (32 / NV - 1)) == 0) {
        const int rank = r + idx / CB, col = idx % CB;
        if (rank < D.k) zr[(int64_t)(D.zoff + rank) * ld + cb * CB + col] = sum;
      }
    }
  }
}

constexpr int M2_THREADS = 256;             // 2 rows a thread: half a window
constexpr int M2_NB = 32;                   // descriptors staged per round
constexpr uint64_t M2_DENSE_FLAG = 1ull << 63;

template <int CB> struct M2Cfg {
  static constexpr int EMAX = CB >= 16 ? 256 : 512;   // entries per sub-round (z rows in shared memory)
};

template <typename T, typename TD, int CB>
__global__ void __launch_bounds__(M2_THREADS) mvm_phase2_kernel(const MvWin* __restrict__ win,
                                                                const P2Desc* __restrict__ d,
                                                                const T* __restrict__ rk, const TD* __restrict__ dn,
                                                                const double* __restrict__ zr,
                                                                const double* __restrict__ xr, int ld, int ncb,
                                                                double* __restrict__ Y, int64_t ldy, int ncols) {
  constexpr int EMAX = M2Cfg<CB>::EMAX;
  constexpr int U = CB >= 16 ? 4 : 8;         // entries whose factor loads are in flight together
  __shared__ P2Desc sd[M2_NB];
  __shared__ int spre[M2_NB + 1];
  __shared__ uint64_t e_off[EMAX];
  __shared__ int32_t e_ro[EMAX];
  __shared__ uint32_t e_m[EMAX];
  __shared__ uint32_t e_rs[EMAX];
  __shared__ __align__(16) double e_z[EMAX * CB];
  const int cb = (int)(blockIdx.x % ncb);
  const int64_t wh = blockIdx.x / ncb;
  const MvWin W = win[wh >> 1];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int base = (int)(wh & 1) * (2 * M2_THREADS) + 2 * threadIdx.x;   // first of this thread's 2 rows
  double acc[2][CB];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int j = 0; j < CB; ++j) acc[q][j] = 0.0;
  for (uint32_t b0 = W.begin; b0 < W.end; b0 += M2_NB) {
    const int nb = (int)min((uint32_t)M2_NB, W.end - b0);
    __syncthreads();
    if (warp == 0) {
      int cnt = 0;
      if (lane < nb) {
        sd[lane] = d[b0 + lane];
        // only leaves that cover rows of this half window are expanded
        const int r0 = sd[lane].row_off, r1 = r0 + (int)sd[lane].m;
        const int h0 = (int)(wh & 1) * (2 * M2_THREADS);
        cnt = (r1 > h0 && r0 < h0 + 2 * M2_THREADS) ? (int)sd[lane].cnt : 0;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      spre[lane + 1] = incl;
      if (lane == 0) spre[0] = 0;
    }
    __syncthreads();
    const int total = spre[nb];
    for (int e0 = 0; e0 < total; e0 += EMAX) {
      const int ne = min(EMAX, total - e0);
      if (e0 > 0) __syncthreads();
      for (int e = threadIdx.x; e < ne; e += blockDim.x) {
        const int ge = e0 + e;
        int lo = 0, hi = nb - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (spre[mid] <= ge) lo = mid; else hi = mid - 1;
        }
        const P2Desc& D = sd[lo];
        const int c = ge - spre[lo];
        const double* zsrc;
        if (D.type == P2_RK) {
          e_off[e] = D.off + (uint64_t)c * D.ld;
          e_rs[e] = 1;
          zsrc = zr + (int64_t)(D.aux + c) * ld + cb * CB;
        } else if (D.type == P2_DENSE) {
          e_off[e] = (D.off + (uint64_t)c * D.ld) | M2_DENSE_FLAG;
          e_rs[e] = 1;
          zsrc = xr + (int64_t)(D.aux + c) * ld + cb * CB;
        } else {
          e_off[e] = (D.off + (uint64_t)c) | M2_DENSE_FLAG;
          e_rs[e] = D.ld;
          zsrc = xr + (int64_t)(D.aux + c) * ld + cb * CB;
        }
#pragma unroll
        for (int j = 0; j < CB; j += 2)
          *reinterpret_cast<double2*>(e_z + e * CB + j) = __ldg(reinterpret_cast<const double2*>(zsrc + j));
        e_ro[e] = D.row_off;
        e_m[e] = D.m;
      }
      __syncthreads();
      for (int e = 0; e < ne; e += U) {
        double2 f[U];
        bool cov = false;                     // some entry of this group covers a row of this thread
#pragma unroll
        for (int u = 0; u < U; ++u) {
          f[u] = make_double2(0.0, 0.0);
          const int ee = e + u;
          if (ee < ne) {
            const int ro = e_ro[ee];
            const int mm = (int)e_m[ee];
            const uint64_t o = e_off[ee];
            const uint32_t rs = e_rs[ee];
            const int lr = base - ro;
            cov = cov || (lr + 1 >= 0 && lr < mm);
            const bool dense = (o & M2_DENSE_FLAG) != 0;
            const uint64_t oo = o & ~M2_DENSE_FLAG;
            if (((ro & 1) == 0) && rs == 1) {
              if (lr >= 0 && lr < mm) f[u] = dense ? Pair<TD>::ld(dn + oo + lr) : Pair<T>::ld(rk + oo + lr);
            } else {
              if (lr >= 0 && lr < mm)
                f[u].x = dense ? Pair<TD>::one(dn + oo + (uint64_t)lr * rs) : Pair<T>::one(rk + oo + lr);
              if (lr + 1 >= 0 && lr + 1 < mm)
                f[u].y = dense ? Pair<TD>::one(dn + oo + (uint64_t)(lr + 1) * rs) : Pair<T>::one(rk + oo + lr + 1);
            }
          }
        }
        // a warp covers 64 consecutive rows: leaves shorter than the half
        // window (dense near-field blocks) leave most warps idle here
        if (!__any_sync(0xffffffffu, cov)) continue;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (e + u < ne) {
            const double* zz = e_z + (e + u) * CB;
#pragma unroll
            for (int j = 0; j < CB; j += 2) {
              const double2 zv = *reinterpret_cast<const double2*>(zz + j);
              acc[0][j] = fma(f[u].x, zv.x, acc[0][j]);
              acc[0][j + 1] = fma(f[u].x, zv.y, acc[0][j + 1]);
              acc[1][j] = fma(f[u].y, zv.x, acc[1][j]);
              acc[1][j + 1] = fma(f[u].y, zv.y, acc[1][j + 1]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int r = base + q;
    if (r < (int)W.nrows) {
#pragma unroll
      for (int j = 0; j < CB; ++j) {
        const int col = cb * CB + j;
        if (col < ncols) Y[(int64_t)(W.row0 + r) + (int64_t)col * ldy] = acc[q][j];
      }
    }
  }
}

// The dense leaves' part of Y = H X alone (the tensor-core kernels add the
// low-rank part afterwards).  One CTA per 128 output rows and column block,
// a warp per 32 rows.  Warp 0 collects the window's dense leaves that cover
// the tile; for each, the CTA stages the X rows of its input segment in shared
// memory (DX_ROWS at a time, coalesced) and every warp whose rows it covers
// streams the leaf column by column (32 consecutive rows a load, eight
// columns in flight) against those rows.  Each warp writes its rows of Y once.
constexpr int DX_ROWS = 64;

template <typename TD, int CB>
__global__ void __launch_bounds__(128) mvm_dense_kernel(const MvWin* __restrict__ win, const P2Desc* __restrict__ d,
                                                        const TD* __restrict__ dn, const double* __restrict__ xr,
                                                        int ld, int ncb, int64_t ntile, double* __restrict__ Y,
                                                        int64_t ldy, int ncols) {
  __shared__ P2Desc sd[32];
  __shared__ int s_cnt;
  __shared__ __align__(16) double xs[DX_ROWS * CB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cb = (int)(blockIdx.x % ncb);
  const int64_t grow = (int64_t)(blockIdx.x / ncb) * 128;      // first output row of the tile
  const MvWin W = win[grow / MV_WROWS];
  const int t0 = (int)(grow - W.row0);                         // tile rows [t0, t0 + 128) of the window
  const int w0 = t0 + 32 * warp;                               // this warp's rows [w0, w0 + 32)
  const int r = w0 + lane;
  double acc[CB];
#pragma unroll
  for (int j = 0; j < CB; ++j) acc[j] = 0.0;
  for (uint32_t b0 = W.begin; b0 < W.end; b0 += 32) {
    __syncthreads();
    if (warp == 0) {
      const uint32_t nb = min(32u, W.end - b0);
      P2Desc D{};
      bool cov = false;
      if ((uint32_t)lane < nb) {
        D = d[b0 + lane];
        cov = D.row_off < t0 + 128 && D.row_off + (int)D.m > t0;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, cov);
      if (cov) sd[__popc(bal & ((1u << lane) - 1u))] = D;
      if (lane == 0) s_cnt = __popc(bal);
    }
    __syncthreads();
    const int cnt = s_cnt;
    for (int li = 0; li < cnt; ++li) {
      const P2Desc L = sd[li];
      const bool wcov = L.row_off < w0 + 32 && L.row_off + (int)L.m > w0;   // uniform per warp
      const int lr = r - L.row_off;
      const bool mine = lr >= 0 && lr < (int)L.m;
      const bool tr = L.type == P2_DENSE_T;
      const TD* col = dn + L.off + (mine ? (tr ? (int64_t)lr * L.ld : (int64_t)lr) : 0);
      const int64_t cs = tr ? 1 : (int64_t)L.ld;                // distance between the leaf's input columns
      for (uint32_t c0 = 0; c0 < L.cnt; c0 += DX_ROWS) {
        const int nr = (int)min((uint32_t)DX_ROWS, L.cnt - c0);
        __syncthreads();                                         // the previous rows are consumed
        for (int e = threadIdx.x; e < nr * (CB / 2); e += blockDim.x) {
          const int rr = e / (CB / 2), jj = e % (CB / 2);
          reinterpret_cast<double2*>(xs)[e] =
              __ldg(reinterpret_cast<const double2*>(xr + (int64_t)(L.aux + c0 + rr) * ld + cb * CB) + jj);
        }
        __syncthreads();
        if (!wcov) continue;
        int c = 0;
        for (; c + 8 <= nr; c += 8) {
          double v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) v[u] = mine ? (double)__ldcs(col + (int64_t)(c0 + c + u) * cs) : 0.0;
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const double* xx = xs + (c + u) * CB;
#pragma unroll
            for (int j = 0; j < CB; j += 2) {
              const double2 x = *reinterpret_cast<const double2*>(xx + j);
              acc[j] = fma(v[u], x.x, acc[j]);
              acc[j + 1] = fma(v[u], x.y, acc[j + 1]);
            }
          }
        }
        for (; c < nr; ++c) {
          const double v = mine ? (double)__ldcs(col + (int64_t)(c0 + c) * cs) : 0.0;
          const double* xx = xs + c * CB;
#pragma unroll
          for (int j = 0; j < CB; j += 2) {
            const double2 x = *reinterpret_cast<const double2*>(xx + j);
            acc[j] = fma(v, x.x, acc[j]);
            acc[j + 1] = fma(v, x.y, acc[j + 1]);
          }
        }
      }
    }
  }
  if (r < (int)W.nrows) {
#pragma unroll
    for (int j = 0; j < CB; ++j) {
      const int cl = cb * CB + j;
      if (cl < ncols) Y[(int64_t)(W.row0 + r) + (int64_t)cl * ldy] = acc[j];
    }
  }
}

// Phase-1 descriptors ordered by input segment: the warps running at the same
// time then read the same rows of XR (L1/L2 hits) instead of c x 8 bytes per
// row from HBM for every leaf.  Stable, so a segment's leaves keep pool order.
// Groups of at most G1 consecutive sorted descriptors with the same segment:
// P.d_g1s[g] is the first descriptor of group g, P.d_g1s[ng1] = np1.
static int ensure_sorted_p1(MvPlan& P) {
  if (P.d_p1s || P.np1 == 0) return HM_OK;
  std::vector<P1Desc> v((size_t)P.np1);
  HM_CUDA_TRY(cudaMemcpy(v.data(), P.d_p1, sizeof(P1Desc) * v.size(), cudaMemcpyDeviceToHost));
  std::stable_sort(v.begin(), v.end(), [](const P1Desc& a, const P1Desc& b) {
    return a.seg0 != b.seg0 ? a.seg0 < b.seg0 : a.len < b.len;
  });
  std::vector<uint32_t> g;
  for (size_t i = 0; i < v.size();) {
    g.push_back((uint32_t)i);
    size_t j = i + 1;
    while (j < v.size() && j - i < (size_t)G1 && v[j].seg0 == v[i].seg0 && v[j].len == v[i].len) ++j;
    i = j;
  }
  P.ng1 = (int64_t)g.size();
  g.push_back((uint32_t)v.size());
  // segment tasks: runs of equal (seg0, len), cut every S1_LEAVES leaves
  std::vector<uint32_t> tk;
  uint32_t maxlen = 0;
  for (size_t i = 0; i < v.size();) {
    size_t j = i + 1;
    while (j < v.size() && j - i < (size_t)S1_LEAVES && v[j].seg0 == v[i].seg0 && v[j].len == v[i].len) ++j;
    tk.push_back((uint32_t)i);
    maxlen = std::max(maxlen, v[i].len);
    i = j;
  }
  P.nt1 = (int64_t)tk.size();
  P.maxlen1 = maxlen;
  tk.push_back((uint32_t)v.size());
  HM_CUDA_TRY(cudaMalloc(&P.d_t1s, sizeof(uint32_t) * tk.size()));
  HM_CUDA_TRY(h2d_sync(P.d_t1s, tk.data(), sizeof(uint32_t) * tk.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_p1s, sizeof(P1Desc) * v.size()));
  HM_CUDA_TRY(h2d_sync(P.d_p1s, v.data(), sizeof(P1Desc) * v.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_g1s, sizeof(uint32_t) * g.size()));
  HM_CUDA_TRY(h2d_sync(P.d_g1s, g.data(), sizeof(uint32_t) * g.size()));
  return HM_OK;
}

template <typename T, int CB>
int launch_multi(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st,
                 bool dense_only = false) {
  using TD = typename std::conditional<std::is_same<T, double>::value, double, float>::type;
  MvPlan& P = trans ? h->bwd : h->fwd;
  if (!dense_only) HM_TRY(ensure_sorted_p1(P));
  const int ld = (int)pad_to(ncols, CB);
  const int ncb = ld / CB;
  const size_t xr_bytes = sizeof(double) * (size_t)(h->n + 2) * ld;
  // the dense-only pass needs no phase-1 results
  const size_t zr_bytes = dense_only ? 0 : sizeof(double) * (size_t)std::max<int64_t>(h->zlen, 1) * ld;
  if (h->xm_bytes < xr_bytes + zr_bytes) {
    if (h->d_xm) cudaFree(h->d_xm);
    h->d_xm = nullptr;
    h->xm_bytes = 0;
    HM_CUDA_TRY(cudaMalloc(&h->d_xm, xr_bytes + zr_bytes));
    h->xm_bytes = xr_bytes + zr_bytes;
  }
  double* xr = (double*)h->d_xm;
  double* zr = (double*)((char*)h->d_xm + xr_bytes);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  {
    const int64_t tot = (h->n + 2) * ld;
    const unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)nsm * 16);
    mvm_xr_kernel<<<g, 256, 0, st>>>(d_x, h->n, h->n, (int)ncols, xr, ld);
  }
  const int64_t nblk = (int64_t)P.nwin * 2 * ncb;
  if (nblk > (int64_t)INT32_MAX) return fail(HM_ERR_UNSUPPORTED, "too many phase-2 blocks");
  if (dense_only) {
    HM_TRY(split_p2(P));
    const int64_t ntile = (h->n + 127) / 128;
    const int64_t blocks = ntile * ncb;
    if (blocks > (int64_t)INT32_MAX) return fail(HM_ERR_UNSUPPORTED, "too many dense-pass blocks");
    mvm_dense_kernel<TD, CB><<<(unsigned)blocks, 128, 0, st>>>(P.d_wind, P.d_p2d, (const TD*)h->d_dense, xr, ld, ncb,
                                                             ntile, d_y, h->n, (int)ncols);
    HM_CUDA_TRY(cudaGetLastError());
    return HM_OK;
  }
  const size_t seg_smem = sizeof(double) * (size_t)P.maxlen1 * (CB + 2);
  if (P.np1 > 0 && seg_smem <= 96 * 1024 && P.nt1 * ncb <= (int64_t)INT32_MAX) {
    HM_CUDA_TRY(smem_attr((const void*)mvm_phase1_seg_kernel<T, CB>, 96 * 1024));
    mvm_phase1_seg_kernel<T, CB><<<(unsigned)(P.nt1 * ncb), 256, seg_smem, st>>>(P.d_p1s, P.d_t1s, P.nt1,
                                                                               (const T*)h->d_rk, xr, ld, ncb, zr);
  } else if (P.np1 > 0) {                        // segments too long to stage: grouped leaves
    const int64_t warps = P.ng1 * ncb;
    const int64_t blocks = std::min<int64_t>((warps + 7) / 8, (int64_t)nsm * 8);
    mvm_phase1_kernel<T, CB><<<(unsigned)blocks, 256, 0, st>>>(P.d_p1s, P.d_g1s, P.ng1, (const T*)h->d_rk, xr, ld,
                                                              ncb, zr);
  }
  mvm_phase2_kernel<T, TD, CB><<<(unsigned)nblk, M2_THREADS, 0, st>>>(
      P.d_win, P.d_p2, (const T*)h->d_rk, (const TD*)h->d_dense, zr, xr, ld, ncb, d_y, h->n, (int)ncols);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

template <typename T>
int multi_t(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st,
            bool dense_only = false) {
  if (ncols <= 4) return launch_multi<T, 4>(h, d_x, d_y, ncols, trans, st, dense_only);
  if (ncols <= 8) return launch_multi<T, 8>(h, d_x, d_y, ncols, trans, st, dense_only);
  return launch_multi<T, 16>(h, d_x, d_y, ncols, trans, st, dense_only);
}

}  // namespace

// FP64 factors (no tensor-core kind for FP64), simt, or factors beyond the
// tensor-core path's range (2^100): the CUDA-core block kernels for the whole
// product.  FP32/BF16 factors: the dense leaves on the CUDA cores (they write
// every row of Y), then the low-rank part on the tensor cores (added into Y).
int matvec_multi_device(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st,
                        bool simt) {
  if (ncols <= 0) return HM_OK;
  if ((h->n + 2) * pad_to(ncols, 16) > (int64_t)1 << 40) return fail(HM_ERR_UNSUPPORTED, "right-hand side block too large");
  switch (h->storage) {
    case HM_F64: return multi_t<double>(h, d_x, d_y, ncols, trans, st);
    case HM_F32: {
      bool tc = false;
      if (!simt) HM_TRY(tc_prepare(h, trans, &tc));
      if (!tc) return multi_t<float>(h, d_x, d_y, ncols, trans, st);
      HM_TRY(multi_t<float>(h, d_x, d_y, ncols, trans, st, true));
      return matvec_multi_tc(h, d_x, d_y, ncols, trans, st);
    }
    default: {
      bool tc = false;
      if (!simt) HM_TRY(tc_prepare(h, trans, &tc));
      if (!tc) return multi_t<__nv_bfloat16>(h, d_x, d_y, ncols, trans, st);
      HM_TRY(multi_t<__nv_bfloat16>(h, d_x, d_y, ncols, trans, st, true));
      return matvec_multi_tc(h, d_x, d_y, ncols, trans, st);
    }
  }
}

}  // namespace hm
