// H-matvec on sm_100a (K4): y = H x and y = H' x over the flattened leaf
// list, the device form of hmat_matvec! (src/harithm.jl:340-354) and
// transpose_hmat_mat_mul (src/harithm.jl:243-260).
//
// Phase 1: one warp per low-rank leaf streams its F1 factor (B for H*x)
//          with 16-byte loads and writes z = F1' x_seg (k values) to z[].
// Phase 2: one CTA per window of 1024 output rows; each lane owns 4 rows and
//          accumulates sum_r F2[:,r] z_r over the low-rank leaves and C x_seg
//          over the dense leaves that cover its rows, and stores y.
// FP64 factors are accumulated in FP64.  FP32 and BF16 factors are
// multiplied and summed in FP32 over the few vectors (phase 1) or entries
// (phase 2) a lane has in flight, and those FP32 partial sums are added in
// FP64: one conversion per group instead of one per element.
// The input is staged as 16-byte aligned shifted copies so that every
// x-segment load in phase 1 is a vector load, whatever the segment start.
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <algorithm>
#include <type_traits>
#include <cstring>

namespace hm {

// ---------------------------------------------------------------------------
// storage traits: 16-byte vector of factors + matching x vector
// ---------------------------------------------------------------------------
template <typename T> struct MvT;
template <> struct MvT<double> {
  static constexpr int VW = 2, U = 4, NR = 2;       // NR: factor columns a warp streams together
  using X = double;
  using R = double2;
  struct XV { double2 a; };
  __device__ static R ld(const double* p) { return __ldcs(reinterpret_cast<const double2*>(p)); }
  __device__ static XV ldx(const double* p) { return XV{__ldg(reinterpret_cast<const double2*>(p))}; }
  __device__ static double dot(const R& f, const XV& x, double s) {
    s = fma(f.x, x.a.x, s);
    return fma(f.y, x.a.y, s);
  }
};
template <> struct MvT<float> {
  static constexpr int VW = 4, U = 4, NR = 2;
  using X = float;
  using R = float4;
  struct XV { float4 a; };
  __device__ static R ld(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
  __device__ static XV ldx(const float* p) { return XV{__ldg(reinterpret_cast<const float4*>(p))}; }
  // FP32 partial sum of one vector (the caller folds it into its FP64 sum)
  __device__ static float dotf(const R& f, const XV& x, float s) {
    s = fmaf(f.x, x.a.x, s);
    s = fmaf(f.y, x.a.y, s);
    s = fmaf(f.z, x.a.z, s);
    return fmaf(f.w, x.a.w, s);
  }
};
__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
template <> struct MvT<__nv_bfloat16> {
  static constexpr int VW = 8, U = 2, NR = 4;       // a BF16 vector is half the bytes: twice the columns
  using X = float;
  using R = uint4;
  struct XV { float4 a, b; };
  __device__ static R ld(const __nv_bfloat16* p) { return __ldcs(reinterpret_cast<const uint4*>(p)); }
  __device__ static XV ldx(const float* p) {
    return XV{__ldg(reinterpret_cast<const float4*>(p)), __ldg(reinterpret_cast<const float4*>(p) + 1)};
  }
  // BF16 -> FP32 is a shift of the bits; FP32 partial sum of one vector
  __device__ static float dotf(const R& f, const XV& x, float s) {
    s = fmaf(bf_lo(f.x), x.a.x, s);
    s = fmaf(bf_hi(f.x), x.a.y, s);
    s = fmaf(bf_lo(f.y), x.a.z, s);
    s = fmaf(bf_hi(f.y), x.a.w, s);
    s = fmaf(bf_lo(f.z), x.b.x, s);
    s = fmaf(bf_hi(f.z), x.b.y, s);
    s = fmaf(bf_lo(f.w), x.b.z, s);
    return fmaf(bf_hi(f.w), x.b.w, s);
  }
};

// shifted copies: copy q holds x[t - q] at index t (zero outside [q, n+q))
template <typename TX>
__global__ void xcopy_kernel(const double* __restrict__ x, int64_t n, TX* __restrict__ xs, int64_t stride, int ncopy) {
  const int64_t tot = stride * ncopy;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = e / stride, t = e % stride;
    const int64_t s = t - q;
    xs[e] = (s >= 0 && s < n) ? (TX)x[s] : (TX)0;
  }
}

// ---------------------------------------------------------------------------
// phase 1: z = F1' x_seg, one warp per low-rank leaf
// ---------------------------------------------------------------------------
#ifndef HM_P1_MINB
#define HM_P1_MINB 1
#endif
template <typename T>
__global__ void __launch_bounds__(256, HM_P1_MINB) mv_phase1_kernel(const P1Desc* __restrict__ d, int64_t nd,
                                                        const T* __restrict__ pool,
                                                        const typename MvT<T>::X* __restrict__ xs,
                                                        int64_t xs_stride, double* __restrict__ z) {
  using Tr = MvT<T>;
  using TX = typename Tr::X;
  constexpr int VW = Tr::VW, U = Tr::U, NR = Tr::NR;
  constexpr int XA = 16 / (int)sizeof(TX);
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = gw; b < nd; b += nw) {
    const P1Desc D = d[b];
    const int q = (XA - (int)(D.seg0 % XA)) % XA;
    const TX* xb = xs + q * xs_stride + D.seg0 + q;
    const int nvec = (int)(D.stride / VW);
    const T* F = pool + D.off;
    for (int r = 0; r < D.k; r += NR) {
      // NR columns r .. r + NR - 1 (those past the rank point at column r and are
      // neither read, beyond the first two, nor written)
      const T* fc[NR];
#pragma unroll
      for (int j = 0; j < NR; ++j) fc[j] = F + (int64_t)(r + j < D.k ? r + j : r) * D.stride;
      double sc[NR];
#pragma unroll
      for (int j = 0; j < NR; ++j) sc[j] = 0.0;
      for (int v0 = lane; v0 < nvec; v0 += 32 * U) {
        typename Tr::R a[NR][U];
        typename Tr::XV xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int v = v0 + 32 * u;
          if (v < nvec) {
#pragma unroll
            for (int j = 0; j < NR; ++j)
              if (j < 2 || r + j < D.k) a[j][u] = Tr::ld(fc[j] + (int64_t)v * VW);   // no reads past the rank
            xv[u] = Tr::ldx(xb + (int64_t)v * VW);
          }
        }
        if constexpr (std::is_same<T, double>::value) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (v0 + 32 * u < nvec) {
#pragma unroll
              for (int j = 0; j < NR; ++j) sc[j] = Tr::dot(a[j][u], xv[u], sc[j]);
            }
          }
        } else {
          // FP32 products and partial sums over the U vectors in flight,
          // folded into the FP64 sums once per group
          float fp[NR];
#pragma unroll
          for (int j = 0; j < NR; ++j) fp[j] = 0.f;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (v0 + 32 * u < nvec) {
#pragma unroll
              for (int j = 0; j < NR; ++j) fp[j] = Tr::dotf(a[j][u], xv[u], fp[j]);
            }
          }
#pragma unroll
          for (int j = 0; j < NR; ++j) sc[j] += (double)fp[j];
        }
      }
#pragma unroll
      for (int j = 0; j < NR; ++j) sc[j] = warp_sum(sc[j]);
      if (lane == 0) {
#pragma unroll
        for (int j = 0; j < NR; ++j)
          if (r + j < D.k) z[D.zoff + r + j] = sc[j];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// phase 2: y(window) = sum over leaves covering the window.  Each lane owns 4
// consecutive output rows; when a leaf starts on a 4-row boundary of the
// window its 4 values come in one vector load (columns are padded to a
// multiple of 4 elements and 16 bytes, padding rows hold zeros).
// ---------------------------------------------------------------------------
constexpr int P2_NB = 32;      // descriptors staged per round
// SPLIT (2, 4 or 8 CTAs per 1024-row window) is chosen per handle by the
// autotuner (hm_autotune); 4 until then
template <int SPLIT> struct P2Shape {
  static constexpr int CROWS = MV_WROWS / SPLIT;   // rows of one CTA
  static constexpr int WARPS = CROWS / 128;        // 32 lanes x 4 rows a warp
  static constexpr int EMAX = 1024 / SPLIT;        // expanded (leaf, column) entries per sub-round
};
constexpr uint64_t P2_DENSE_FLAG = 1ull << 63;

// 4 consecutive rows of one column are loaded as raw words and converted to
// FP64 only when they are multiplied: a conversion next to its load would
// make the warp wait for that load before issuing the next entry's loads.
template <typename T> struct Row4;
template <> struct Row4<double> {               // dense leaves: double as well
  static constexpr int U = 4;
  struct Raw { double2 a, b; };
  __device__ static Raw zero() { return Raw{make_double2(0.0, 0.0), make_double2(0.0, 0.0)}; }
  __device__ static Raw ld(const double* p) {
    return Raw{__ldcs(reinterpret_cast<const double2*>(p)), __ldcs(reinterpret_cast<const double2*>(p) + 1)};
  }
  __device__ static Raw ldd(const double* p) { return ld(p); }
  __device__ static void put(Raw& r, int q, double v) {
    if (q == 0) r.a.x = v; else if (q == 1) r.a.y = v; else if (q == 2) r.b.x = v; else r.b.y = v;
  }
  __device__ static void cvt(const Raw& r, bool, double (&v)[4]) { v[0] = r.a.x; v[1] = r.a.y; v[2] = r.b.x; v[3] = r.b.y; }
};
template <> struct Row4<float> {                // dense leaves: float
  static constexpr int U = 8;
  using Raw = float4;
  __device__ static Raw zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  __device__ static Raw ld(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
  __device__ static Raw ldd(const float* p) { return ld(p); }
  __device__ static void put(Raw& r, int q, float v) {
    if (q == 0) r.x = v; else if (q == 1) r.y = v; else if (q == 2) r.z = v; else r.w = v;
  }
  __device__ static void cvt(const Raw& r, bool, double (&v)[4]) { v[0] = r.x; v[1] = r.y; v[2] = r.z; v[3] = r.w; }
  __device__ static void cvtf(const Raw& r, bool, float (&v)[4]) { v[0] = r.x; v[1] = r.y; v[2] = r.z; v[3] = r.w; }
};
template <> struct Row4<__nv_bfloat16> {        // dense leaves: float (raw float bits)
  static constexpr int U = 8;
  using Raw = uint4;
  __device__ static Raw zero() { return make_uint4(0u, 0u, 0u, 0u); }
  __device__ static Raw ld(const __nv_bfloat16* p) {
    const uint2 a = __ldcs(reinterpret_cast<const uint2*>(p));
    return make_uint4(a.x, a.y, 0u, 0u);
  }
  __device__ static Raw ldd(const float* p) {
    return __ldcs(reinterpret_cast<const uint4*>(p));
  }
  __device__ static void put(Raw& r, int q, float v) {
    const uint32_t b = __float_as_uint(v);
    if (q == 0) r.x = b; else if (q == 1) r.y = b; else if (q == 2) r.z = b; else r.w = b;
  }
  __device__ static void put(Raw& r, int q, __nv_bfloat16 v) {
    const uint32_t b = (uint32_t)__bfloat16_as_ushort(v);
    if (q == 0) r.x = (r.x & 0xffff0000u) | b;
    else if (q == 1) r.x = (r.x & 0x0000ffffu) | (b << 16);
    else if (q == 2) r.y = (r.y & 0xffff0000u) | b;
    else r.y = (r.y & 0x0000ffffu) | (b << 16);
  }
  __device__ static void cvt(const Raw& r, bool dense, double (&v)[4]) {
    if (dense) {
      v[0] = __uint_as_float(r.x); v[1] = __uint_as_float(r.y);
      v[2] = __uint_as_float(r.z); v[3] = __uint_as_float(r.w);
    } else {
      v[0] = bf_lo(r.x); v[1] = bf_hi(r.x); v[2] = bf_lo(r.y); v[3] = bf_hi(r.y);
    }
  }
  __device__ static void cvtf(const Raw& r, bool dense, float (&v)[4]) {
    if (dense) {
      v[0] = __uint_as_float(r.x); v[1] = __uint_as_float(r.y);
      v[2] = __uint_as_float(r.z); v[3] = __uint_as_float(r.w);
    } else {
      v[0] = bf_lo(r.x); v[1] = bf_hi(r.x); v[2] = bf_lo(r.y); v[3] = bf_hi(r.y);
    }
  }
};

template <typename T, typename TD, int SPLIT>
__global__ void __launch_bounds__(P2Shape<SPLIT>::WARPS * 32) mv_phase2_kernel(const MvWin* __restrict__ win,
                                                                  const P2Desc* __restrict__ d,
                                                                  const T* __restrict__ rk, const TD* __restrict__ dn,
                                                                  const double* __restrict__ z,
                                                                  const double* __restrict__ x,
                                                                  double* __restrict__ y) {
  constexpr int U = Row4<T>::U;
  constexpr int P2_SPLIT = SPLIT, P2_CROWS = P2Shape<SPLIT>::CROWS, P2_EMAX = P2Shape<SPLIT>::EMAX;
  __shared__ P2Desc sd[P2_NB];
  __shared__ int spre[P2_NB + 1];
  __shared__ uint64_t e_off[P2_EMAX];
  __shared__ int32_t e_ro[P2_EMAX];
  __shared__ uint32_t e_m[P2_EMAX];
  __shared__ uint32_t e_rs[P2_EMAX];
  __shared__ double e_z[P2_EMAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const MvWin W = win[blockIdx.x / P2_SPLIT];
  const int h0 = (int)(blockIdx.x % P2_SPLIT) * P2_CROWS;   // this CTA's rows of the window
  const int base = h0 + 4 * (warp * 32 + lane);  // first of this lane's rows in the window
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t b0 = W.begin; b0 < W.end; b0 += P2_NB) {
    const int nb = (int)min((uint32_t)P2_NB, W.end - b0);
    __syncthreads();
    if (warp == 0) {
      int cnt = 0;
      if (lane < nb) {
        sd[lane] = d[b0 + lane];
        // only leaves with rows in this CTA's part of the window are expanded
        const int r0 = sd[lane].row_off, r1 = r0 + (int)sd[lane].m;
        cnt = (r1 > h0 && r0 < h0 + P2_CROWS) ? (int)sd[lane].cnt : 0;
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      spre[lane + 1] = incl;
      if (lane == 0) spre[0] = 0;
    }
    __syncthreads();
    const int total = spre[nb];
    for (int e0 = 0; e0 < total; e0 += P2_EMAX) {
      const int ne = min(P2_EMAX, total - e0);
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
        if (D.type == P2_RK) {
          e_off[e] = D.off + (uint64_t)c * D.ld;
          e_rs[e] = 1;
          e_z[e] = z[D.aux + c];
        } else if (D.type == P2_DENSE) {
          e_off[e] = (D.off + (uint64_t)c * D.ld) | P2_DENSE_FLAG;
          e_rs[e] = 1;
          e_z[e] = x[D.aux + c];
        } else {
          e_off[e] = (D.off + (uint64_t)c) | P2_DENSE_FLAG;
          e_rs[e] = D.ld;
          e_z[e] = x[D.aux + c];
        }
        e_ro[e] = D.row_off;
        e_m[e] = D.m;
      }
      __syncthreads();
      for (int e = 0; e < ne; e += U) {
        typename Row4<T>::Raw raw[U];
        double zz[U];
        bool isd[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          raw[u] = Row4<T>::zero();
          zz[u] = 0.0;
          isd[u] = false;
          const int ee = e + u;
          if (ee < ne) {
            const int ro = e_ro[ee];
            const int mm = (int)e_m[ee];
            const uint64_t o = e_off[ee];
            const uint32_t rs = e_rs[ee];
            const int lr = base - ro;
            const bool dense = (o & P2_DENSE_FLAG) != 0;
            zz[u] = e_z[ee];
            isd[u] = dense;
            if (((ro & 3) == 0) && rs == 1) {
              if (lr >= 0 && lr < mm) {
                if (dense) raw[u] = Row4<T>::ldd(dn + (o & ~P2_DENSE_FLAG) + lr);
                else raw[u] = Row4<T>::ld(rk + o + lr);
              }
            } else {
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const int r = lr + q;
                if (r >= 0 && r < mm) {
                  if (dense) Row4<T>::put(raw[u], q, __ldg(dn + (o & ~P2_DENSE_FLAG) + (uint64_t)r * rs));
                  else Row4<T>::put(raw[u], q, rk[o + (uint64_t)r]);
                }
              }
            }
          }
        }
        if constexpr (std::is_same<T, double>::value) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            double v[4];
            Row4<T>::cvt(raw[u], isd[u], v);
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fma(v[q], zz[u], acc[q]);
          }
        } else {
          // FP32 products and partial sums over the U entries in flight,
          // folded into the FP64 row sums once per group
          float part[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int u = 0; u < U; ++u) {
            float v[4];
            Row4<T>::cvtf(raw[u], isd[u], v);
            const float zf = (float)zz[u];
#pragma unroll
            for (int q = 0; q < 4; ++q) part[q] = fmaf(v[q], zf, part[q]);
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[q] += (double)part[q];
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (base + q < (int)W.nrows) y[W.row0 + base + q] = acc[q];
}

// ---------------------------------------------------------------------------
// phase 2 by tree clusters: one warp per unit (at most 128 rows of one output
// cluster and all the leaves of that cluster), R = 1, 2 or 4 consecutive rows
// a lane by the unit's size.  Every entry starts on the unit's first row, so a
// lane's R values come in one aligned load (columns are padded to a multiple
// of 4 elements and 16 bytes; values past the unit's last row are loaded but
// never stored).  The result is added into y.
// ---------------------------------------------------------------------------
constexpr int CL_E = 64;       // expanded (leaf, column) entries per warp round
constexpr int CL_WARPS = 8;

template <int R> __device__ __forceinline__ void cl_ld(const double* p, double (&v)[R]) {
  if constexpr (R == 1) {
    v[0] = __ldcs(p);
  } else if constexpr (R == 2) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    v[0] = a.x; v[1] = a.y;
  } else {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}
template <int R> __device__ __forceinline__ void cl_ld(const float* p, float (&v)[R]) {
  if constexpr (R == 1) {
    v[0] = __ldcs(p);
  } else if constexpr (R == 2) {
    const float2 a = __ldcs(reinterpret_cast<const float2*>(p));
    v[0] = a.x; v[1] = a.y;
  } else {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
}

struct ClSmem {                 // one warp's staging
  P2Desc sd[32];
  int spre[33];
  uint32_t e_rs[CL_E];
  uint64_t e_off[CL_E];
  double e_z[CL_E];
};

template <typename T, int R>
__device__ __forceinline__ void cl_unit(const MvWin& W, const P2Desc* __restrict__ d, const T* __restrict__ rk,
                                        const T* __restrict__ dn, const double* __restrict__ z,
                                        const double* __restrict__ x, double* __restrict__ y, ClSmem& sm, int lane) {
  constexpr int U0 = (sizeof(T) == 8 ? 16 : 32) / R;   // 128 bytes in flight a lane, 8 entries at most
  constexpr int U = U0 > 8 ? 8 : U0;
  const int base = R * lane;
  const int nrows = (int)W.nrows;
  const bool act = base < nrows;
  double acc[R];
#pragma unroll
  for (int q = 0; q < R; ++q) acc[q] = 0.0;
  for (uint32_t b0 = W.begin; b0 < W.end; b0 += 32) {
    const int nb = (int)min(32u, W.end - b0);
    __syncwarp();
    int cnt = 0;
    if (lane < nb) {
      sm.sd[lane] = d[b0 + lane];
      cnt = (int)sm.sd[lane].cnt;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    sm.spre[lane + 1] = incl;
    if (lane == 0) sm.spre[0] = 0;
    __syncwarp();
    const int total = sm.spre[nb];
    for (int e0 = 0; e0 < total; e0 += CL_E) {
      const int ne = min(CL_E, total - e0);
      __syncwarp();
      for (int e = lane; e < ne; e += 32) {
        const int ge = e0 + e;
        int lo = 0, hi = nb - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sm.spre[mid] <= ge) lo = mid; else hi = mid - 1;
        }
        const P2Desc& D = sm.sd[lo];
        const int c = ge - sm.spre[lo];
        if (D.type == P2_RK) {
          sm.e_off[e] = D.off + (uint64_t)c * D.ld;
          sm.e_rs[e] = 1;
          sm.e_z[e] = z[D.aux + c];
        } else if (D.type == P2_DENSE) {
          sm.e_off[e] = (D.off + (uint64_t)c * D.ld) | P2_DENSE_FLAG;
          sm.e_rs[e] = 1;
          sm.e_z[e] = x[D.aux + c];
        } else {
          sm.e_off[e] = (D.off + (uint64_t)c) | P2_DENSE_FLAG;
          sm.e_rs[e] = D.ld;
          sm.e_z[e] = x[D.aux + c];
        }
      }
      __syncwarp();
      if (!act) continue;
      for (int e = 0; e < ne; e += U) {
        T v[U][R];
        T zz[U];                               // the FP32 path multiplies by z rounded to FP32
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
          for (int q = 0; q < R; ++q) v[u][q] = T(0);
          zz[u] = T(0);
          const int ee = e + u;
          if (ee < ne) {
            const uint64_t o = sm.e_off[ee];
            const uint32_t rs = sm.e_rs[ee];
            const T* p = (o & P2_DENSE_FLAG) ? dn + (o & ~P2_DENSE_FLAG) : rk + o;
            zz[u] = (T)sm.e_z[ee];
            if (rs == 1) {
              cl_ld<R>(p + base, v[u]);
            } else {
#pragma unroll
              for (int q = 0; q < R; ++q)
                if (base + q < nrows) v[u][q] = __ldg(p + (uint64_t)(base + q) * rs);
            }
          }
        }
        if constexpr (std::is_same<T, double>::value) {
#pragma unroll
          for (int u = 0; u < U; ++u)
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] = fma(v[u][q], zz[u], acc[q]);
        } else {
          // FP32 products and partial sums over the U entries in flight,
          // folded into the FP64 row sums once per group
          float part[R];
#pragma unroll
          for (int q = 0; q < R; ++q) part[q] = 0.f;
#pragma unroll
          for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int q = 0; q < R; ++q) part[q] = fmaf(v[u][q], zz[u], part[q]);
          }
#pragma unroll
          for (int q = 0; q < R; ++q) acc[q] += (double)part[q];
        }
      }
    }
  }
  if (act) {
#pragma unroll
    for (int q = 0; q < R; ++q)
      if (base + q < nrows) y[W.row0 + base + q] += acc[q];
  }
}

template <typename T>
__global__ void __launch_bounds__(CL_WARPS * 32, 3) mv_phase2c_kernel(const MvWin* __restrict__ units, int nu,
                                                                   const P2Desc* __restrict__ d,
                                                                   const T* __restrict__ rk, const T* __restrict__ dn,
                                                                   const double* __restrict__ z,
                                                                   const double* __restrict__ x,
                                                                   double* __restrict__ y) {
  __shared__ ClSmem sm[CL_WARPS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * CL_WARPS + warp;
  if (u >= nu) return;                         // warps are independent: no block barrier follows
  const MvWin W = units[u];
  if (W.nrows > 64) cl_unit<T, 4>(W, d, rk, dn, z, x, y, sm[warp], lane);
  else if (W.nrows > 32) cl_unit<T, 2>(W, d, rk, dn, z, x, y, sm[warp], lane);
  else cl_unit<T, 1>(W, d, rk, dn, z, x, y, sm[warp], lane);
}

// ---------------------------------------------------------------------------
// plan construction
// ---------------------------------------------------------------------------
void free_mv_plan(MvPlan& p) {
  if (p.d_p1) cudaFree(p.d_p1);
  if (p.d_p1s) cudaFree(p.d_p1s);
  if (p.d_g1s) cudaFree(p.d_g1s);
  if (p.d_t1s) cudaFree(p.d_t1s);
  if (p.d_p2) cudaFree(p.d_p2);
  if (p.d_win) cudaFree(p.d_win);
  if (p.d_p2d) cudaFree(p.d_p2d);
  if (p.d_wind) cudaFree(p.d_wind);
  if (p.d_p2r) cudaFree(p.d_p2r);
  if (p.d_winr) cudaFree(p.d_winr);
  if (p.d_cd) cudaFree(p.d_cd);
  if (p.d_cu) cudaFree(p.d_cu);
  p = MvPlan{};
}

// Phase 2 by tree clusters (MvPlan::cl_*).  The leaves are grouped by their
// output cluster (the row cluster for H*x, the column cluster for H'*x) and the
// cluster is cut into 128-row units, so every entry of a unit covers all the
// unit's rows from its first: each lane's rows come in one aligned vector load
// wherever the cluster boundaries fall.  Units of one tree level are disjoint;
// the levels run one launch after another and add into y.  z offsets follow
// the pool order of the low-rank leaves, as in build_mv_descriptors.
constexpr int CL_ROWS = 128;                   // rows of a unit at most (32 lanes x 4 rows)
static int build_cluster_plan(hm_handle* h, int trans, MvPlan& P) {
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  std::vector<int64_t> rk;                       // low-rank leaves in pool order
  for (size_t i = 0; i < h->leaves.size(); ++i)
    if (h->leaves[i].type == T_RK) rk.push_back((int64_t)i);
  std::stable_sort(rk.begin(), rk.end(), [&](int64_t a, int64_t b) { return h->leaves[a].off < h->leaves[b].off; });
  std::vector<uint32_t> zoff(h->leaves.size(), 0);
  int64_t z = 0;
  for (int64_t li : rk) { zoff[li] = (uint32_t)z; z += h->leaves[li].k; }
  const int64_t ncl = (int64_t)h->cl_s.size();
  std::vector<std::vector<int64_t>> by(ncl);     // leaves by output cluster
  int32_t maxdepth = 0;
  for (size_t i = 0; i < h->leaves.size(); ++i) {
    const Leaf& L = h->leaves[i];
    if (L.type == T_RK && L.k == 0) continue;
    const int32_t c = trans ? L.t : L.s;
    by[c].push_back((int64_t)i);
    maxdepth = std::max(maxdepth, h->cl_depth[c]);
  }
  std::vector<std::vector<int64_t>> lev(maxdepth + 1);   // clusters by tree level, in row order
  for (int64_t c = 0; c < ncl; ++c)
    if (!by[c].empty()) lev[h->cl_depth[c]].push_back(c);
  for (auto& v : lev)
    std::sort(v.begin(), v.end(), [&](int64_t a, int64_t b) { return h->cl_s[a] < h->cl_s[b]; });
  std::vector<P2Desc> d;
  std::vector<MvWin> w;
  P.cl_level.assign(1, 0);
  for (int32_t l = maxdepth; l >= 0; --l) {
    for (int64_t c : lev[l]) {
      const int64_t c0 = h->cl_s[c], m = h->cl_e[c] - h->cl_s[c];
      for (int64_t r0 = 0; r0 < m; r0 += CL_ROWS) {
        MvWin W{};
        W.row0 = (uint32_t)(c0 + r0);
        W.nrows = (uint32_t)std::min<int64_t>(CL_ROWS, m - r0);
        W.begin = (uint32_t)d.size();
        for (int64_t li : by[c]) {
          const Leaf& L = h->leaves[li];
          const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
          P2Desc D{};
          D.m = W.nrows;
          if (L.type == T_RK) {
            D.type = P2_RK;
            D.off = (trans ? L.off : L.off + npad * L.k) + r0;
            D.ld = (uint32_t)(trans ? npad : mpad);
            D.aux = zoff[li];
            D.cnt = (uint32_t)L.k;
          } else {
            const int64_t ldc = col_pad(L.m, deb);
            D.type = trans ? P2_DENSE_T : P2_DENSE;
            D.off = L.off + (trans ? r0 * ldc : r0);
            D.ld = (uint32_t)ldc;
            D.aux = (uint32_t)(trans ? L.row0 : L.col0);
            D.cnt = (uint32_t)(trans ? L.m : L.n);
          }
          d.push_back(D);
        }
        W.end = (uint32_t)d.size();
        w.push_back(W);
      }
    }
    P.cl_level.push_back((int32_t)w.size());
  }
  if (d.size() > (size_t)UINT32_MAX || w.size() > (size_t)INT32_MAX)
    return fail(HM_ERR_UNSUPPORTED, "too many cluster descriptors");
  if (d.empty()) d.push_back(P2Desc{});
  if (w.empty()) w.push_back(MvWin{});
  HM_CUDA_TRY(cudaMalloc(&P.d_cd, sizeof(P2Desc) * d.size()));
  HM_CUDA_TRY(h2d_sync(P.d_cd, d.data(), sizeof(P2Desc) * d.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_cu, sizeof(MvWin) * w.size()));
  HM_CUDA_TRY(h2d_sync(P.d_cu, w.data(), sizeof(MvWin) * w.size()));
  P.cl_built = true;
  return HM_OK;
}

int build_mv_descriptors(hm_handle* h, const std::vector<int64_t>& order, int trans) {
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  const int64_t n = h->n;
  MvPlan& P = trans ? h->bwd : h->fwd;
  free_mv_plan(P);
  if (n > (int64_t)UINT32_MAX / 2) return fail(HM_ERR_UNSUPPORTED, "n above 2^31");
  // z slots in pool order (shared by both directions)
  std::vector<uint32_t> zoff(h->leaves.size(), 0);
  int64_t z = 0;
  for (int64_t li : order)
    if (h->leaves[li].type == T_RK) { zoff[li] = (uint32_t)z; z += h->leaves[li].k; }
  if (z > (int64_t)UINT32_MAX) return fail(HM_ERR_UNSUPPORTED, "too many low-rank terms");
  if (!trans) {
    if (h->d_z) cudaFree(h->d_z);
    h->d_z = nullptr;
    h->zlen = z;
    if (z) HM_CUDA_TRY(cudaMalloc(&h->d_z, sizeof(double) * z));
  }
  std::vector<P1Desc> p1;
  p1.reserve(order.size());
  for (int64_t li : order) {
    const Leaf& L = h->leaves[li];
    if (L.type != T_RK || L.k == 0) continue;
    P1Desc D{};
    const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
    if (!trans) { D.off = L.off; D.seg0 = (uint32_t)L.col0; D.len = L.n; D.stride = (uint32_t)npad; }
    else { D.off = L.off + npad * L.k; D.seg0 = (uint32_t)L.row0; D.len = L.m; D.stride = (uint32_t)mpad; }
    D.zoff = zoff[li];
    D.k = (uint16_t)L.k;
    p1.push_back(D);
  }
  const int64_t nwin = (n + MV_WROWS - 1) / MV_WROWS;
  std::vector<std::vector<P2Desc>> per(nwin);
  for (int64_t li : order) {
    const Leaf& L = h->leaves[li];
    if (L.type == T_RK && L.k == 0) continue;
    const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
    const int64_t o0 = trans ? L.col0 : L.row0;
    const int64_t oe = o0 + (trans ? L.n : L.m);
    P2Desc D{};
    D.m = (uint32_t)(oe - o0);
    if (L.type == T_RK) {
      D.type = P2_RK;
      D.off = trans ? L.off : L.off + npad * L.k;
      D.ld = (uint32_t)(trans ? npad : mpad);
      D.aux = zoff[li];
      D.cnt = (uint32_t)L.k;
    } else {
      const int64_t ldc = col_pad(L.m, deb);
      D.type = trans ? P2_DENSE_T : P2_DENSE;
      D.off = L.off;
      D.ld = (uint32_t)ldc;
      D.aux = (uint32_t)(trans ? L.row0 : L.col0);
      D.cnt = (uint32_t)(trans ? L.m : L.n);
    }
    for (int64_t w = o0 / MV_WROWS; w * MV_WROWS < oe; ++w) {
      P2Desc E = D;
      E.row_off = (int32_t)(o0 - w * MV_WROWS);
      per[w].push_back(E);
    }
  }
  std::vector<P2Desc> p2;
  std::vector<MvWin> wins(nwin);
  for (int64_t w = 0; w < nwin; ++w) {
    wins[w].row0 = (uint32_t)(w * MV_WROWS);
    wins[w].nrows = (uint32_t)std::min<int64_t>(MV_WROWS, n - w * MV_WROWS);
    wins[w].begin = (uint32_t)p2.size();
    p2.insert(p2.end(), per[w].begin(), per[w].end());
    wins[w].end = (uint32_t)p2.size();
    std::vector<P2Desc>().swap(per[w]);
  }
  if (p2.size() > (size_t)UINT32_MAX) return fail(HM_ERR_UNSUPPORTED, "too many matvec descriptors");
  P.np1 = (int64_t)p1.size();
  P.np2 = (int64_t)p2.size();
  P.nwin = (int32_t)nwin;
  if (!p1.empty()) {
    HM_CUDA_TRY(cudaMalloc(&P.d_p1, sizeof(P1Desc) * p1.size()));
    HM_CUDA_TRY(h2d_sync(P.d_p1, p1.data(), sizeof(P1Desc) * p1.size()));
  }
  if (!p2.empty()) {
    HM_CUDA_TRY(cudaMalloc(&P.d_p2, sizeof(P2Desc) * p2.size()));
    HM_CUDA_TRY(h2d_sync(P.d_p2, p2.data(), sizeof(P2Desc) * p2.size()));
  }
  HM_CUDA_TRY(cudaMalloc(&P.d_win, sizeof(MvWin) * nwin));
  HM_CUDA_TRY(h2d_sync(P.d_win, wins.data(), sizeof(MvWin) * nwin));
  return HM_OK;
}

// ---------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------
static int ensure_xs(hm_handle* h, size_t bytes) {
  if (h->xs_bytes >= bytes) return HM_OK;
  if (h->d_xs) cudaFree(h->d_xs);
  h->d_xs = nullptr;
  h->xs_bytes = 0;
  HM_CUDA_TRY(cudaMalloc(&h->d_xs, bytes));
  h->xs_bytes = bytes;
  return HM_OK;
}

// The window lists split by leaf kind: the dense leaves alone (the passes that
// treat them separately: tensor-core calls, BF16 single-column products) and
// the low-rank leaves alone.
int split_p2(MvPlan& P) {
  if (P.d_wind || P.nwin == 0) return HM_OK;
  std::vector<P2Desc> v((size_t)P.np2);
  std::vector<MvWin> win((size_t)P.nwin);
  if (P.np2 > 0) HM_CUDA_TRY(cudaMemcpy(v.data(), P.d_p2, sizeof(P2Desc) * v.size(), cudaMemcpyDeviceToHost));
  HM_CUDA_TRY(cudaMemcpy(win.data(), P.d_win, sizeof(MvWin) * win.size(), cudaMemcpyDeviceToHost));
  std::vector<P2Desc> dd, rr;
  std::vector<MvWin> wd(win), wr(win);
  for (size_t w = 0; w < win.size(); ++w) {
    wd[w].begin = (uint32_t)dd.size();
    wr[w].begin = (uint32_t)rr.size();
    for (uint32_t i = win[w].begin; i < win[w].end; ++i) (v[i].type == P2_RK ? rr : dd).push_back(v[i]);
    wd[w].end = (uint32_t)dd.size();
    wr[w].end = (uint32_t)rr.size();
  }
  if (dd.empty()) dd.push_back(P2Desc{});        // keeps the pointers valid; no window refers to them
  if (rr.empty()) rr.push_back(P2Desc{});
  HM_CUDA_TRY(cudaMalloc(&P.d_p2r, sizeof(P2Desc) * rr.size()));
  HM_CUDA_TRY(h2d_sync(P.d_p2r, rr.data(), sizeof(P2Desc) * rr.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_winr, sizeof(MvWin) * wr.size()));
  HM_CUDA_TRY(h2d_sync(P.d_winr, wr.data(), sizeof(MvWin) * wr.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_p2d, sizeof(P2Desc) * dd.size()));
  HM_CUDA_TRY(h2d_sync(P.d_p2d, dd.data(), sizeof(P2Desc) * dd.size()));
  HM_CUDA_TRY(cudaMalloc(&P.d_wind, sizeof(MvWin) * wd.size()));   // last: marks the split as complete
  HM_CUDA_TRY(h2d_sync(P.d_wind, wd.data(), sizeof(MvWin) * wd.size()));
  return HM_OK;
}

// y = the dense leaves' part of H x (one column): a warp per 32 output rows
// walks its window's dense descriptors; the leaves covering its rows are read
// column by column (32 consecutive rows a load, eight columns in flight).
template <typename TD>
__global__ void __launch_bounds__(256) mv_dense1_kernel(const MvWin* __restrict__ win, const P2Desc* __restrict__ d,
                                                        const TD* __restrict__ dn, const double* __restrict__ x,
                                                        int64_t nslab, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gw >= nslab) return;
  const int64_t grow = gw * 32;
  const MvWin W = win[grow / MV_WROWS];
  const int r0 = (int)(grow - W.row0), r = r0 + lane;
  double acc = 0.0;
  for (uint32_t i = W.begin; i < W.end; ++i) {
    const P2Desc D = d[i];
    if (D.row_off >= r0 + 32 || D.row_off + (int)D.m <= r0) continue;
    const int lr = r - D.row_off;
    const bool mine = lr >= 0 && lr < (int)D.m;
    const bool tr = D.type == P2_DENSE_T;
    const TD* col = dn + D.off + (mine ? (tr ? (int64_t)lr * D.ld : (int64_t)lr) : 0);
    const int64_t cs = tr ? 1 : (int64_t)D.ld;
    const double* xs = x + D.aux;
    uint32_t c = 0;
    for (; c + 8 <= D.cnt; c += 8) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = mine ? (double)__ldcs(col + (int64_t)(c + u) * cs) : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u) acc = fma(v[u], __ldg(xs + c + u), acc);
    }
    for (; c < D.cnt; ++c) acc = fma(mine ? (double)__ldcs(col + (int64_t)c * cs) : 0.0, __ldg(xs + c), acc);
  }
  if (r < (int)W.nrows) y[W.row0 + r] = acc;
}

// BF16 factors: y += the low-rank leaves' part, each lane owning 8
// consecutive output rows (one 16-byte load of 8 BF16 values where the leaf
// starts on an 8-row boundary of the window, two 8-byte loads on a 4-row
// boundary, element loads elsewhere; padding rows hold zeros).  Twice the rows
// of the 4-row kernel per entry: BF16 halves the bytes of an entry, and the
// 4-row form ran out of issue slots before HBM.
template <int SPLIT> struct P2Shape8 {
  static constexpr int CROWS = MV_WROWS / SPLIT;   // rows of one CTA
  static constexpr int WARPS = CROWS / 256;        // 32 lanes x 8 rows a warp
  static constexpr int EMAX = 1024 / SPLIT;
};
template <int SPLIT>
__global__ void __launch_bounds__(P2Shape8<SPLIT>::WARPS * 32) mv_phase2_bf16_kernel(
    const MvWin* __restrict__ win, const P2Desc* __restrict__ d, const __nv_bfloat16* __restrict__ rk,
    const double* __restrict__ z, double* __restrict__ y) {
  constexpr int U = 8;
  constexpr int CROWS = P2Shape8<SPLIT>::CROWS, EMAX = P2Shape8<SPLIT>::EMAX;
  __shared__ P2Desc sd[P2_NB];
  __shared__ int spre[P2_NB + 1];
  __shared__ uint64_t e_off[EMAX];
  __shared__ int32_t e_ro[EMAX];
  __shared__ uint32_t e_m[EMAX];
  __shared__ double e_z[EMAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const MvWin W = win[blockIdx.x / SPLIT];
  const int h0 = (int)(blockIdx.x % SPLIT) * CROWS;
  const int base = h0 + 8 * (warp * 32 + lane);
  const uint16_t* rkb = reinterpret_cast<const uint16_t*>(rk);
  double acc[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) acc[q] = 0.0;
  for (uint32_t b0 = W.begin; b0 < W.end; b0 += P2_NB) {
    const int nb = (int)min((uint32_t)P2_NB, W.end - b0);
    __syncthreads();
    if (warp == 0) {
      int cnt = 0;
      if (lane < nb) {
        sd[lane] = d[b0 + lane];
        const int r0 = sd[lane].row_off, r1 = r0 + (int)sd[lane].m;
        cnt = (r1 > h0 && r0 < h0 + CROWS) ? (int)sd[lane].cnt : 0;
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
        e_off[e] = D.off + (uint64_t)c * D.ld;
        e_z[e] = z[D.aux + c];
        e_ro[e] = D.row_off;
        e_m[e] = D.m;
      }
      __syncthreads();
      for (int e = 0; e < ne; e += U) {
        uint4 raw[U];
        double zz[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          raw[u] = make_uint4(0u, 0u, 0u, 0u);
          zz[u] = 0.0;
          const int ee = e + u;
          if (ee < ne) {
            const int ro = e_ro[ee];
            const int mm = (int)e_m[ee];
            const uint64_t o = e_off[ee];
            const int lr = base - ro;
            zz[u] = e_z[ee];
            if ((ro & 7) == 0) {
              if (lr >= 0 && lr < mm) raw[u] = __ldcs(reinterpret_cast<const uint4*>(rk + o + lr));
            } else if ((ro & 3) == 0) {
              if (lr >= 0 && lr < mm) {
                const uint2 a = __ldcs(reinterpret_cast<const uint2*>(rk + o + lr));
                raw[u].x = a.x; raw[u].y = a.y;
              }
              if (lr + 4 >= 0 && lr + 4 < mm) {
                const uint2 b = __ldcs(reinterpret_cast<const uint2*>(rk + o + lr + 4));
                raw[u].z = b.x; raw[u].w = b.y;
              }
            } else {
              uint32_t wv[4] = {0u, 0u, 0u, 0u};
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int r = lr + q;
                if (r >= 0 && r < mm) wv[q >> 1] |= (uint32_t)rkb[o + (uint64_t)r] << (16 * (q & 1));
              }
              raw[u] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            }
          }
        }
        // FP32 products and partial sums over the entries in flight, folded
        // into the FP64 row sums once per group
        float part[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) part[q] = 0.f;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const float zf = (float)zz[u];
          const uint32_t w4[4] = {raw[u].x, raw[u].y, raw[u].z, raw[u].w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            part[2 * q] = fmaf(bf_lo(w4[q]), zf, part[2 * q]);
            part[2 * q + 1] = fmaf(bf_hi(w4[q]), zf, part[2 * q + 1]);
          }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] += (double)part[q];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q)
    if (base + q < (int)W.nrows) y[W.row0 + base + q] += acc[q];
}

template <typename T>
static int matvec_t(hm_handle* h, const double* d_x, double* d_y, int trans, cudaStream_t st, cudaEvent_t* ev) {
  using TX = typename MvT<T>::X;
  constexpr int XA = 16 / (int)sizeof(TX);
  MvPlan& P = trans ? h->bwd : h->fwd;
  if (std::is_same<T, __nv_bfloat16>::value) HM_TRY(split_p2(P));
  const int64_t stride = pad_to(h->n + 64, 64);
  HM_TRY(ensure_xs(h, sizeof(TX) * stride * XA));
  TX* xs = (TX*)h->d_xs;
  if (ev) HM_CUDA_TRY(cudaEventRecord(ev[0], st));
  {
    int64_t tot = stride * XA;
    unsigned g = (unsigned)std::min<int64_t>((tot + 255) / 256, 148 * 16);
    xcopy_kernel<TX><<<g, 256, 0, st>>>(d_x, h->n, xs, stride, XA);
  }
  if (ev) HM_CUDA_TRY(cudaEventRecord(ev[1], st));
  if (P.np1 > 0) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    // one wave of resident CTAs: the warps stride over equal-sized leaves and
    // finish together (a grid of several partial waves leaves a tail)
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mv_phase1_kernel<T>, 256, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    int64_t blocks = std::min<int64_t>((P.np1 + 7) / 8, (int64_t)nsm * per_sm * std::max(1, h->tune.p1_waves));
    mv_phase1_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(P.d_p1, P.np1, (const T*)h->d_rk, xs, stride, h->d_z);
  }
  if (ev) HM_CUDA_TRY(cudaEventRecord(ev[2], st));
  // dense leaves are FP64 with FP64 factors and FP32 otherwise
  using TD = typename std::conditional<std::is_same<T, double>::value, double, float>::type;
  if constexpr (std::is_same<T, __nv_bfloat16>::value) {
    // dense leaves (FP32) first, written into y; then the BF16 low-rank part added
    const int64_t nslab = (h->n + 31) / 32;
    mv_dense1_kernel<float><<<(unsigned)((nslab + 7) / 8), 256, 0, st>>>(P.d_wind, P.d_p2d,
                                                                         (const float*)h->d_dense, d_x, nslab, d_y);
    if (h->tune.p2_split == 2)
      mv_phase2_bf16_kernel<2><<<(unsigned)(P.nwin * 2), P2Shape8<2>::WARPS * 32, 0, st>>>(
          P.d_winr, P.d_p2r, (const __nv_bfloat16*)h->d_rk, h->d_z, d_y);
    else                                       // splits 4 and 8: one warp a quarter window
      mv_phase2_bf16_kernel<4><<<(unsigned)(P.nwin * 4), P2Shape8<4>::WARPS * 32, 0, st>>>(
          P.d_winr, P.d_p2r, (const __nv_bfloat16*)h->d_rk, h->d_z, d_y);
  } else if (h->tune.p2_split == 1) {
    if (!P.cl_built) HM_TRY(build_cluster_plan(h, trans, P));
    HM_CUDA_TRY(cudaMemsetAsync(d_y, 0, sizeof(double) * h->n, st));
    for (size_t l = 0; l + 1 < P.cl_level.size(); ++l) {
      const int u0 = P.cl_level[l], nu = P.cl_level[l + 1] - u0;
      if (nu == 0) continue;
      mv_phase2c_kernel<T><<<(unsigned)((nu + CL_WARPS - 1) / CL_WARPS), CL_WARPS * 32, 0, st>>>(
          P.d_cu + u0, nu, P.d_cd, (const T*)h->d_rk, (const T*)h->d_dense, h->d_z, d_x, d_y);
    }
  } else {
    auto p2 = [&](auto split) {
      constexpr int S = decltype(split)::value;
      mv_phase2_kernel<T, TD, S><<<(unsigned)(P.nwin * S), P2Shape<S>::WARPS * 32, 0, st>>>(
          P.d_win, P.d_p2, (const T*)h->d_rk, (const TD*)h->d_dense, h->d_z, d_x, d_y);
    };
    switch (h->tune.p2_split) {
      case 2: p2(std::integral_constant<int, 2>{}); break;
      case 8: p2(std::integral_constant<int, 8>{}); break;
      default: p2(std::integral_constant<int, 4>{});
    }
  }
  if (ev) HM_CUDA_TRY(cudaEventRecord(ev[3], st));
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

int matvec_device(hm_handle* h, const double* d_x, double* d_y, int trans, cudaStream_t st, cudaEvent_t* ev) {
  switch (h->storage) {
    case HM_F64: return matvec_t<double>(h, d_x, d_y, trans, st, ev);
    case HM_F32: return matvec_t<float>(h, d_x, d_y, trans, st, ev);
    default: return matvec_t<__nv_bfloat16>(h, d_x, d_y, trans, st, ev);
  }
}

// ---------------------------------------------------------------------------
// residual r = b - H x with compensated (double-double) sums, for iterative
// refinement: every product is split exactly (TwoProduct by FMA) and every
// sum carries its rounding error (TwoSum), the dot product and sum algorithms
// of Ogita, Rump & Oishi (2005), "Accurate sum and dot product".  The result
// is as accurate as if H x were summed in twice the FP64 precision, so the
// refinement is not stopped by the rounding of H x near b.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void dd_add_prod(double& p, double& c, double a, double b) {
  const double h = a * b;
  const double r = fma(a, b, -h);          // a b = h + r exactly
  double q;
  two_sum(p, h, p, q);
  c += q + r;
}

// z = F1' x per low-rank leaf and rank, as hi + lo; one warp per leaf
template <typename T>
__global__ void __launch_bounds__(256) mvdd_phase1_kernel(const P1Desc* __restrict__ d, int64_t nd,
                                                          const T* __restrict__ pool, const double* __restrict__ x,
                                                          double* __restrict__ zh, double* __restrict__ zl) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t b = gw; b < nd; b += nw) {
    const P1Desc D = d[b];
    for (int r = 0; r < D.k; ++r) {
      const T* f = pool + D.off + (int64_t)r * D.stride;
      double p = 0.0, c = 0.0;
      for (uint32_t j = lane; j < D.len; j += 32) dd_add_prod(p, c, from_store<T>(f[j]), x[D.seg0 + j]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double p2 = __shfl_xor_sync(0xffffffffu, p, o), c2 = __shfl_xor_sync(0xffffffffu, c, o);
        double q;
        two_sum(p, p2, p, q);
        c += c2 + q;
      }
      if (lane == 0) {
        const double hi = p + c;
        zh[D.zoff + r] = hi;
        zl[D.zoff + r] = c - (hi - p);
      }
    }
  }
}

// r = b - (sum over the window's leaves) per output row, one thread a row; a
// window is split over MVDD_SPLIT CTAs of MV_WROWS / MVDD_SPLIT rows (the
// double-double sums are latency-bound: one CTA per window left most SMs idle)
constexpr int MVDD_SPLIT = 8;
constexpr int MVDD_ROWS = MV_WROWS / MVDD_SPLIT;
template <typename T, typename TD>
__global__ void __launch_bounds__(MVDD_ROWS) mvdd_phase2_kernel(const MvWin* __restrict__ win,
                                                                const P2Desc* __restrict__ d, const T* __restrict__ rk,
                                                                const TD* __restrict__ dn, const double* __restrict__ zh,
                                                                const double* __restrict__ zl,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ bvec, double* __restrict__ rvec) {
  const MvWin W = win[blockIdx.x / MVDD_SPLIT];
  const int r0 = (int)(blockIdx.x % MVDD_SPLIT) * MVDD_ROWS;      // this CTA's rows [r0, r0 + MVDD_ROWS)
  const uint32_t row = (uint32_t)(r0 + threadIdx.x);
  if (row < W.nrows) {
    double p = 0.0, c = 0.0;
    for (uint32_t e = W.begin; e < W.end; ++e) {
      const P2Desc D = d[e];
      if (D.row_off >= r0 + MVDD_ROWS || D.row_off + (int)D.m <= r0) continue;   // the whole CTA skips it
      const int lr = (int)row - D.row_off;
      if (lr < 0 || lr >= (int)D.m) continue;
      if (D.type == P2_RK) {
        for (uint32_t q = 0; q < D.cnt; ++q) {
          const double v = from_store<T>(rk[D.off + (uint64_t)q * D.ld + lr]);
          dd_add_prod(p, c, v, zh[D.aux + q]);
          c = fma(v, zl[D.aux + q], c);
        }
      } else if (D.type == P2_DENSE) {
        for (uint32_t q = 0; q < D.cnt; ++q)
          dd_add_prod(p, c, (double)dn[D.off + (uint64_t)q * D.ld + lr], x[D.aux + q]);
      } else {
        for (uint32_t q = 0; q < D.cnt; ++q)
          dd_add_prod(p, c, (double)dn[D.off + (uint64_t)q + (uint64_t)lr * D.ld], x[D.aux + q]);
      }
    }
    const uint32_t i = W.row0 + row;
    double t, q;
    two_sum(bvec[i], -p, t, q);
    rvec[i] = t + (q - c);
  }
}

template <typename T>
static int residual_t(hm_handle* h, const double* d_x, const double* d_b, double* d_r, int trans, cudaStream_t st) {
  using TD = typename std::conditional<std::is_same<T, double>::value, double, float>::type;
  const MvPlan& P = trans ? h->bwd : h->fwd;
  const size_t need = sizeof(double) * 2 * (size_t)std::max<int64_t>(h->zlen, 1);
  if (h->dd_bytes < need) {
    if (h->d_dd) cudaFree(h->d_dd);
    h->d_dd = nullptr;
    h->dd_bytes = 0;
    cudaError_t e = cudaMalloc(&h->d_dd, need);
    if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("residual buffers: ") + cudaGetErrorString(e));
    h->dd_bytes = need;
  }
  double* zh = (double*)h->d_dd;
  double* zl = zh + std::max<int64_t>(h->zlen, 1);
  if (P.np1 > 0) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int64_t blocks = std::min<int64_t>((P.np1 + 7) / 8, (int64_t)nsm * 8);
    mvdd_phase1_kernel<T><<<(unsigned)blocks, 256, 0, st>>>(P.d_p1, P.np1, (const T*)h->d_rk, d_x, zh, zl);
  }
  mvdd_phase2_kernel<T, TD><<<(unsigned)(P.nwin * MVDD_SPLIT), MVDD_ROWS, 0, st>>>(
      P.d_win, P.d_p2, (const T*)h->d_rk, (const TD*)h->d_dense, zh, zl, d_x, d_b, d_r);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

int residual_device(hm_handle* h, const double* d_x, const double* d_b, double* d_r, int trans, cudaStream_t st) {
  switch (h->storage) {
    case HM_F64: return residual_t<double>(h, d_x, d_b, d_r, trans, st);
    case HM_F32: return residual_t<float>(h, d_x, d_b, d_r, trans, st);
    default: return residual_t<__nv_bfloat16>(h, d_x, d_b, d_r, trans, st);
  }
}

// ---------------------------------------------------------------------------
// exact FP64 rows (K14): y_i = sum_j K(x_rows[i], x_j) x_j + shift * x_rows[i]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) exact_rows_kernel(KernelDesc kd, const double* __restrict__ geom, int64_t n,
                                                         const int64_t* __restrict__ rows,
                                                         const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double red[32];
  const int64_t i = rows[blockIdx.x];
  double s = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) s = fma(kernel_eval(kd, geom, n, i, j), x[j], s);
  s = block_sum(s, red);
  if (threadIdx.x == 0) y[blockIdx.x] = s + kd.shift * x[i];
}

int exact_rows_device(hm_handle* h, const int64_t* d_rows, int64_t nrows, const double* d_x, double* d_y,
                      cudaStream_t st) {
  if (nrows <= 0) return HM_OK;
  for (int64_t b0 = 0; b0 < nrows; b0 += (1ll << 30)) {
    unsigned nb = (unsigned)std::min<int64_t>(nrows - b0, 1ll << 30);
    exact_rows_kernel<<<nb, 512, 0, st>>>(h->kd, h->d_geom, h->n, d_rows + b0, d_x, d_y + b0);
  }
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

// ---------------------------------------------------------------------------
// densify (to_fmat, src/utils.jl:162-192), leaf factors, shift, scale, copy
// ---------------------------------------------------------------------------
struct LeafDev {
  int64_t row0, col0, off;
  int32_t m, n, k, type;
};

template <typename T, typename TD>
__global__ void to_dense_kernel(const LeafDev* __restrict__ L, const T* __restrict__ rk, const TD* __restrict__ dn,
                                int64_t n, double* __restrict__ out) {
  const LeafDev D = L[blockIdx.x];
  const int eb = (int)sizeof(T), deb = (int)sizeof(TD);
  const int64_t tot = (int64_t)D.m * D.n;
  for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
    const int i = (int)(e % D.m), j = (int)(e / D.m);
    double v;
    if (D.type == T_DENSE) {
      v = (double)dn[D.off + i + (int64_t)j * col_pad_dev(D.m, deb)];
    } else {
      const int64_t npad = col_pad_dev(D.n, eb), mpad = col_pad_dev(D.m, eb);
      const T* B = rk + D.off;
      const T* A = B + npad * D.k;
      v = 0.0;
      for (int q = 0; q < D.k; ++q) v = fma(from_store<T>(A[i + q * mpad]), from_store<T>(B[j + q * npad]), v);
    }
    out[(D.row0 + i) + (D.col0 + j) * n] = v;
  }
}

int to_dense(const hm_handle* h, double* d_out) {
  std::vector<LeafDev> L(h->leaves.size());
  for (size_t i = 0; i < L.size(); ++i) {
    const Leaf& x = h->leaves[i];
    L[i] = LeafDev{x.row0, x.col0, x.off, x.m, x.n, x.k, x.type};
  }
  if (L.empty()) return HM_OK;
  LeafDev* dL = nullptr;
  HM_CUDA_TRY(cudaMalloc(&dL, sizeof(LeafDev) * L.size()));
  HM_CUDA_TRY(cudaMemcpyAsync(dL, L.data(), sizeof(LeafDev) * L.size(), cudaMemcpyHostToDevice, h->stream));
  const unsigned nb = (unsigned)L.size();
  switch (h->storage) {
    case HM_F64:
      to_dense_kernel<double, double><<<nb, 256, 0, h->stream>>>(dL, (const double*)h->d_rk, (const double*)h->d_dense, h->n, d_out);
      break;
    case HM_F32:
      to_dense_kernel<float, float><<<nb, 256, 0, h->stream>>>(dL, (const float*)h->d_rk, (const float*)h->d_dense, h->n, d_out);
      break;
    default:
      to_dense_kernel<__nv_bfloat16, float><<<nb, 256, 0, h->stream>>>(dL, (const __nv_bfloat16*)h->d_rk, (const float*)h->d_dense, h->n, d_out);
  }
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  cudaFree(dL);
  return HM_OK;
}

static inline double bf16_bits_to_double(uint16_t b) {
  uint32_t w = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &w, 4);
  return (double)f;
}

int leaf_factors_f64(const hm_handle* h, int64_t leaf, double* A, double* B) {
  const Leaf& L = h->leaves[leaf];
  if (L.type != T_RK) return fail(HM_ERR_ARG, "leaf is not low-rank");
  const int eb = elem_bytes(h->storage);
  const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
  const int64_t tot = (npad + mpad) * L.k;
  std::vector<char> buf(tot * eb);
  if (tot) HM_CUDA_TRY(cudaMemcpy(buf.data(), (const char*)h->d_rk + L.off * eb, tot * eb, cudaMemcpyDeviceToHost));
  auto get = [&](int64_t e) -> double {
    if (eb == 8) return ((const double*)buf.data())[e];
    if (eb == 4) return (double)((const float*)buf.data())[e];
    return bf16_bits_to_double(((const uint16_t*)buf.data())[e]);
  };
  for (int q = 0; q < L.k; ++q) {
    for (int j = 0; j < L.n; ++j) B[j + (int64_t)q * L.n] = get(j + q * npad);
    for (int i = 0; i < L.m; ++i) A[i + (int64_t)q * L.m] = get(npad * L.k + i + q * mpad);
  }
  return HM_OK;
}

template <typename TD>
__global__ void shift_kernel(const int64_t* __restrict__ offs, const int32_t* __restrict__ ms, int nleaf,
                             const int32_t* __restrict__ lds, TD* dn, double lam) {
  const int b = blockIdx.x;
  for (int i = threadIdx.x; i < ms[b]; i += blockDim.x) {
    TD* p = dn + offs[b] + i + (int64_t)i * lds[b];
    *p = (TD)((double)*p + lam);
  }
}

int apply_shift(hm_handle* h, double lam) {
  std::vector<int64_t> offs;
  std::vector<int32_t> ms, lds;
  const int deb = dense_elem_bytes(h->storage);
  for (auto& L : h->leaves)
    if (L.type == T_DENSE && L.row0 == L.col0 && L.m == L.n) {
      offs.push_back(L.off);
      ms.push_back(L.m);
      lds.push_back((int32_t)col_pad(L.m, deb));
    }
  if (!offs.empty()) {
    int64_t* d_o = nullptr;
    int32_t *d_m = nullptr, *d_l = nullptr;
    HM_CUDA_TRY(cudaMalloc(&d_o, 8 * offs.size()));
    HM_CUDA_TRY(cudaMalloc(&d_m, 4 * ms.size()));
    HM_CUDA_TRY(cudaMalloc(&d_l, 4 * lds.size()));
    HM_CUDA_TRY(h2d_sync(d_o, offs.data(), 8 * offs.size()));
    HM_CUDA_TRY(h2d_sync(d_m, ms.data(), 4 * ms.size()));
    HM_CUDA_TRY(h2d_sync(d_l, lds.data(), 4 * lds.size()));
    if (h->storage == HM_F64)
      shift_kernel<double><<<(unsigned)offs.size(), 128, 0, h->stream>>>(d_o, d_m, (int)offs.size(), d_l, (double*)h->d_dense, lam);
    else
      shift_kernel<float><<<(unsigned)offs.size(), 128, 0, h->stream>>>(d_o, d_m, (int)offs.size(), d_l, (float*)h->d_dense, lam);
    HM_CUDA_TRY(cudaGetLastError());
    HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
    cudaFree(d_o); cudaFree(d_m); cudaFree(d_l);
  }
  h->kd.shift += lam;
  return HM_OK;
}

template <typename T>
__global__ void scale_kernel(T* p, int64_t cnt, double u) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
    p[e] = to_store<T>(from_store<T>(p[e]) * u);
}

int apply_scale(hm_handle* h, double u) {
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  // dense pool: every element (padding is zero and stays zero)
  if (h->dense_bytes) {
    if (h->storage == HM_F64) scale_kernel<double><<<592, 256, 0, h->stream>>>((double*)h->d_dense, h->dense_bytes / deb, u);
    else scale_kernel<float><<<592, 256, 0, h->stream>>>((float*)h->d_dense, h->dense_bytes / deb, u);
  }
  // low-rank leaves: the A factor only, as u*H scales H.A (src/harithm.jl:487)
  for (auto& L : h->leaves) {
    if (L.type != T_RK || L.k == 0) continue;
    const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
    const int64_t o = L.off + npad * L.k, cnt = mpad * L.k;
    unsigned g = (unsigned)std::min<int64_t>((cnt + 255) / 256, 64);
    if (h->storage == HM_F64) scale_kernel<double><<<g, 256, 0, h->stream>>>((double*)h->d_rk + o, cnt, u);
    else if (h->storage == HM_F32) scale_kernel<float><<<g, 256, 0, h->stream>>>((float*)h->d_rk + o, cnt, u);
    else scale_kernel<__nv_bfloat16><<<g, 256, 0, h->stream>>>((__nv_bfloat16*)h->d_rk + o, cnt, u);
  }
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->kd.shift *= u;
  return HM_OK;
}

static int dup(void** dst, const void* src, size_t bytes) {
  *dst = nullptr;
  if (!bytes || !src) return HM_OK;
  cudaError_t e = cudaMalloc(dst, bytes);
  if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("copy: ") + cudaGetErrorString(e));
  HM_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyDeviceToDevice));
  return HM_OK;
}

int copy_handle(const hm_handle* h, hm_handle** out) {
  hm_handle* c = new hm_handle();
  c->prm = h->prm; c->n = h->n; c->dim = h->dim; c->device = h->device; c->kd = h->kd;
  c->cl_s = h->cl_s; c->cl_e = h->cl_e; c->cl_left = h->cl_left; c->cl_right = h->cl_right;
  c->cl_depth = h->cl_depth; c->nodes = h->nodes; c->leaves = h->leaves; c->depth = h->depth;
  c->storage = h->storage; c->kmax = h->kmax; c->rk_bytes = h->rk_bytes; c->dense_bytes = h->dense_bytes;
  c->zlen = h->zlen;
  c->tune = h->tune;                           // the same launch shapes: the same sums in the same order
  // h's pending work lands before the copies read it (they run on the legacy
  // stream, which the handles' non-blocking streams do not order with)
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) { delete c; return fail(HM_ERR_CUDA, cudaGetErrorString(e)); }
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return fail(HM_ERR_CUDA, cudaGetErrorString(e)); }
  int s = HM_OK;
  auto chk = [&](int st) { if (s == HM_OK) s = st; };
  chk(dup((void**)&c->d_geom, h->d_geom, sizeof(double) * h->n * h->dim));
  chk(dup(&c->d_rk, h->d_rk, h->rk_bytes));
  chk(dup(&c->d_dense, h->d_dense, h->dense_bytes));
  chk(dup((void**)&c->d_z, h->d_z, sizeof(double) * h->zlen));
  chk(dup((void**)&c->d_piv, h->d_piv, sizeof(int32_t) * h->piv_count));
  c->piv_count = h->d_piv ? h->piv_count : 0;
  for (int t = 0; t < 2 && s == HM_OK; ++t) {
    const MvPlan& a = t ? h->bwd : h->fwd;
    MvPlan& b = t ? c->bwd : c->fwd;
    b.np1 = a.np1; b.np2 = a.np2; b.nwin = a.nwin;
    chk(dup((void**)&b.d_p1, a.d_p1, sizeof(P1Desc) * a.np1));
    chk(dup((void**)&b.d_p2, a.d_p2, sizeof(P2Desc) * a.np2));
    chk(dup((void**)&b.d_win, a.d_win, sizeof(MvWin) * a.nwin));
  }
  if (s == HM_OK && h->lu) s = lu_copy(h, c);
  c->factorized = h->factorized;
  // and the copies land before c's kernels read them
  if (s == HM_OK && cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess) s = fail(HM_ERR_CUDA, "copy");
  if (s != HM_OK) {
    free_handle_data(c);
    cudaStreamDestroy(c->stream);
    delete c;
    return s;
  }
  *out = c;
  return HM_OK;
}

}  // namespace hm
