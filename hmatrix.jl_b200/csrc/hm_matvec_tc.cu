// Multi-RHS H-matvec on the 5th-generation tensor cores (tcgen05, sm_100a):
// Y = H X (or H' X) for an n x c block of right-hand sides with FP32 or BF16
// stored factors, the device form of *(Hmat, Matrix) (src/harithm.jl:
// 317-329), which the reference evaluates one column at a time.
//
// Phase 1 (Z = F1' X_seg): the factor columns of all low-rank leaves that
//   share one input segment are stacked into 128-row M-tiles; one tcgen05 MMA
//   chain per tile computes Z_tile = F1_stack' X_seg (K = segment points,
//   N = columns) into a TMEM accumulator.  The factor rows are gathered into
//   shared memory by cp.async (their pool offsets are irregular), the X tiles
//   come pre-tiled from HBM by 1-D bulk copies (TMA engine).
// Phase 2 (Y += F2 Z): output windows of 512 rows (4 M-tiles); K runs over
//   the low-rank columns that touch the window (their Z rows are laid out
//   contiguously per window by phase 1's epilogue), A = F2 columns in
//   M-major form (rows contiguous in the pool).  Dense leaves are added by
//   the CUDA-core block kernel first.
//
// Accuracy.  FP32 factors use three TF32 products per term (F_hi X_hi +
// F_hi X_lo + F_lo X_hi, the split of Ootomo & Yokota 2022), BF16 factors
// are exact in BF16 and X is split into two BF16 parts (F X_1 + F X_2); the
// accumulation is FP32 in TMEM, and the FP32 sums are added into FP64 Y.
// Both splits round to nearest and leave exact values of the narrow format,
// so the hardware's own input conversion does not matter.
//
// Pipeline per CTA (persistent, one per SM): warps 0-3 produce stages
// (cp.async gathers, the split of FP32 factors into hi/lo, the bulk copy of
// the X / Z tile), warp 8 issues the MMAs (one thread), warps 4-7 drain the
// TMEM accumulators (tcgen05.ld).  mbarriers link the roles; every wait is
// bounded and a timeout sets an error word and ends the kernel cleanly.
#include "hm_internal.h"
#include "hm_tc.cuh"

#include <algorithm>
#include <vector>

namespace hm {

struct TcCol1 {            // phase-1 M row: one factor column of F1
  uint64_t off;            // pool element offset of the column's first entry
  uint32_t zp0, zp1;       // its Z slots: zpl[zp0 .. zp1)
};
struct TcItem1 {           // up to TC_T tiles of one input segment
  uint32_t col0, ncol;     // columns [col0, col0 + ncol) of the column table
  uint32_t seg0, len;      // input index range of the segment
};
struct TcZ2 {              // phase-2 K column (a Z slot) inside its window
  int64_t a_off;           // pool element offset of F2 at window row rlo
  int32_t rlo, rhi;        // rows [rlo, rhi) of the window it covers
};
struct TcItem2 {           // one output window
  uint32_t row0, nrows;
  uint32_t zb, ze;         // its Z slots [zb, ze)
};

struct TcPlan {
  TcCol1* d_col1 = nullptr;
  int64_t ncol1 = 0;
  TcItem1* d_item1 = nullptr;
  int64_t nitem1 = 0;
  uint32_t* d_zpl = nullptr;
  int64_t nzpl = 0;
  TcZ2* d_z2 = nullptr;
  int64_t nz2 = 0;
  TcItem2* d_item2 = nullptr;
  int64_t nitem2 = 0;
  bool aligned = true;     // every phase-2 column starts on a 16-byte row group
};

namespace {

constexpr int TC_T = 4;              // 128-row M-tiles per work item
constexpr int TC_WR = 128 * TC_T;    // rows of a phase-2 output window
constexpr int TC_KB = 4;             // 16-byte K blocks per pipeline stage
constexpr int TC_STAGES = 3;
constexpr int TC_THREADS = 288;      // warps 0-3 producers, 4-7 epilogue, 8 MMA
constexpr int TC_PROD = 128;
constexpr uint32_t TC_WAIT = 1u << 22;   // polls of a bounded mbarrier wait

template <typename T> struct TcT;
template <> struct TcT<float> {
  static constexpr int KE = 4;                      // elements per 16 bytes
  static constexpr int KIND = 0;                    // kind::tf32
  static constexpr int FMT = tc::FMT_TF32;
  static constexpr bool SPLIT = true;               // A = A_hi + A_lo
  using Bits = uint32_t;
  __device__ static float hi(float x) { return tc::tf32_rn(x); }
  __device__ static Bits bits(float x) { return __float_as_uint(x); }
};
template <> struct TcT<__nv_bfloat16> {
  static constexpr int KE = 8;
  static constexpr int KIND = 1;                    // kind::f16, BF16 inputs
  static constexpr int FMT = tc::FMT_BF16;
  static constexpr bool SPLIT = false;              // BF16 factors are exact
  using Bits = uint16_t;
  __device__ static float hi(float x) { return tc::bf16_rn(x); }
  __device__ static Bits bits(float x) { return (uint16_t)(__float_as_uint(x) >> 16); }
};

// ---------------------------------------------------------------------------
// X tiles for the B operand: XT[q][kb][part][n][e] holds part (0: hi, 1: lo)
// of X[t - q][cb*NC + n] at K index t = kb*KE + e (zero outside [0, n)).  The
// KE shifted copies let every segment start on a 16-byte K block; a block of
// 2*NC rows x 16 bytes is exactly the canonical K-major core-matrix layout.
// ---------------------------------------------------------------------------
template <typename T, int NC>
__global__ void tc_xt_kernel(const double* __restrict__ X, int64_t n, int64_t ldx, int ncols, int cb,
                             typename TcT<T>::Bits* __restrict__ xt, int64_t nkb) {
  constexpr int KE = TcT<T>::KE;
  const int64_t blk = 2 * NC * KE;
  const int64_t per_copy = nkb * blk;
  const int64_t tot = (int64_t)KE * per_copy;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = e / per_copy, r = e - q * per_copy;
    const int64_t kb = r / blk;
    int rem = (int)(r - kb * blk);
    const int part = rem / (NC * KE);
    rem -= part * NC * KE;
    const int nn = rem / KE, el = rem - nn * KE;
    const int64_t t = kb * KE + el - q;
    const int col = cb * NC + nn;
    float v = 0.f;
    if (t >= 0 && t < n && col < ncols) {
      const float x = (float)X[t + (int64_t)col * ldx];
      const float h = TcT<T>::hi(x);
      v = part == 0 ? h : TcT<T>::hi(x - h);
    }
    xt[e] = TcT<T>::bits(v);
  }
}

// zero the Z tiles from block kb0 on (the padding after the last slot)
template <typename T>
__global__ void tc_zero_kernel(typename TcT<T>::Bits* __restrict__ p, int64_t cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
    p[e] = 0;
}

// shared memory of one CTA
template <typename T, int NC>
struct TcSmem {
  static constexpr int A_TILE = 128 * TC_KB * 16;                     // bytes of one 128-row A tile
  static constexpr int A_STAGE = TC_T * A_TILE;
  static constexpr int A_LO = TcT<T>::SPLIT ? A_STAGE : 0;
  static constexpr int B_STAGE = TC_KB * 2 * NC * 16;
  static constexpr int STAGE = A_STAGE + A_LO + B_STAGE;
  static constexpr int BAR_OFF = TC_STAGES * STAGE;
  static constexpr int BYTES = BAR_OFF + 256;
  static constexpr int TMEM_COLS = TC_T * 2 * NC <= 32 ? 32 : (TC_T * 2 * NC <= 64 ? 64 : (TC_T * 2 * NC <= 128 ? 128 : (TC_T * 2 * NC <= 256 ? 256 : 512)));
  static_assert(BYTES <= 227 * 1024, "stages exceed the shared memory of a CTA");
  static_assert(TC_T * 2 * NC <= 512, "accumulators exceed TMEM");
};

struct TcBars {
  uint64_t full[TC_STAGES];
  uint64_t empty[TC_STAGES];
  uint64_t acc_full;
  uint64_t acc_empty;
  uint64_t done;           // the MMA issuer's last commit: every MMA finished
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void tc_fail(int* err, TcBars* b, int code) {
  atomicOr(&b->abort, 1);
  atomicOr(err, code);
}
__device__ __forceinline__ bool tc_aborted(const TcBars* b) { return *(volatile const int*)&b->abort != 0; }

// barriers, TMEM; called by all threads
__device__ __forceinline__ uint32_t tc_setup(TcBars* bars, int warp, uint32_t tmem_cols) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      tc::mbar_init(&bars->full[s], TC_PROD + 1);    // 128 producers + the bulk-copy arrival
      tc::mbar_init(&bars->empty[s], 1);             // one tcgen05.commit
    }
    tc::mbar_init(&bars->acc_full, 1);
    tc::mbar_init(&bars->acc_empty, 128);            // the 4 epilogue warps
    tc::mbar_init(&bars->done, 1);
    bars->abort = 0;
    tc::fence_mbar_init();
  }
  if (warp == 4) tc::tmem_alloc(&bars->tmem, tmem_cols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  return bars->tmem;
}

// end of the kernel: the MMA issuer has waited for its last MMAs; free TMEM
__device__ __forceinline__ void tc_teardown(TcBars* bars, int warp, uint32_t tmem, uint32_t tmem_cols) {
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, tmem_cols);
  }
}

// the MMA issuer's last step: one commit and a bounded wait for it
__device__ __forceinline__ void tc_mma_drain(TcBars* bars, int* err) {
  tc::mma_commit(&bars->done);
  if (!tc::mbar_wait(&bars->done, 0u, TC_WAIT)) tc_fail(err, bars, 16);
}

// ---------------------------------------------------------------------------
// phase 1
// ---------------------------------------------------------------------------
template <typename T, int NC>
struct P1Args {
  const TcItem1* items;
  int64_t nitems;
  const TcCol1* cols;
  const uint32_t* zpl;
  const T* pool;
  const typename TcT<T>::Bits* xt;   // XT of this column block
  int64_t xt_copy;                   // elements of one shifted copy
  typename TcT<T>::Bits* zt;         // Z tiles
  int* err;
};

template <typename T, int NC>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_phase1_kernel(P1Args<T, NC> a) {
  using Tr = TcT<T>;
  using S = TcSmem<T, NC>;
  constexpr int KE = Tr::KE;
  constexpr int KC = TC_KB * KE;                    // K values per stage
  extern __shared__ __align__(1024) uint8_t smem[];
  TcBars* bars = reinterpret_cast<TcBars*>(smem + S::BAR_OFF);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t tmem = tc_setup(bars, warp, S::TMEM_COLS);
  const uint32_t sbase = tc::smem_u32(smem);

  if (warp < 4) {
    // ---------------- producers ----------------
    const int tid = threadIdx.x;
    uint32_t it = 0;                                // stage iterations issued
    uint32_t fin = 0;                               // stage iterations finished (split + arrive)
    auto finish = [&](uint32_t f) {
      const int s = (int)(f % TC_STAGES);
      if constexpr (Tr::SPLIT) {
        // this thread's own chunks: A_hi in place, A_lo beside it
#pragma unroll
        for (int j = 0; j < TC_T * 128 * TC_KB / TC_PROD; ++j) {
          const uint32_t off = (uint32_t)(tid + TC_PROD * j) * 16;
          float4 v = *reinterpret_cast<const float4*>(smem + s * S::STAGE + off);
          float4 h, l;
          h.x = tc::tf32_rn(v.x); l.x = tc::tf32_rn(v.x - h.x);
          h.y = tc::tf32_rn(v.y); l.y = tc::tf32_rn(v.y - h.y);
          h.z = tc::tf32_rn(v.z); l.z = tc::tf32_rn(v.z - h.z);
          h.w = tc::tf32_rn(v.w); l.w = tc::tf32_rn(v.w - h.w);
          *reinterpret_cast<float4*>(smem + s * S::STAGE + off) = h;
          *reinterpret_cast<float4*>(smem + s * S::STAGE + S::A_STAGE + off) = l;
        }
      }
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(&bars->full[s]);
    };
    for (int64_t w = blockIdx.x; w < a.nitems; w += gridDim.x) {
      const TcItem1 I = a.items[w];
      const int q = (KE - (int)(I.seg0 % KE)) % KE;
      const int64_t kb0 = ((int64_t)I.seg0 + q) / KE;
      const int nk = (int)((I.len + KC - 1) / KC);
      // the rows this thread feeds: chunk ci = tid + 128 j -> tile j / 4,
      // row 8 (tid / 32) + tid % 8 + 32 (j % 4), K block (tid / 8) % 4
      uint64_t coff[TC_T * 4];
      bool cval[TC_T * 4];
#pragma unroll
      for (int j = 0; j < TC_T * 4; ++j) {
        const int t = j / 4;
        const int row = 8 * (tid / 32) + tid % 8 + 32 * (j % 4);
        const uint32_t c = (uint32_t)(t * 128 + row);
        cval[j] = c < I.ncol;
        coff[j] = cval[j] ? a.cols[I.col0 + c].off : 0;
      }
      const int b = (tid / 8) % TC_KB;
      for (int kc = 0; kc < nk; ++kc, ++it) {
        const int s = (int)(it % TC_STAGES);
        const uint32_t ph = (it / TC_STAGES) & 1u;
        if (!tc::mbar_wait(&bars->empty[s], ph ^ 1u, TC_WAIT)) { tc_fail(a.err, bars, 1); break; }
        if (tc_aborted(bars)) break;
        const uint32_t abase = sbase + s * S::STAGE;
        if (tid == 0) {
          tc::mbar_arrive_expect_tx(&bars->full[s], S::B_STAGE);
          const typename Tr::Bits* src = a.xt + (int64_t)q * a.xt_copy + (kb0 + (int64_t)kc * TC_KB) * (2 * NC * KE);
          tc::bulk_g2s(abase + S::A_STAGE + S::A_LO, src, S::B_STAGE, &bars->full[s]);
        }
        const int64_t e0 = (int64_t)kc * KC + b * KE;      // first element of this thread's K block
        const int64_t left = (int64_t)I.len - e0;
        const uint32_t bytes = left >= KE ? 16u : (left > 0 ? (uint32_t)left * (uint32_t)sizeof(T) : 0u);
#pragma unroll
        for (int j = 0; j < TC_T * 4; ++j) {
          const uint32_t dst = abase + (uint32_t)(tid + TC_PROD * j) * 16;
          const T* src = cval[j] && bytes ? a.pool + coff[j] + e0 : a.pool;
          tc::cp_async16(dst, src, cval[j] ? bytes : 0u);
        }
        tc::cp_async_commit();
        if (it >= TC_STAGES - 1) {
          tc::cp_async_wait<TC_STAGES - 1>();
          finish(fin++);
        }
      }
      if (tc_aborted(bars)) break;
    }
    // drain: finish the stages still in flight
    tc::cp_async_wait<0>();
    while (fin < it) finish(fin++);
  } else if (warp == 8) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t LBO_A = 128, SBO_A = TC_KB * 128;       // K-major A tiles
      constexpr uint32_t LBO_B = 2 * NC * 16, SBO_B = 128;        // K-major [hi | lo] X tiles
      const uint32_t id_full = tc::idesc(Tr::FMT, 2 * NC, 0, 0);
      const uint32_t id_half = tc::idesc(Tr::FMT, NC, 0, 0);
      uint32_t it = 0, item = 0;
      bool ok = true;
      for (int64_t w = blockIdx.x; w < a.nitems && ok; w += gridDim.x, ++item) {
        const TcItem1 I = a.items[w];
        const int nk = (int)((I.len + KC - 1) / KC);
        const int ntile = (int)((I.ncol + 127) / 128);
        if (!tc::mbar_wait(&bars->acc_empty, (item & 1u) ^ 1u, TC_WAIT)) { tc_fail(a.err, bars, 2); ok = false; break; }
        tc::tc_fence_after();
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = (int)(it % TC_STAGES);
          const uint32_t ph = (it / TC_STAGES) & 1u;
          if (!tc::mbar_wait(&bars->full[s], ph, TC_WAIT)) { tc_fail(a.err, bars, 4); ok = false; break; }
          tc::tc_fence_after();
          const uint32_t abase = sbase + s * S::STAGE;
          const uint32_t bbase = abase + S::A_STAGE + S::A_LO;
          for (int t = 0; t < ntile; ++t) {
#pragma unroll
            for (int ks = 0; ks < TC_KB / 2; ++ks) {
              const uint64_t bd = tc::smem_desc(bbase + ks * 2 * LBO_B, LBO_B, SBO_B);
              const uint64_t ad = tc::smem_desc(abase + t * S::A_TILE + ks * 2 * LBO_A, LBO_A, SBO_A);
              tc::mma<Tr::KIND>(tmem + t * 2 * NC, ad, bd, id_full, (kc > 0 || ks > 0) ? 1u : 0u);
              if constexpr (Tr::SPLIT) {
                const uint64_t al = tc::smem_desc(abase + S::A_STAGE + t * S::A_TILE + ks * 2 * LBO_A, LBO_A, SBO_A);
                tc::mma<Tr::KIND>(tmem + t * 2 * NC, al, bd, id_half, 1u);
              }
            }
          }
          tc::mma_commit(&bars->empty[s]);
        }
        if (ok) tc::mma_commit(&bars->acc_full);
      }
      tc_mma_drain(bars, a.err);
    }
  } else {
    // ---------------- epilogue (warps 4-7: TMEM lanes 32 (warp - 4) ..) ----------------
    const int ew = warp - 4;
    uint32_t item = 0;
    for (int64_t w = blockIdx.x; w < a.nitems; w += gridDim.x, ++item) {
      const TcItem1 I = a.items[w];
      if (!tc::mbar_wait(&bars->acc_full, item & 1u, TC_WAIT)) { tc_fail(a.err, bars, 8); break; }
      tc::tc_fence_after();
      const int ntile = (int)((I.ncol + 127) / 128);
      for (int t = 0; t < ntile; ++t) {
        const uint32_t row = (uint32_t)(t * 128 + 32 * ew + lane);
        const bool valid = row < I.ncol;
        TcCol1 C{};
        if (valid) C = a.cols[I.col0 + row];
#pragma unroll
        for (int j0 = 0; j0 < NC; j0 += 16) {
          float d0[16], d1[16];
          const uint32_t ta = tmem + ((uint32_t)(32 * ew) << 16) + (uint32_t)(t * 2 * NC + j0);
          tc::tmem_ld16(ta, d0);
          tc::tmem_ld16(ta + NC, d1);
          if (valid) {
            for (uint32_t zi = C.zp0; zi < C.zp1; ++zi) {
              const uint32_t zp = a.zpl[zi];
              typename Tr::Bits* zb = a.zt + (int64_t)(zp / KE) * (2 * NC * KE) + (zp % KE);
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const float z = d0[j] + d1[j];
                const float h = Tr::hi(z);
                zb[(j0 + j) * KE] = Tr::bits(h);
                zb[NC * KE + (j0 + j) * KE] = Tr::bits(Tr::hi(z - h));
              }
            }
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&bars->acc_empty);
    }
  }
  tc_teardown(bars, warp, tmem, S::TMEM_COLS);
}

// ---------------------------------------------------------------------------
// phase 2
// ---------------------------------------------------------------------------
// Phase-2 A tiles are M-major (a factor column's rows are contiguous).  The
// 16-byte chunk ci of a 128-row tile holds rows KE g .. KE g + KE - 1 of its K
// column k; a2_chunk gives (g, k) and the chunk's byte offset in the tile.
//  BF16 (KE 8): no swizzle, core matrices of 8 K x 16 bytes: (k / 8) 2048 +
//    g 128 + (k % 8) 16; descriptor LBO = 2048 (along K), SBO = 128 (along M).
//  TF32 (KE 4): M-major TF32 operands take the 128-byte swizzle with 32-byte
//    atoms (descriptor layout 1): atoms of 32 rows (128 bytes) x 4 K rows
//    whose 32-byte pieces are permuted by XOR with k % 4; the 4 row atoms
//    512 bytes apart (LBO), groups of 4 K 2048 bytes apart (SBO).  Eight
//    consecutive chunks fill one 128-byte atom row (no bank conflicts) and
//    read 128 contiguous bytes of one factor column.
template <int KE>
__device__ __forceinline__ uint32_t a2_chunk(int ci, int& g, int& k) {
  if constexpr (KE == 8) {
    k = 8 * (ci / 128) + (ci % 8);
    g = (ci / 8) % 16;
    return (uint32_t)ci * 16u;
  } else {
    const int g8 = ci % 8;
    k = (ci / 8) % 16;
    g = (ci / 128) * 8 + g8;
    return (uint32_t)((g / 8) * 512 + (k / 4) * 2048 + (k % 4) * 128 + ((((g % 8) >> 1) ^ (k % 4)) << 5) +
                      (g & 1) * 16);
  }
}
// descriptor of K step ks (32 bytes of K) of the phase-2 A tile at `tile`
template <int KE>
__device__ __forceinline__ uint64_t a2_desc(uint32_t tile, int ks) {
  if constexpr (KE == 8) return tc::smem_desc(tile + ks * 2 * 2048, 2048, 128, 0);
  else return tc::smem_desc(tile + ks * 2 * 2048, 512, 2048, 1);
}
template <typename T, int NC>
struct P2Args {
  const TcItem2* items;
  int64_t nitems;
  const TcZ2* z2;
  const T* pool;
  const typename TcT<T>::Bits* zt;
  double* Y;
  int64_t ldy;
  int ncols, cb;
  int* err;
};

template <typename T, int NC>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_phase2_kernel(P2Args<T, NC> a) {
  using Tr = TcT<T>;
  using S = TcSmem<T, NC>;
  constexpr int KE = Tr::KE;
  constexpr int KC = TC_KB * KE;                    // K values (Z slots) per stage
  extern __shared__ __align__(1024) uint8_t smem[];
  TcBars* bars = reinterpret_cast<TcBars*>(smem + S::BAR_OFF);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t tmem = tc_setup(bars, warp, S::TMEM_COLS);
  const uint32_t sbase = tc::smem_u32(smem);

  if (warp < 4) {
    const int tid = threadIdx.x;
    uint32_t it = 0, fin = 0;
    auto finish = [&](uint32_t f) {
      const int s = (int)(f % TC_STAGES);
      if constexpr (Tr::SPLIT) {
        // exactly the chunks this thread filled (cp.async.wait_group covers
        // only this thread's own copies)
#pragma unroll
        for (int j = 0; j < TC_T * 4; ++j) {
          int g, k;
          const uint32_t off = (uint32_t)((j / 4) * S::A_TILE) + a2_chunk<KE>(tid + TC_PROD * (j % 4), g, k);
          float4 v = *reinterpret_cast<const float4*>(smem + s * S::STAGE + off);
          float4 h, l;
          h.x = tc::tf32_rn(v.x); l.x = tc::tf32_rn(v.x - h.x);
          h.y = tc::tf32_rn(v.y); l.y = tc::tf32_rn(v.y - h.y);
          h.z = tc::tf32_rn(v.z); l.z = tc::tf32_rn(v.z - h.z);
          h.w = tc::tf32_rn(v.w); l.w = tc::tf32_rn(v.w - h.w);
          *reinterpret_cast<float4*>(smem + s * S::STAGE + off) = h;
          *reinterpret_cast<float4*>(smem + s * S::STAGE + S::A_STAGE + off) = l;
        }
      }
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(&bars->full[s]);
    };
    for (int64_t w = blockIdx.x; w < a.nitems; w += gridDim.x) {
      const TcItem2 I = a.items[w];
      const int64_t zc0 = (int64_t)(I.zb / KE) * KE;
      const int nk = (int)((I.ze - zc0 + KC - 1) / KC);
      for (int kc = 0; kc < nk; ++kc, ++it) {
        const int s = (int)(it % TC_STAGES);
        const uint32_t ph = (it / TC_STAGES) & 1u;
        if (!tc::mbar_wait(&bars->empty[s], ph ^ 1u, TC_WAIT)) { tc_fail(a.err, bars, 1); break; }
        if (tc_aborted(bars)) break;
        const uint32_t abase = sbase + s * S::STAGE;
        const int64_t zc = zc0 + (int64_t)kc * KC;
        if (tid == 0) {
          tc::mbar_arrive_expect_tx(&bars->full[s], S::B_STAGE);
          tc::bulk_g2s(abase + S::A_STAGE + S::A_LO, a.zt + (zc / KE) * (2 * NC * KE), S::B_STAGE, &bars->full[s]);
        }
        // chunk ci = tid + 128 (j % 4) of tile j / 4: rows KE g.. of K column k
        int64_t zcur = -1;
        TcZ2 Z{};
#pragma unroll
        for (int j = 0; j < TC_T * 4; ++j) {
          const int t = j / 4;
          const int ci = tid + TC_PROD * (j % 4);
          int g, k;
          const uint32_t coff = a2_chunk<KE>(ci, g, k);
          const int64_t zp = zc + k;
          uint8_t* dsm = smem + s * S::STAGE + t * S::A_TILE + coff;
          const uint32_t dst = abase + (uint32_t)(t * S::A_TILE) + coff;
          if (zp < (int64_t)I.zb || zp >= (int64_t)I.ze) {
            *reinterpret_cast<uint4*>(dsm) = make_uint4(0u, 0u, 0u, 0u);
            continue;
          }
          if (zp != zcur) { Z = a.z2[zp]; zcur = zp; }
          const int i0 = t * 128 + g * KE;               // first window row of the chunk
          const int64_t so = Z.a_off + (i0 - Z.rlo);     // source element of row i0
          if (i0 >= Z.rlo && i0 + KE <= Z.rhi && (so % KE) == 0) {
            tc::cp_async16(dst, a.pool + so, 16u);
          } else if (i0 + KE <= Z.rlo || i0 >= Z.rhi) {
            *reinterpret_cast<uint4*>(dsm) = make_uint4(0u, 0u, 0u, 0u);
          } else {
            // a partly covered or unaligned row group: element by element
            union { typename Tr::Bits e[KE]; uint4 u; } v;
#pragma unroll
            for (int e = 0; e < KE; ++e) {
              const int i = i0 + e;
              v.e[e] = 0;
              if (i >= Z.rlo && i < Z.rhi)
                v.e[e] = *reinterpret_cast<const typename Tr::Bits*>(a.pool + Z.a_off + (i - Z.rlo));
            }
            *reinterpret_cast<uint4*>(dsm) = v.u;
          }
        }
        tc::cp_async_commit();
        if (it >= TC_STAGES - 1) {
          tc::cp_async_wait<TC_STAGES - 1>();
          finish(fin++);
        }
      }
      if (tc_aborted(bars)) break;
    }
    tc::cp_async_wait<0>();
    while (fin < it) finish(fin++);
  } else if (warp == 8) {
    if (lane == 0) {
      constexpr uint32_t LBO_B = 2 * NC * 16, SBO_B = 128;
      const uint32_t id_full = tc::idesc(Tr::FMT, 2 * NC, 1, 0);
      const uint32_t id_half = tc::idesc(Tr::FMT, NC, 1, 0);
      uint32_t it = 0, item = 0;
      bool ok = true;
      for (int64_t w = blockIdx.x; w < a.nitems && ok; w += gridDim.x, ++item) {
        const TcItem2 I = a.items[w];
        const int64_t zc0 = (int64_t)(I.zb / KE) * KE;
        const int nk = (int)((I.ze - zc0 + KC - 1) / KC);
        const int ntile = (int)((I.nrows + 127) / 128);
        if (!tc::mbar_wait(&bars->acc_empty, (item & 1u) ^ 1u, TC_WAIT)) { tc_fail(a.err, bars, 2); ok = false; break; }
        tc::tc_fence_after();
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = (int)(it % TC_STAGES);
          const uint32_t ph = (it / TC_STAGES) & 1u;
          if (!tc::mbar_wait(&bars->full[s], ph, TC_WAIT)) { tc_fail(a.err, bars, 4); ok = false; break; }
          tc::tc_fence_after();
          const uint32_t abase = sbase + s * S::STAGE;
          const uint32_t bbase = abase + S::A_STAGE + S::A_LO;
          for (int t = 0; t < ntile; ++t) {
#pragma unroll
            for (int ks = 0; ks < TC_KB / 2; ++ks) {
              const uint64_t bd = tc::smem_desc(bbase + ks * 2 * LBO_B, LBO_B, SBO_B);
              const uint64_t ad = a2_desc<KE>(abase + t * S::A_TILE, ks);
              tc::mma<Tr::KIND>(tmem + t * 2 * NC, ad, bd, id_full, (kc > 0 || ks > 0) ? 1u : 0u);
              if constexpr (Tr::SPLIT) {
                const uint64_t al = a2_desc<KE>(abase + S::A_STAGE + t * S::A_TILE, ks);
                tc::mma<Tr::KIND>(tmem + t * 2 * NC, al, bd, id_half, 1u);
              }
            }
          }
          tc::mma_commit(&bars->empty[s]);
        }
        if (ok) tc::mma_commit(&bars->acc_full);
      }
      tc_mma_drain(bars, a.err);
    }
  } else {
    const int ew = warp - 4;
    uint32_t item = 0;
    for (int64_t w = blockIdx.x; w < a.nitems; w += gridDim.x, ++item) {
      const TcItem2 I = a.items[w];
      if (!tc::mbar_wait(&bars->acc_full, item & 1u, TC_WAIT)) { tc_fail(a.err, bars, 8); break; }
      tc::tc_fence_after();
      const int ntile = (int)((I.nrows + 127) / 128);
      for (int t = 0; t < ntile; ++t) {
        const uint32_t row = (uint32_t)(t * 128 + 32 * ew + lane);
        const bool valid = row < I.nrows;
        double* yr = a.Y + (int64_t)I.row0 + row;
#pragma unroll
        for (int j0 = 0; j0 < NC; j0 += 16) {
          float d0[16], d1[16];
          const uint32_t ta = tmem + ((uint32_t)(32 * ew) << 16) + (uint32_t)(t * 2 * NC + j0);
          tc::tmem_ld16(ta, d0);
          tc::tmem_ld16(ta + NC, d1);
          if (valid) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int col = a.cb * NC + j0 + j;
              if (col < a.ncols) yr[(int64_t)col * a.ldy] += (double)(d0[j] + d1[j]);
            }
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&bars->acc_empty);
    }
  }
  tc_teardown(bars, warp, tmem, S::TMEM_COLS);
}

// ---------------------------------------------------------------------------
// Self-test of the operand layouts and descriptors used above: one 128 x 2NC
// accumulator D = A B' over one pipeline stage's K, with A staged exactly as
// phase 1 (K-major) or phase 2 (M-major) stage it and B as the X / Z tiles.
// The tiles sit at the start of a 200 KB shared allocation (A at 0, B at
// 96 KB), far inside it, so every address the descriptors can produce stays
// in the allocation.
// ---------------------------------------------------------------------------
constexpr int SELF_SMEM = 200 * 1024;
constexpr int SELF_B_OFF = 96 * 1024;

template <typename T, int NC, bool A_MN>
__global__ void __launch_bounds__(128, 1) tc_selftest_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                           float* __restrict__ D, int* __restrict__ err) {
  using Tr = TcT<T>;
  constexpr int KE = Tr::KE;
  constexpr int KC = TC_KB * KE;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  typename Tr::Bits* sa = reinterpret_cast<typename Tr::Bits*>(smem);
  typename Tr::Bits* sb = reinterpret_cast<typename Tr::Bits*>(smem + SELF_B_OFF);
  // A (128 x KC, row-major input) in the tile layout of the kernels
  for (int e = tid; e < 128 * KC; e += 128) {
    const int i = e / KC, k = e % KC;
    int off;                                           // element offset in the tile
    if (!A_MN) {
      // phase 1: row i, K block b: (i / 8) * KB * 128 + b * 128 + (i % 8) * 16 bytes
      off = ((i / 8) * TC_KB * 128 + (k / KE) * 128 + (i % 8) * 16) / (int)sizeof(T) + k % KE;
    } else {
      // phase 2: the chunk of rows KE g .. of column k, laid out by a2_chunk
      int ci = 0;
      if (KE == 8) ci = (k / 8) * 128 + ((i / KE) % 16) * 8 + (k % 8);
      else ci = ((i / KE) / 8) * 128 + (k % 16) * 8 + (i / KE) % 8;
      int gg, kk;
      off = (int)(a2_chunk<KE>(ci, gg, kk) / sizeof(T)) + i % KE;
    }
    sa[off] = Tr::bits(A[e]);
  }
  // B (2NC x KC, row-major input) as XT / ZT blocks: [b][n][e]
  for (int e = tid; e < 2 * NC * KC; e += 128) {
    const int nn = e / KC, k = e % KC;
    sb[(k / KE) * (2 * NC * KE) + nn * KE + k % KE] = Tr::bits(B[e]);
  }
  if (tid == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  tc::fence_proxy_async_smem();
  if (warp == 0) tc::tmem_alloc(&tslot, 2 * NC < 32 ? 32 : 2 * NC);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tslot;
  if (tid == 0) {
    const uint32_t abase = tc::smem_u32(smem), bbase = tc::smem_u32(smem + SELF_B_OFF);
    constexpr uint32_t LBO_B = 2 * NC * 16, SBO_B = 128;
    const uint32_t id = tc::idesc(Tr::FMT, 2 * NC, A_MN ? 1 : 0, 0);
#pragma unroll
    for (int ks = 0; ks < TC_KB / 2; ++ks) {
      const uint64_t bd = tc::smem_desc(bbase + ks * 2 * LBO_B, LBO_B, SBO_B);
      uint64_t ad;
      if (!A_MN) ad = tc::smem_desc(abase + ks * 2 * 128, 128, TC_KB * 128);
      else ad = a2_desc<KE>(abase, ks);
      tc::mma<Tr::KIND>(tmem, ad, bd, id, ks > 0 ? 1u : 0u);
    }
    tc::mma_commit(&bar);
  }
  __syncwarp();
  if (!tc::mbar_wait(&bar, 0u, TC_WAIT) && lane == 0) atomicOr(err, 1);
  tc::tc_fence_after();
  for (int j0 = 0; j0 < 2 * NC; j0 += 16) {
    float d[16];
    tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)j0, d);
#pragma unroll
    for (int j = 0; j < 16; ++j) D[(32 * warp + lane) * 2 * NC + j0 + j] = d[j];
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 2 * NC < 32 ? 32 : 2 * NC);
  }
}

template <typename T, int NC, bool A_MN>
int run_selftest(const float* A, const float* B, float* D) {
  constexpr int KC = TC_KB * TcT<T>::KE;
  float *dA = nullptr, *dB = nullptr, *dD = nullptr;
  int* dE = nullptr;
  struct Guard {
    void** p[4];
    ~Guard() { for (void** q : p) if (*q) cudaFree(*q); }
  } guard{{(void**)&dA, (void**)&dB, (void**)&dD, (void**)&dE}};
  HM_CUDA_TRY(cudaMalloc(&dA, sizeof(float) * 128 * KC));
  HM_CUDA_TRY(cudaMalloc(&dB, sizeof(float) * 2 * NC * KC));
  HM_CUDA_TRY(cudaMalloc(&dD, sizeof(float) * 128 * 2 * NC));
  HM_CUDA_TRY(cudaMalloc(&dE, sizeof(int)));
  HM_CUDA_TRY(cudaMemset(dE, 0, sizeof(int)));
  HM_CUDA_TRY(cudaMemcpy(dA, A, sizeof(float) * 128 * KC, cudaMemcpyHostToDevice));
  HM_CUDA_TRY(cudaMemcpy(dB, B, sizeof(float) * 2 * NC * KC, cudaMemcpyHostToDevice));
  HM_CUDA_TRY(smem_attr((const void*)tc_selftest_kernel<T, NC, A_MN>, SELF_SMEM));
  tc_selftest_kernel<T, NC, A_MN><<<1, 128, SELF_SMEM>>>(dA, dB, dD, dE);
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaDeviceSynchronize());
  int e = 0;
  HM_CUDA_TRY(cudaMemcpy(&e, dE, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(HM_ERR_TIMEOUT, "tensor-core self-test: the MMA did not complete");
  HM_CUDA_TRY(cudaMemcpy(D, dD, sizeof(float) * 128 * 2 * NC, cudaMemcpyDeviceToHost));
  return HM_OK;
}

}  // namespace

int tc_selftest(int kind, int a_mn, int nc, const float* A, const float* B, float* D) {
  if (kind == 0) {
    if (nc == 16) return a_mn ? run_selftest<float, 16, true>(A, B, D) : run_selftest<float, 16, false>(A, B, D);
    if (nc == 64) return a_mn ? run_selftest<float, 64, true>(A, B, D) : run_selftest<float, 64, false>(A, B, D);
  } else {
    if (nc == 16)
      return a_mn ? run_selftest<__nv_bfloat16, 16, true>(A, B, D) : run_selftest<__nv_bfloat16, 16, false>(A, B, D);
    if (nc == 64)
      return a_mn ? run_selftest<__nv_bfloat16, 64, true>(A, B, D) : run_selftest<__nv_bfloat16, 64, false>(A, B, D);
  }
  return fail(HM_ERR_ARG, "self-test: kind 0 (tf32) or 1 (bf16), nc 16 or 64");
}

// ---------------------------------------------------------------------------
// plan: built on the host once per direction, on first use
// ---------------------------------------------------------------------------
void free_tc_plan(TcPlan*& p) {
  if (!p) return;
  if (p->d_col1) cudaFree(p->d_col1);
  if (p->d_item1) cudaFree(p->d_item1);
  if (p->d_zpl) cudaFree(p->d_zpl);
  if (p->d_z2) cudaFree(p->d_z2);
  if (p->d_item2) cudaFree(p->d_item2);
  delete p;
  p = nullptr;
}

template <typename V>
static int upload_vec(V** d, const std::vector<V>& v) {
  *d = nullptr;
  if (v.empty()) return HM_OK;
  cudaError_t e = cudaMalloc((void**)d, sizeof(V) * v.size());
  if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("tensor-core matvec plan: ") + cudaGetErrorString(e));
  HM_CUDA_TRY(cudaMemcpy(*d, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice));
  return HM_OK;
}

static int build_tc_plan(hm_handle* h, int trans, TcPlan** out) {
  const int eb = elem_bytes(h->storage);
  struct Lf { int64_t li; int64_t zoff; };
  // low-rank leaves in pool order with their z offsets (the order of the
  // CUDA-core plans: leaves sorted by row group)
  std::vector<int64_t> order(h->leaves.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int64_t)i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
    return h->leaves[x].off < h->leaves[y].off;
  });
  std::vector<Lf> rk;
  int64_t z = 0;
  for (int64_t li : order) {
    const Leaf& L = h->leaves[li];
    if (L.type != T_RK || L.k == 0) continue;
    rk.push_back({li, z});
    z += L.k;
  }
  const int64_t zlen = z;
  TcPlan* P = new TcPlan();
  // ---- phase 2: windows of TC_WR output rows; Z slots window by window
  const int64_t n = h->n;
  const int64_t nwin = (n + TC_WR - 1) / TC_WR;
  std::vector<std::vector<int32_t>> per(nwin);      // rk indices touching each window
  for (size_t i = 0; i < rk.size(); ++i) {
    const Leaf& L = h->leaves[rk[i].li];
    const int64_t o0 = trans ? L.col0 : L.row0, o1 = o0 + (trans ? L.n : L.m);
    for (int64_t w = o0 / TC_WR; w * TC_WR < o1; ++w) per[w].push_back((int32_t)i);
  }
  std::vector<TcZ2> z2;
  std::vector<TcItem2> it2;
  std::vector<uint32_t> zp_count(zlen + 1, 0);        // Z slots of each z, then prefix
  for (int64_t w = 0; w < nwin; ++w)
    for (int32_t i : per[w]) {
      const Leaf& L = h->leaves[rk[i].li];
      for (int r = 0; r < L.k; ++r) zp_count[rk[i].zoff + r + 1]++;
    }
  for (int64_t q = 0; q < zlen; ++q) zp_count[q + 1] += zp_count[q];
  std::vector<uint32_t> zpl(zp_count[zlen]), fillpos(zp_count.begin(), zp_count.end() - 1);
  for (int64_t w = 0; w < nwin; ++w) {
    if (per[w].empty()) continue;
    TcItem2 I{};
    I.row0 = (uint32_t)(w * TC_WR);
    I.nrows = (uint32_t)std::min<int64_t>(TC_WR, n - w * TC_WR);
    I.zb = (uint32_t)z2.size();
    for (int32_t i : per[w]) {
      const Leaf& L = h->leaves[rk[i].li];
      const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
      const int64_t o0 = trans ? L.col0 : L.row0, o1 = o0 + (trans ? L.n : L.m);
      const int64_t lo = std::max<int64_t>(o0, w * TC_WR), hi = std::min<int64_t>(o1, (w + 1) * TC_WR);
      for (int r = 0; r < L.k; ++r) {
        // F2: A (m x k, stride mpad) for H*x, B (n x k, stride npad) for H'*x
        const int64_t col = trans ? L.off + (int64_t)r * npad : L.off + npad * L.k + (int64_t)r * mpad;
        TcZ2 Z{};
        Z.a_off = col + (lo - o0);
        Z.rlo = (int32_t)(lo - w * TC_WR);
        Z.rhi = (int32_t)(hi - w * TC_WR);
        if ((o0 % (16 / eb)) != 0) P->aligned = false;
        zpl[fillpos[rk[i].zoff + r]++] = (uint32_t)z2.size();
        z2.push_back(Z);
      }
    }
    I.ze = (uint32_t)z2.size();
    it2.push_back(I);
    std::vector<int32_t>().swap(per[w]);
  }
  if (z2.size() > (size_t)UINT32_MAX / 2) { delete P; return fail(HM_ERR_UNSUPPORTED, "too many low-rank terms for the tensor-core plan"); }
  // ---- phase 1: factor columns of F1 grouped by input segment
  std::vector<int32_t> ord1(rk.size());
  for (size_t i = 0; i < rk.size(); ++i) ord1[i] = (int32_t)i;
  auto seg = [&](int32_t i) {
    const Leaf& L = h->leaves[rk[i].li];
    return trans ? std::make_pair(L.row0, (int64_t)L.m) : std::make_pair(L.col0, (int64_t)L.n);
  };
  std::stable_sort(ord1.begin(), ord1.end(), [&](int32_t x, int32_t y) { return seg(x) < seg(y); });
  std::vector<TcCol1> col1;
  std::vector<TcItem1> it1;
  for (size_t i = 0; i < ord1.size();) {
    const auto sg = seg(ord1[i]);
    size_t j = i;
    const uint32_t c0 = (uint32_t)col1.size();
    while (j < ord1.size() && seg(ord1[j]) == sg) {
      const Leaf& L = h->leaves[rk[ord1[j]].li];
      const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
      for (int r = 0; r < L.k; ++r) {
        TcCol1 C{};
        C.off = trans ? (uint64_t)(L.off + npad * L.k + (int64_t)r * mpad) : (uint64_t)(L.off + (int64_t)r * npad);
        C.zp0 = zp_count[rk[ord1[j]].zoff + r];
        C.zp1 = zp_count[rk[ord1[j]].zoff + r + 1];
        col1.push_back(C);
      }
      ++j;
    }
    const uint32_t c1 = (uint32_t)col1.size();
    for (uint32_t c = c0; c < c1; c += 128 * TC_T) {
      TcItem1 I{};
      I.col0 = c;
      I.ncol = std::min<uint32_t>(128 * TC_T, c1 - c);
      I.seg0 = (uint32_t)sg.first;
      I.len = (uint32_t)sg.second;
      it1.push_back(I);
    }
    i = j;
  }
  P->ncol1 = (int64_t)col1.size();
  P->nitem1 = (int64_t)it1.size();
  P->nzpl = (int64_t)zpl.size();
  P->nz2 = (int64_t)z2.size();
  P->nitem2 = (int64_t)it2.size();
  int s = HM_OK;
  if (s == HM_OK) s = upload_vec(&P->d_col1, col1);
  if (s == HM_OK) s = upload_vec(&P->d_item1, it1);
  if (s == HM_OK) s = upload_vec(&P->d_zpl, zpl);
  if (s == HM_OK) s = upload_vec(&P->d_z2, z2);
  if (s == HM_OK) s = upload_vec(&P->d_item2, it2);
  if (s != HM_OK) { free_tc_plan(P); return s; }
  *out = P;
  return HM_OK;
}

// ---------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------
template <typename T, int NC>
static int launch_tc(hm_handle* h, TcPlan& P, const double* d_x, double* d_y, int64_t ncols, cudaStream_t st) {
  using Bits = typename TcT<T>::Bits;
  using S = TcSmem<T, NC>;
  constexpr int KE = TcT<T>::KE;
  const int64_t n = h->n;
  const int64_t nkb = (n + 2 * KE) / KE + TC_KB + 2;            // XT blocks per shifted copy
  const int64_t xt_copy = nkb * 2 * NC * KE;
  const int64_t zkb = (P.nz2 + KE - 1) / KE + TC_KB + 2;        // Z blocks (with zero padding)
  const size_t xt_bytes = sizeof(Bits) * (size_t)(KE * xt_copy);
  const size_t zt_bytes = sizeof(Bits) * (size_t)(zkb * 2 * NC * KE);
  const size_t need = xt_bytes + zt_bytes + 256;
  if (h->tc_bytes < need) {
    if (h->d_tc) cudaFree(h->d_tc);
    h->d_tc = nullptr;
    h->tc_bytes = 0;
    cudaError_t e = cudaMalloc(&h->d_tc, need);
    if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("tensor-core matvec buffers: ") + cudaGetErrorString(e));
    h->tc_bytes = need;
  }
  if (!h->d_tc_err) {
    HM_CUDA_TRY(cudaMalloc(&h->d_tc_err, sizeof(int)));
    HM_CUDA_TRY(cudaMemsetAsync(h->d_tc_err, 0, sizeof(int), st));
  }
  Bits* xt = (Bits*)h->d_tc;
  Bits* zt = (Bits*)((char*)h->d_tc + ((xt_bytes + 255) / 256) * 256);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  HM_CUDA_TRY(smem_attr((const void*)tc_phase1_kernel<T, NC>, S::BYTES));
  HM_CUDA_TRY(smem_attr((const void*)tc_phase2_kernel<T, NC>, S::BYTES));
  // Z padding past the last slot stays zero (its A columns are zero too, and
  // 0 * garbage could be NaN)
  {
    const int64_t z0 = (P.nz2 / KE) * (2 * NC * KE);
    const int64_t cnt = zkb * 2 * NC * KE - z0;
    tc_zero_kernel<T><<<(unsigned)std::min<int64_t>((cnt + 255) / 256, 1024), 256, 0, st>>>(zt + z0, cnt);
  }
  const int ncb = (int)((ncols + NC - 1) / NC);
  for (int cb = 0; cb < ncb; ++cb) {
    const int64_t tot = KE * xt_copy;
    tc_xt_kernel<T, NC><<<(unsigned)std::min<int64_t>((tot + 255) / 256, (int64_t)nsm * 32), 256, 0, st>>>(
        d_x, n, n, (int)ncols, cb, xt, nkb);
    if (P.nitem1 > 0) {
      P1Args<T, NC> a1{P.d_item1, P.nitem1, P.d_col1, P.d_zpl, (const T*)h->d_rk, xt, xt_copy, zt, h->d_tc_err};
      tc_phase1_kernel<T, NC><<<(unsigned)std::min<int64_t>(nsm, P.nitem1), TC_THREADS, S::BYTES, st>>>(a1);
    }
    if (P.nitem2 > 0) {
      P2Args<T, NC> a2{P.d_item2, P.nitem2, P.d_z2, (const T*)h->d_rk, zt, d_y, n, (int)ncols, cb, h->d_tc_err};
      tc_phase2_kernel<T, NC><<<(unsigned)std::min<int64_t>(nsm, P.nitem2), TC_THREADS, S::BYTES, st>>>(a2);
    }
  }
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

// column block NC: the autotuner's choice for this many columns, else the
// smallest block of 16, 32, 64 that holds them
template <typename T>
static int tc_dispatch(hm_handle* h, TcPlan& P, const double* d_x, double* d_y, int64_t ncols, cudaStream_t st) {
  const int bucket = ncols <= 16 ? 0 : (ncols <= 32 ? 1 : 2);
  int nc = h->tune.tc_nc[bucket];
  if (nc == 0) nc = bucket == 0 ? 16 : (bucket == 1 ? 32 : 64);
  if (nc == 16) return launch_tc<T, 16>(h, P, d_x, d_y, ncols, st);
  if (nc == 32) return launch_tc<T, 32>(h, P, d_x, d_y, ncols, st);
  return launch_tc<T, 64>(h, P, d_x, d_y, ncols, st);
}

// Y += the low-rank part of H X (H' X) on the tensor cores; the caller has
// written the dense part into Y.
int matvec_multi_tc(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st) {
  if (h->storage != HM_F32 && h->storage != HM_BF16)
    return fail(HM_ERR_UNSUPPORTED, "tensor-core matvec: FP32 or BF16 factors only");
  TcPlan*& P = trans ? h->tc_bwd : h->tc_fwd;
  if (!P) HM_TRY(build_tc_plan(h, trans, &P));
  if (h->storage == HM_F32) return tc_dispatch<float>(h, *P, d_x, d_y, ncols, st);
  return tc_dispatch<__nv_bfloat16>(h, *P, d_x, d_y, ncols, st);
}

// Reads (and clears) the error word of the tensor-core kernels: non-zero
// when a bounded wait gave up.
int tc_status(hm_handle* h, cudaStream_t st) {
  if (!h->d_tc_err) return HM_OK;
  int v = 0;
  HM_CUDA_TRY(cudaMemcpyAsync(&v, h->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  if (v != 0) {
    HM_CUDA_TRY(cudaMemsetAsync(h->d_tc_err, 0, sizeof(int), st));
    return fail(HM_ERR_TIMEOUT, "tensor-core matvec: a pipeline wait gave up (code " + std::to_string(v) + ")");
  }
  return HM_OK;
}

}  // namespace hm
