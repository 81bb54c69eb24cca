// Multi-RHS H-matvec on the 5th-generation tensor cores (tcgen05, sm_100a):
// Y = H X (or H' X) for an n x c block of right-hand sides with FP32 or BF16
// stored factors, the device form of *(Hmat, Matrix) (src/harithm.jl:
// 317-329), which the reference evaluates one column at a time.
//
// Phase 1 (Z = F1' X_seg): the factor columns of the low-rank leaves that
//   share one input segment are cut into 128-column M-tiles; one tcgen05 MMA
//   chain per tile computes Z_tile = F1_tile' X_seg (K = segment points,
//   N = right-hand-side columns) into a TMEM accumulator.
// Phase 2 (Y += F2 Z): an output window of 512 rows keeps its Z slots (the k
//   values of every leaf that touches the window) contiguous; one MMA chain
//   per 128-row tile of a window runs K over the window's slots.  The dense
//   leaves are added by the CUDA-core block kernel first.
//
// Data movement.  Factor columns are contiguous in the pool, so a pipeline
// stage takes one contiguous piece of each factor column it needs (phase 1:
// KC values = 256 bytes of each of the tile's 128 columns; phase 2: the
// tile's rows of each of KC columns) into a raw shared-memory stage, by
// 16-byte cp.async gathers of four producer warps (16 lanes per 256-byte
// piece, so every warp instruction reads whole 128-byte lines) whose
// completion arrives on the stage's mbarrier without blocking the producers
// (cp.async.mbarrier.arrive.noinc).  A 1-D bulk copy per factor column would
// be simpler, but each lane's bulk copy issues separately (about 80 cycles a
// copy measured), which capped a single producer warp near 1 TB/s.  The X / Z
// tile of the stage, one contiguous block pre-tiled in the MMA's K-major
// core-matrix layout, arrives by one bulk copy of the TMA engine.  Converter warps read the
// raw stage row by row (one TMEM lane per thread), split FP32 values into TF32
// hi and lo parts, and write the A operand straight into tensor memory
// (tcgen05.st); the MMA reads A from TMEM and B from shared memory.  Shared
// memory thus carries each factor byte twice (bulk-copy write, converter read)
// instead of five times when hi/lo operand tiles are staged in shared memory.
//
// Accuracy.  FP32 factors use three TF32 products per term (F_hi X_hi +
// F_hi X_lo + F_lo X_hi, the split of Ootomo & Yokota 2022), BF16 factors
// are exact in BF16 and X is split into two BF16 parts (F X_1 + F X_2); the
// accumulation is FP32 in TMEM, and the FP32 sums are added into FP64 Y.
// Both splits round to nearest and leave exact values of the narrow format,
// so the hardware's own input conversion does not matter.
//
// Roles per CTA (persistent, one per SM, 13 warps): warps 8-11 produce stages;
// warps 0-7 convert them into two TMEM A buffers (warp w: TMEM lanes
// 32 (w % 4) .., the K half w / 4 of each stage, two converter warps per SM
// sub-partition) and drain the accumulator of the previous tile (tcgen05.ld)
// once its MMAs are known to be done; warp 12 issues the MMAs (one thread).
// The two TMEM accumulators alternate between tiles.  mbarriers link
// the roles; every wait is bounded, and a timeout sets an error word and ends
// the kernel cleanly once the copies and MMAs in flight have finished.
#include "hm_internal.h"
#include "hm_tc.cuh"

#include <algorithm>
#include <vector>

namespace hm {

struct TcCol1 {            // phase-1 M row: one factor column of F1
  uint64_t off;            // pool element offset of the column's first entry
  uint32_t zp0, zp1;       // its Z slots: zpl[zp0 .. zp1)
};
struct TcItem1 {           // one tile of up to 128 columns of one input segment
  uint32_t col0, ncol;     // columns [col0, col0 + ncol) of the column table
  uint32_t seg0, len;      // input index range of the segment
};
struct TcZ2 {              // phase-2 K column (a Z slot) inside its window
  int64_t a_off;           // pool element offset of F2 at window row rlo
  int32_t rlo, rhi;        // rows [rlo, rhi) of the window it covers
};
struct TcItem2 {           // one tile of up to 128 rows of an output window
  uint32_t row0, nrows;    // first output row of the tile, its rows
  uint32_t zb, ze;         // the window's Z slots [zb, ze)
  uint32_t toff;           // row offset of the tile inside its window
  uint32_t pad;
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
  bool checked = false;    // `usable` is up to date with the factor pool
  bool usable = false;     // every factor entry is at most 2^100 in magnitude (no NaN)
};

namespace {

constexpr int TC_WR = 512;           // rows of a phase-2 window
constexpr int TC_PW = 4;                          // producer warps
constexpr int TC_MMA_WARP = 8 + TC_PW;             // warps 0-7 convert + drain, 8 .. produce, then MMA
constexpr int TC_THREADS = 32 * (TC_MMA_WARP + 1);
constexpr int TC_PROD0 = 256;                      // first producer thread
constexpr int TC_NPROD = 32 * TC_PW;
constexpr int TC_NA_MAX = 4;         // TMEM A buffers, at most
constexpr int TC_TMEM_COLS = 512;    // one CTA per SM (shared memory), so all of TMEM
constexpr uint32_t TC_WAIT = 1u << 22;   // polls of a bounded mbarrier wait
// Phase 2 adds its FP32 accumulator into the FP64 Y every NC / 2 stages
// (32 NC Z slots for FP32 factors, 64 NC for BF16): a window's K runs over
// every leaf that touches it (thousands of terms at n = 2^20), and one FP32 sum
// over all of them would lose accuracy as n grows.  The segment grows with the
// column block so that the Y traffic of the adds (16 NC bytes a tile row) stays
// an eighth of the factor bytes a segment streams.
template <int NC> constexpr int tc_kseg2() { return NC / 2; }

template <typename T> struct TcT;
template <> struct TcT<float> {
  static constexpr int KE = 4;                      // elements per 16 bytes
  static constexpr int KC = 64;                     // K values per stage (256 bytes of a column)
  static constexpr int KM = 8;                      // K values per MMA
  static constexpr int ACOLS = 2 * KC;              // TMEM columns of an A buffer: hi | lo
  static constexpr int KIND = 0;                    // kind::tf32
  static constexpr int FMT = tc::FMT_TF32;
  static constexpr bool SPLIT = true;               // A = A_hi + A_lo
  static constexpr int SIG = 11;                    // significant bits of the narrow format
  static constexpr int SHIFT = 0;                   // its bits: the FP32 pattern >> SHIFT
  using Bits = uint32_t;
  __device__ static float hi(float x) { return tc::tf32_rn(x); }
  __device__ static Bits bits(float x) { return __float_as_uint(x); }
};
template <> struct TcT<__nv_bfloat16> {
  static constexpr int KE = 8;
  static constexpr int KC = 128;
  static constexpr int KM = 16;
  static constexpr int ACOLS = KC / 2;              // two BF16 values per 32-bit column
  static constexpr int KIND = 1;                    // kind::f16, BF16 inputs
  static constexpr int FMT = tc::FMT_BF16;
  static constexpr bool SPLIT = false;              // BF16 factors are exact
  static constexpr int SIG = 8;
  static constexpr int SHIFT = 16;
  using Bits = uint16_t;
  __device__ static float hi(float x) { return tc::bf16_rn(x); }
  __device__ static Bits bits(float x) { return (uint16_t)(__float_as_uint(x) >> 16); }
};

// shared memory and TMEM of one CTA
template <typename T, int NC>
struct TcCfg {
  using Tr = TcT<T>;
  static constexpr int KE = Tr::KE, KC = Tr::KC, ES = (int)sizeof(T);
  static constexpr int S = NC <= 16 ? 5 : (NC <= 32 ? 4 : 3);   // pipeline stages
  static constexpr int B_BYTES = KC * 2 * NC * ES;           // the X / Z tile of a stage (hi | lo parts)
  static constexpr int RS1 = KC * ES + 16;                   // phase-1 raw row: one column's KC values (+16: banks)
  static constexpr int RAW1 = 128 * RS1;
  static constexpr int RS2 = (128 + KE) * ES;                // phase-2 raw row: one slot's 128 rows (+KE: shift)
  static constexpr int RAW2 = KC * RS2;
  static constexpr int META = KC * 16;                       // phase-2 slot table: rows [lo, hi), word offset
  static constexpr int RAW = RAW1 > RAW2 + META ? RAW1 : RAW2 + META;
  static constexpr int STAGE = (B_BYTES + RAW + 1023) / 1024 * 1024;
  static constexpr int BAR_OFF = S * STAGE;
  static constexpr int BYTES = BAR_OFF + 512;
  // Accumulation chains: the MMAs into one accumulator run one after the
  // other, and a chain of small MMAs (N = 2 NC) is slower than the stream of
  // factor bytes; two independent accumulators per tile (FP32: the hi and the
  // lo products; BF16: even and odd K steps) halve the chain, where TMEM
  // holds them beside two A buffers.  An accumulator buffer is ACCW columns:
  // chain 0 (2 NC) then chain 1 (NC for the lo products, 2 NC for BF16).
  static constexpr int ACCW2 = 2 * NC + (Tr::SPLIT ? NC : 2 * NC);
  static constexpr int NCH = 2 * Tr::ACOLS + 2 * ACCW2 <= TC_TMEM_COLS ? 2 : 1;
  static constexpr int ACCW = NCH == 2 ? ACCW2 : 2 * NC;
  // as many TMEM A buffers as fit beside the two accumulator buffers (at most
  // 4): the converters run up to NA stages ahead of the MMAs' completion
  static constexpr int NA_FIT = (TC_TMEM_COLS - 2 * ACCW) / Tr::ACOLS;
  static constexpr int NA = NA_FIT < TC_NA_MAX ? NA_FIT : TC_NA_MAX;
  static constexpr int ACC0 = NA * Tr::ACOLS;                // first accumulator column
  static_assert(NA >= 2, "two A buffers at least");
  static_assert(BYTES <= 227 * 1024, "stages exceed the shared memory of a CTA");
  static_assert(ACC0 + 2 * ACCW <= TC_TMEM_COLS, "A buffers and accumulators exceed TMEM");
  static_assert(RS1 % 16 == 0 && RS2 % 16 == 0 && B_BYTES % 16 == 0, "bulk copies move 16-byte units");
  static_assert(KC % TC_PW == 0 && KC % Tr::KM == 0, "a stage is whole MMAs and whole producer warps");
};

struct TcBars {
  uint64_t full[5];        // raw stage landed (the producers' cp.async arrivals)
  uint64_t bfull[5];       // the stage's B tile landed (bulk-copy bytes + one arrival)
  uint64_t empty[5];       // the MMAs that read the stage's B tile finished (tcgen05.commit)
  uint64_t afull[TC_NA_MAX];   // A buffer written (256 converter threads)
  uint64_t aempty[TC_NA_MAX];  // the MMAs that read the A buffer finished
  uint64_t accfull[2];     // accumulator complete (commit after a tile's last MMA)
  uint64_t accempty[2];    // accumulator drained (256 converter threads)
  uint64_t done;           // the MMA issuer's last commit: every MMA finished
  uint32_t tmem;
  int abort;
};
static_assert(sizeof(TcBars) <= 512, "barrier block");
static_assert((TcT<float>::KE & (TcT<float>::KE - 1)) == 0 && (TcT<__nv_bfloat16>::KE & (TcT<__nv_bfloat16>::KE - 1)) == 0,
              "K blocks of a power-of-two size");
static_assert(TcT<float>::KC * 4 == 256 && TcT<__nv_bfloat16>::KC * 2 == 256, "phase-1 pieces are 16 x 16 bytes");

__device__ __forceinline__ void tc_fail(int* err, TcBars* b, int code) {
  atomicOr(&b->abort, 1);
  atomicOr(err, code);
}
__device__ __forceinline__ bool tc_aborted(const TcBars* b) { return *(volatile const int*)&b->abort != 0; }

// Bounded wait that also gives up once another role has aborted; a timeout
// records `code`.
__device__ __forceinline__ bool tc_wait(TcBars* b, uint64_t* bar, uint32_t parity, int* err, int code) {
  for (uint32_t i = 0; i < TC_WAIT; ++i) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 63u && tc_aborted(b)) return false;
  }
  tc_fail(err, b, code);
  return false;
}
// the same for a whole warp: every lane waits, the outcome is uniform
__device__ __forceinline__ bool tc_wait_warp(TcBars* b, uint64_t* bar, uint32_t parity, int* err, int code) {
  const bool ok = tc_wait(b, bar, parity, err, code);
  return __all_sync(0xffffffffu, ok) != 0;
}

// barriers, TMEM; called by all threads.  full_count: arrivals that complete
// a raw stage.
__device__ __forceinline__ uint32_t tc_setup(TcBars* b, int warp, int nstage, uint32_t full_count) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < nstage; ++s) {
      tc::mbar_init(&b->full[s], full_count);
      tc::mbar_init(&b->bfull[s], 1);
      tc::mbar_init(&b->empty[s], 1);
    }
    for (int q = 0; q < TC_NA_MAX; ++q) {
      tc::mbar_init(&b->afull[q], 256);
      tc::mbar_init(&b->aempty[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      tc::mbar_init(&b->accfull[q], 1);
      tc::mbar_init(&b->accempty[q], 256);
    }
    tc::mbar_init(&b->done, 1);
    b->abort = 0;
    tc::fence_mbar_init();
  }
  if (warp == 4) tc::tmem_alloc(&b->tmem, TC_TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  return b->tmem;
}

// end of the kernel: copies and MMAs have finished; free TMEM
__device__ __forceinline__ void tc_teardown(TcBars* b, int warp, uint32_t tmem) {
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, TC_TMEM_COLS);
  }
}

// The B-tile producer's last step: every bulk copy it issued has landed.  The
// wait ignores an abort (shared memory must not be released under copies in
// flight) but stays bounded.  `it` stages were issued, stage s last by the
// largest iteration below `it` that is s mod nstage.
__device__ __forceinline__ void tc_copies_drain(TcBars* b, uint32_t it, int nstage, int* err) {
  for (int s = 0; s < nstage && (uint32_t)s < it; ++s) {
    const uint32_t last = it - 1 - ((it - 1 - (uint32_t)s) % (uint32_t)nstage);
    if (!tc::mbar_wait(&b->bfull[s], (last / (uint32_t)nstage) & 1u, TC_WAIT)) tc_fail(err, b, 32);
  }
}

// MMA issuer (one thread): per tile, K stages of A (TMEM) x B (shared
// memory); nk_of(w) gives tile w's stages.  Every kseg stages of a tile form
// one accumulation segment: a fresh accumulator (q = segment parity) that the
// converters drain when it completes.
template <typename T, int NC, typename NkOf>
__device__ __forceinline__ void tc_mma_role(TcBars* b, uint32_t sbase, uint32_t tmem, int64_t nitems, NkOf nk_of,
                                            int kseg, int* err) {
  using Tr = TcT<T>;
  using C = TcCfg<T, NC>;
  constexpr uint32_t LBO_B = 2 * NC * 16, SBO_B = 128;        // K-major [hi | lo] B tiles
  const uint32_t id_full = tc::idesc(Tr::FMT, 2 * NC, 0, 0);
  const uint32_t id_half = tc::idesc(Tr::FMT, NC, 0, 0);
  uint32_t it = 0, j = 0;                                      // stages, segments
  bool ok = true;
  int nk = blockIdx.x < nitems ? nk_of(blockIdx.x) : 0;
  for (int64_t w = blockIdx.x; w < nitems && ok; w += gridDim.x) {
    const int nk_next = w + gridDim.x < nitems ? nk_of(w + gridDim.x) : 0;   // loaded ahead of its use
    for (int k0 = 0; k0 < nk && ok; k0 += kseg, ++j) {
      const int k1 = min(nk, k0 + kseg);
      const uint32_t q = j & 1u;
      if (!tc_wait(b, &b->accempty[q], ((j >> 1) & 1u) ^ 1u, err, 2)) { ok = false; break; }
      tc::tc_fence_after();
      const uint32_t dacc = tmem + (uint32_t)C::ACC0 + q * C::ACCW;
      for (int kc = k0; kc < k1; ++kc, ++it) {
        const int s = (int)(it % C::S), a = (int)(it % C::NA);
        if (!tc_wait(b, &b->bfull[s], (it / C::S) & 1u, err, 4)) { ok = false; break; }
        if (!tc_wait(b, &b->afull[a], (it / C::NA) & 1u, err, 4)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t bbase = sbase + (uint32_t)(s * C::STAGE);
        const uint32_t abuf = tmem + (uint32_t)(a * Tr::ACOLS);
#pragma unroll
        for (int ks = 0; ks < Tr::KC / Tr::KM; ++ks) {
          const uint64_t bd = tc::smem_desc(bbase + ks * 2 * LBO_B, LBO_B, SBO_B);
          if constexpr (Tr::SPLIT) {
            // hi products into chain 0, lo products into chain 1 (or chain 0)
            tc::mma_ts<Tr::KIND>(dacc, abuf + ks * 8, bd, id_full, (kc > k0 || ks > 0) ? 1u : 0u);
            if constexpr (C::NCH == 2)
              tc::mma_ts<Tr::KIND>(dacc + 2 * NC, abuf + Tr::KC + ks * 8, bd, id_half, (kc > k0 || ks > 0) ? 1u : 0u);
            else
              tc::mma_ts<Tr::KIND>(dacc, abuf + Tr::KC + ks * 8, bd, id_half, 1u);
          } else {
            // K steps alternate between the chains
            const uint32_t ch = C::NCH == 2 ? (uint32_t)(ks & 1) : 0u;
            tc::mma_ts<Tr::KIND>(dacc + ch * 2 * NC, abuf + ks * 8, bd, id_full,
                                 (kc > k0 || ks >= C::NCH) ? 1u : 0u);
          }
        }
        tc::mma_commit(&b->empty[s]);
        tc::mma_commit(&b->aempty[a]);
      }
      if (ok) tc::mma_commit(&b->accfull[q]);
    }
    nk = nk_next;
  }
  tc::mma_commit(&b->done);
  if (!tc::mbar_wait(&b->done, 0u, TC_WAIT)) tc_fail(err, b, 16);
}

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

// max |x| over the factor pool as an FP32 bit pattern (NaN sorts above every
// number): the converters split without a magnitude check, which is exact
// while |x| <= 2^100
template <typename T>
__global__ void pool_maxabs_kernel(const T* __restrict__ p, int64_t cnt, unsigned* __restrict__ out) {
  unsigned m = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
    m = max(m, __float_as_uint(fabsf((float)p[e])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// zero the Z tiles from block kb0 on (the padding after the last slot)
template <typename T>
__global__ void tc_zero_kernel(typename TcT<T>::Bits* __restrict__ p, int64_t cnt) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
    p[e] = 0;
}

// The accumulator of columns [j0, j0 + 8) of one tile row (this thread's
// lane): the sum of the chains' partial products (tcgen05.ld, warp-wide).
template <typename T, int NC>
__device__ __forceinline__ void acc_load8(uint32_t ta, float (&d)[8]) {
  using C = TcCfg<T, NC>;
  float a[8], b[8];
  tc::tmem_ld8(ta, a);                         // chain 0, first half: hi x X_hi (FP32) / x X_1 (BF16)
  tc::tmem_ld8(ta + NC, b);                    // chain 0, second half: hi x X_lo / x X_2
#pragma unroll
  for (int i = 0; i < 8; ++i) d[i] = a[i] + b[i];
  if constexpr (C::NCH == 2) {
    tc::tmem_ld8(ta + 2 * NC, a);              // chain 1: lo x X_hi (FP32) / odd K steps x X_1 (BF16)
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i] += a[i];
    if constexpr (!TcT<T>::SPLIT) {
      tc::tmem_ld8(ta + 3 * NC, b);            // odd K steps x X_2
#pragma unroll
      for (int i = 0; i < 8; ++i) d[i] += b[i];
    }
  }
}

// ---------------------------------------------------------------------------
// converters: raw shared-memory rows -> TMEM A rows (this thread's lane)
// ---------------------------------------------------------------------------
// Each converter warp writes 32 TMEM columns of the stage's A buffer, half h
// (FP32: K values [32 h, 32 h + 32) as hi and lo; BF16: columns
// [32 h, 32 h + 32), i.e. K values [64 h, 64 h + 64)).
// phase 1: `raw` is this row's KC values (a factor column's chunk), of which
// the first kl are valid (the rest is padding or stale and becomes zero)
__device__ __forceinline__ void conv1(const uint8_t* raw, int kl, uint32_t ta, int h, float*) {
  constexpr int KC = TcT<float>::KC;
#pragma unroll
  for (int c0 = 32 * h; c0 < 32 * h + 32; c0 += 16) {
    float x[16];
    uint32_t hi[16], lo[16];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const float4 x4 = *reinterpret_cast<const float4*>(raw + (c0 + 4 * v) * 4);
      x[4 * v + 0] = x4.x;
      x[4 * v + 1] = x4.y;
      x[4 * v + 2] = x4.z;
      x[4 * v + 3] = x4.w;
    }
    if (c0 + 16 > kl) {
#pragma unroll
      for (int e = 0; e < 16; ++e) x[e] = c0 + e < kl ? x[e] : 0.f;
    }
    tc::split_fast<11>(x, hi, lo);        // factor magnitudes were checked when the plan was built
    tc::tmem_st16(ta + c0, hi);
    tc::tmem_st16(ta + KC + c0, lo);
  }
}
__device__ __forceinline__ void conv1(const uint8_t* raw, int kl, uint32_t ta, int h, __nv_bfloat16*) {
#pragma unroll
  for (int c0 = 32 * h; c0 < 32 * h + 32; c0 += 16) {          // 16 columns = 32 values
    uint32_t wv[16];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const uint4 u = *reinterpret_cast<const uint4*>(raw + 4 * (c0 + 4 * v));
      const uint32_t us[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = 2 * (c0 + 4 * v + e);           // values k (low half) and k + 1 (high half)
        uint32_t x = us[e];
        if (k >= kl) x = 0u;
        else if (k + 1 >= kl) x &= 0xFFFFu;
        wv[4 * v + e] = x;
      }
    }
    tc::tmem_st16(ta + c0, wv);
  }
}

// phase 2: slot k's tile row m sits at element meta[k].z + m of the raw
// area when m - meta[k].x < meta[k].y (the covered rows), else is 0
__device__ __forceinline__ float slot_val(const uint8_t* rb, const int4* meta, int k, int m, float*) {
  const int4 md = meta[k];
  const float v = reinterpret_cast<const float*>(rb)[md.z + m];
  return (uint32_t)(m - md.x) < (uint32_t)md.y ? v : 0.f;
}
__device__ __forceinline__ uint32_t slot_val(const uint8_t* rb, const int4* meta, int k, int m, __nv_bfloat16*) {
  const int4 md = meta[k];
  const uint32_t v = reinterpret_cast<const uint16_t*>(rb)[md.z + m];
  return (uint32_t)(m - md.x) < (uint32_t)md.y ? v : 0u;
}
__device__ __forceinline__ void conv2(const uint8_t* rb, const int4* meta, int m, uint32_t ta, int h, float* tag) {
  constexpr int KC = TcT<float>::KC;
#pragma unroll 1
  for (int c0 = 32 * h; c0 < 32 * h + 32; c0 += 16) {
    float x[16];
    uint32_t hi[16], lo[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = slot_val(rb, meta, c0 + j, m, tag);
    tc::split_fast<11>(x, hi, lo);        // factor magnitudes were checked when the plan was built
    tc::tmem_st16(ta + c0, hi);
    tc::tmem_st16(ta + KC + c0, lo);
  }
}
__device__ __forceinline__ void conv2(const uint8_t* rb, const int4* meta, int m, uint32_t ta, int h,
                                      __nv_bfloat16* tag) {
#pragma unroll 1
  for (int c0 = 32 * h; c0 < 32 * h + 32; c0 += 16) {
    uint32_t wv[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int k = 2 * (c0 + j);
      wv[j] = slot_val(rb, meta, k, m, tag) | (slot_val(rb, meta, k + 1, m, tag) << 16);
    }
    tc::tmem_st16(ta + c0, wv);
  }
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
  using C = TcCfg<T, NC>;
  constexpr int KE = Tr::KE, KC = Tr::KC;
  extern __shared__ __align__(1024) uint8_t smem[];
  TcBars* bars = reinterpret_cast<TcBars*>(smem + C::BAR_OFF);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t tmem = tc_setup(bars, warp, C::S, TC_NPROD);    // the producers' cp.async arrivals
  const uint32_t sbase = tc::smem_u32(smem);
  auto nk_of = [&](int64_t w) { return (int)((a.items[w].len + KC - 1) / KC); };

  if (warp >= 8 && warp < TC_MMA_WARP) {
    // ---------------- producers: the X tile (one bulk copy) and 256 bytes of each column ----------------
    // thread pt copies 16-byte piece q of the columns cg, cg + CG, .., (CG = 2 TC_PW column groups)
    // (the tile's column offsets are loaded into registers once per tile:
    // re-reading them every stage put a load latency in front of each stage's
    // copies; the first stage's wait is covered by the stages already queued)
    constexpr int CG = TC_NPROD / 16, CPT = 128 / CG;      // column groups, columns per thread
    const int pt = threadIdx.x - TC_PROD0;
    const int q = pt & 15, cg = pt >> 4;
    uint32_t it = 0;
    int64_t w = blockIdx.x;
    TcItem1 I = w < a.nitems ? a.items[w] : TcItem1{};
    bool stop = false;
    while (w < a.nitems && !stop) {
      const int64_t w2 = w + gridDim.x;
      const TcItem1 I2 = w2 < a.nitems ? a.items[w2] : TcItem1{};
      const int qs = (KE - (int)(I.seg0 % KE)) % KE;
      const int64_t kb0 = ((int64_t)I.seg0 + qs) / KE;
      const int64_t plen = pad_to((int64_t)I.len, KE);       // stored column length
      const int nk = (int)((I.len + KC - 1) / KC);
      uint64_t coff[CPT];
#pragma unroll
      for (int j = 0; j < CPT; ++j) {
        const uint32_t c = (uint32_t)(cg + CG * j);
        coff[j] = c < I.ncol ? __ldg(&a.cols[I.col0 + c].off) : 0;
      }
      for (int kc = 0; kc < nk; ++kc) {
        const int s = (int)(it % C::S);
        if (!tc_wait(bars, &bars->empty[s], ((it / C::S) & 1u) ^ 1u, a.err, 1)) { stop = true; break; }
        const uint32_t st = sbase + (uint32_t)(s * C::STAGE);
        const int64_t e0 = (int64_t)kc * KC;
        if (pt == 0) {
          tc::mbar_arrive_expect_tx(&bars->bfull[s], (uint32_t)C::B_BYTES);
          tc::bulk_g2s(st, a.xt + (int64_t)qs * a.xt_copy + (kb0 + e0 / KE) * (2 * NC * KE), C::B_BYTES,
                       &bars->bfull[s]);
        }
        const int64_t el = e0 + q * KE;                       // first element of this thread's piece
        const bool in = el < plen;
        const uint32_t dst = st + C::B_BYTES + q * 16;
#pragma unroll
        for (int j = 0; j < CPT; ++j) {
          const uint32_t c = (uint32_t)(cg + CG * j);
          const bool ok = in && c < I.ncol;
          tc::cp_async16(dst + c * C::RS1, ok ? (const void*)(a.pool + coff[j] + el) : (const void*)a.pool,
                         ok ? 16u : 0u);
        }
        tc::cp_async_mbar_arrive(&bars->full[s]);
        ++it;
        if (kc == 0 && q == 0) {
          // the next tile's column entries into L2 while this one streams
#pragma unroll
          for (int j = 0; j < CPT; ++j) {
            const uint32_t c = (uint32_t)(cg + CG * j);
            if (c < I2.ncol) asm volatile("prefetch.global.L2 [%0];" ::"l"(&a.cols[I2.col0 + c]));
          }
        }
      }
      w = w2;
      I = I2;
    }
    tc::cp_async_wait_all();
    if (pt == 0) tc_copies_drain(bars, it, C::S, a.err);
  } else if (warp == TC_MMA_WARP) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) tc_mma_role<T, NC>(bars, sbase, tmem, a.nitems, nk_of, 1 << 30, a.err);   // one segment a tile
  } else if (warp < 8) {
    // ---------------- converters (thread = TMEM lane m = tile row = factor column m) + drain ----------------
    const int m = 32 * (warp & 3) + lane, h = warp >> 2;
    const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
    // drain of tile jj: Z slots of row m, accumulator columns [h NC / 2, h NC / 2 + NC / 2)
    auto drain = [&](const TcItem1& J, uint32_t jj) -> bool {
      const uint32_t q = jj & 1u;
      const bool valid = (uint32_t)m < J.ncol;
      TcCol1 Cc{};
      if (valid) Cc = a.cols[J.col0 + m];
      if (!tc_wait_warp(bars, &bars->accfull[q], (jj >> 1) & 1u, a.err, 8)) return false;
      tc::tc_fence_after();
#pragma unroll 1
      for (int j0 = h * (NC / 2); j0 < (h + 1) * (NC / 2); j0 += 8) {
        float zz[8];
        acc_load8<T, NC>(tmem + lb + (uint32_t)(C::ACC0 + q * C::ACCW + j0), zz);
        if (valid) {
          uint32_t zh[8], zl[8];
          tc::split_n<Tr::SIG>(zz, zh, zl);
          for (uint32_t zi = Cc.zp0; zi < Cc.zp1; ++zi) {
            const uint32_t zp = a.zpl[zi];
            typename Tr::Bits* zb = a.zt + (int64_t)(zp / KE) * (2 * NC * KE) + (zp % KE);
#pragma unroll
            for (int jj2 = 0; jj2 < 8; ++jj2) {
              zb[(j0 + jj2) * KE] = (typename Tr::Bits)(zh[jj2] >> Tr::SHIFT);
              zb[NC * KE + (j0 + jj2) * KE] = (typename Tr::Bits)(zl[jj2] >> Tr::SHIFT);
            }
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&bars->accempty[q]);
      return true;
    };
    uint32_t it = 0, j = 0;
    bool stop = false, pend = false;
    TcItem1 Ip{};
    TcItem1 I = blockIdx.x < a.nitems ? a.items[blockIdx.x] : TcItem1{};
    for (int64_t w = blockIdx.x; w < a.nitems && !stop; w += gridDim.x, ++j) {
      const TcItem1 I2 = w + gridDim.x < a.nitems ? a.items[w + gridDim.x] : TcItem1{};
      const int nk = (int)((I.len + KC - 1) / KC);
      const bool row = (uint32_t)m < I.ncol;
      // the previous tile is drained after stage kd of this one: converting
      // stage NA - 1 needed the A buffer of the previous tile's last stage
      // back, so by then its MMAs (and its accumulator) are complete
      const int kd = min(C::NA - 1, nk - 1);
      for (int kc = 0; kc < nk; ++kc, ++it) {
        const int s = (int)(it % C::S), ab = (int)(it % C::NA);
        if (!tc_wait_warp(bars, &bars->full[s], (it / C::S) & 1u, a.err, 64)) { stop = true; break; }
        if (!tc_wait_warp(bars, &bars->aempty[ab], ((it / C::NA) & 1u) ^ 1u, a.err, 64)) { stop = true; break; }
        tc::tc_fence_after();
        const uint8_t* raw = smem + s * C::STAGE + C::B_BYTES + m * C::RS1;
        const int kl = row ? (int)min((int64_t)KC, (int64_t)I.len - (int64_t)kc * KC) : 0;
        conv1(raw, kl, tmem + lb + (uint32_t)(ab * Tr::ACOLS), h, (T*)nullptr);
        tc::tmem_wait_st();
        tc::tc_fence_before();
        tc::mbar_arrive(&bars->afull[ab]);
        if (pend && kc == kd) {
          pend = false;
          if (!drain(Ip, j - 1)) { stop = true; break; }
        }
      }
      Ip = I;
      pend = !stop;
      I = I2;
    }
    if (pend) drain(Ip, j - 1);
  }
  tc_teardown(bars, warp, tmem);
}

// ---------------------------------------------------------------------------
// phase 2
// ---------------------------------------------------------------------------
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
  using C = TcCfg<T, NC>;
  constexpr int KE = Tr::KE, KC = Tr::KC, ES = C::ES;
  extern __shared__ __align__(1024) uint8_t smem[];
  TcBars* bars = reinterpret_cast<TcBars*>(smem + C::BAR_OFF);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t tmem = tc_setup(bars, warp, C::S, TC_NPROD + TC_PW);   // cp.async arrivals + slot-table arrivals
  const uint32_t sbase = tc::smem_u32(smem);
  auto nk_of = [&](int64_t w) {
    const TcItem2 I = a.items[w];
    return (int)((I.ze - (I.zb / KE) * KE + KC - 1) / KC);
  };

  if (warp >= 8 && warp < TC_MMA_WARP) {
    // ---------------- producers: the Z tile (one bulk copy) and each slot's rows of the tile ----------------
    // warp pw handles slots SPW pw .. SPW pw + SPW - 1 of a stage; lane i
    // (< SPW) holds slot SPW pw + i's descriptor, loaded one stage ahead; per
    // slot the warp copies the rows lane by lane (16 bytes a lane) and lane 0
    // writes the slot table entry
    constexpr int SPW = KC / TC_PW;
    static_assert(SPW <= 32, "one descriptor per lane");
    const int pw = warp - 8;
    uint32_t it = 0;
    auto load_desc = [&](const TcItem2& J, int kc) {
      const int64_t zp = (int64_t)(J.zb / KE) * KE + (int64_t)kc * KC + SPW * pw + (lane % SPW);
      return (lane < SPW && zp >= (int64_t)J.zb && zp < (int64_t)J.ze) ? a.z2[zp] : TcZ2{0, 0, 0};
    };
    int64_t w = blockIdx.x;
    TcItem2 I = w < a.nitems ? a.items[w] : TcItem2{};
    int nk = w < a.nitems ? nk_of(w) : 0;
    TcItem2 In = w + gridDim.x < a.nitems ? a.items[w + gridDim.x] : TcItem2{};
    TcZ2 cur = w < a.nitems ? load_desc(I, 0) : TcZ2{0, 0, 0};
    int kc = 0;
    while (w < a.nitems) {
      // the next stage's cursor and descriptors
      int64_t w2 = w;
      int kc2 = kc + 1, nk2 = nk;
      TcItem2 I2 = I;
      if (kc2 == nk) {
        w2 = w + gridDim.x;
        kc2 = 0;
        I2 = In;
        nk2 = w2 < a.nitems ? (int)((I2.ze - (I2.zb / KE) * KE + KC - 1) / KC) : 0;
      }
      const TcZ2 nxt = w2 < a.nitems ? load_desc(I2, kc2) : TcZ2{0, 0, 0};
      {
        // the descriptors of the stage after that into L2 (one 128-byte line
        // holds 8 of them)
        const int64_t zq = (int64_t)(I2.zb / KE) * KE + (int64_t)(kc2 + 1) * KC + SPW * pw + 8 * lane;
        if (w2 < a.nitems && 8 * lane < SPW && zq < (int64_t)I2.ze)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a.z2 + zq));
      }
      // this stage
      const int s = (int)(it % C::S);
      if (!tc_wait_warp(bars, &bars->empty[s], ((it / C::S) & 1u) ^ 1u, a.err, 1)) break;
      const uint32_t st = sbase + (uint32_t)(s * C::STAGE);
      int4* meta = reinterpret_cast<int4*>(smem + s * C::STAGE + C::B_BYTES + C::RAW2);
      const int64_t zc = (int64_t)(I.zb / KE) * KE + (int64_t)kc * KC;
      if (pw == 0 && lane == 0) {
        tc::mbar_arrive_expect_tx(&bars->bfull[s], (uint32_t)C::B_BYTES);
        tc::bulk_g2s(st, a.zt + (zc / KE) * (2 * NC * KE), C::B_BYTES, &bars->bfull[s]);
      }
      // lane i (< SPW): slot SPW pw + i's copy and table entry
      const int toff = (int)I.toff;
      int64_t src = 0;
      uint32_t dsto = 0, nb = 0;
      if (lane < SPW) {
        const int k = SPW * pw + lane;
        const int r0 = max(cur.rlo, toff), r1 = min(cur.rhi, toff + 128);
        int4 md = make_int4(0, 0, 0, 0);
        if (r0 < r1) {
          // element offset of window row i: g(i) = a_off + i - rlo; the raw row
          // holds g(toff) - sh .. in 16-byte units (sh = g(toff) mod KE)
          const int64_t gt = cur.a_off + (toff - cur.rlo);
          const int shl = (int)(gt & (KE - 1));                 // KE is a power of two
          const int64_t g0 = cur.a_off + (r0 - cur.rlo), g1 = cur.a_off + (r1 - cur.rlo);
          const int64_t slo = g0 & ~(int64_t)(KE - 1);
          const int64_t shi = (g1 + KE - 1) & ~(int64_t)(KE - 1);
          src = slo;
          dsto = (uint32_t)(C::B_BYTES + k * C::RS2 + (slo - (gt - shl)) * ES);
          nb = (uint32_t)((shi - slo) * ES);
          md = make_int4(r0 - toff, r1 - r0, k * (C::RS2 / ES) + shl, 0);
        }
        meta[k] = md;
      }
      // the copies, slot by slot, 16 bytes a lane (whole 128-byte lines per instruction)
#pragma unroll 4
      for (int i = 0; i < SPW; ++i) {
        const uint32_t nbi = __shfl_sync(0xffffffffu, nb, i);
        const int64_t srci = (int64_t)__shfl_sync(0xffffffffu, (long long)src, i);
        const uint32_t dsti = __shfl_sync(0xffffffffu, dsto, i);
        if ((uint32_t)lane * 16u < nbi) tc::cp_async16(st + dsti + lane * 16, a.pool + srci + lane * KE, 16u);
        if (lane == 0 && nbi > 512u) tc::cp_async16(st + dsti + 512, a.pool + srci + 32 * KE, 16u);
      }
      __threadfence_block();                                  // the table entries before lane 0's release
      __syncwarp();
      tc::cp_async_mbar_arrive(&bars->full[s]);
      if (lane == 0) tc::mbar_arrive(&bars->full[s]);        // the slot table (release)
      ++it;
      if (w2 != w) In = w2 + gridDim.x < a.nitems ? a.items[w2 + gridDim.x] : TcItem2{};
      w = w2;
      kc = kc2;
      nk = nk2;
      I = I2;
      cur = nxt;
    }
    tc::cp_async_wait_all();
    if (pw == 0 && lane == 0) tc_copies_drain(bars, it, C::S, a.err);
  } else if (warp == TC_MMA_WARP) {
    if (lane == 0) tc_mma_role<T, NC>(bars, sbase, tmem, a.nitems, nk_of, tc_kseg2<NC>(), a.err);
  } else if (warp < 8) {
    // ---------------- converters (thread = TMEM lane m = tile row m) + drain ----------------
    const int m = 32 * (warp & 3) + lane, h = warp >> 2;
    const uint32_t lb = (uint32_t)(32 * (warp & 3)) << 16;
    // drain of tile jj: Y rows of the tile += accumulator columns of half h
    auto drain = [&](const TcItem2& J, uint32_t jj) -> bool {
      const uint32_t q = jj & 1u;
      if (!tc_wait_warp(bars, &bars->accfull[q], (jj >> 1) & 1u, a.err, 8)) return false;
      tc::tc_fence_after();
      const bool valid = (uint32_t)m < J.nrows;
      double* yr = a.Y + (int64_t)J.row0 + m;
#pragma unroll 1
      for (int j0 = h * (NC / 2); j0 < (h + 1) * (NC / 2); j0 += 8) {
        float dd[8];
        acc_load8<T, NC>(tmem + lb + (uint32_t)(C::ACC0 + q * C::ACCW + j0), dd);
        if (valid) {
#pragma unroll
          for (int jj2 = 0; jj2 < 8; ++jj2) {
            const int col = a.cb * NC + j0 + jj2;
            if (col < a.ncols) yr[(int64_t)col * a.ldy] += (double)dd[jj2];
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&bars->accempty[q]);
      return true;
    };
    uint32_t it = 0, j = 0;                              // stages, accumulation segments
    bool stop = false, pend = false;
    TcItem2 Ip{};
    TcItem2 I = blockIdx.x < a.nitems ? a.items[blockIdx.x] : TcItem2{};
    for (int64_t w = blockIdx.x; w < a.nitems && !stop; w += gridDim.x) {
      const TcItem2 I2 = w + gridDim.x < a.nitems ? a.items[w + gridDim.x] : TcItem2{};
      const int nk = (int)((I.ze - (I.zb / KE) * KE + KC - 1) / KC);
      for (int k0 = 0; k0 < nk && !stop; k0 += tc_kseg2<NC>(), ++j) {
        const int k1 = min(nk, k0 + tc_kseg2<NC>());
        const int kd = k0 + min(C::NA - 1, k1 - k0 - 1);  // as in phase 1, per segment
        for (int kc = k0; kc < k1; ++kc, ++it) {
          const int s = (int)(it % C::S), ab = (int)(it % C::NA);
          if (!tc_wait_warp(bars, &bars->full[s], (it / C::S) & 1u, a.err, 64)) { stop = true; break; }
          if (!tc_wait_warp(bars, &bars->aempty[ab], ((it / C::NA) & 1u) ^ 1u, a.err, 64)) { stop = true; break; }
          tc::tc_fence_after();
          const uint8_t* rb = smem + s * C::STAGE + C::B_BYTES;
          conv2(rb, reinterpret_cast<const int4*>(rb + C::RAW2), m, tmem + lb + (uint32_t)(ab * Tr::ACOLS), h,
                (T*)nullptr);
          tc::tmem_wait_st();
          tc::tc_fence_before();
          tc::mbar_arrive(&bars->afull[ab]);
          if (pend && kc == kd) {
            pend = false;
            if (!drain(Ip, j - 1)) { stop = true; break; }
          }
        }
        Ip = I;
        pend = !stop;
      }
      I = I2;
    }
    if (pend) drain(Ip, j - 1);
  }
  tc_teardown(bars, warp, tmem);
}

// ---------------------------------------------------------------------------
// Self-test of the operand layouts and descriptors used above: one 128 x 2NC
// accumulator D = A B' over K = 2 MMAs, with B staged as the X / Z tiles and
// A either as a K-major shared-memory tile (a_src 0) or in tensor memory as
// the converters write it (a_src 2).  The tiles sit at the start of a 200 KB
// shared allocation (A at 0, B at 96 KB), far inside it, so every address
// the descriptors can produce stays in the allocation.
// ---------------------------------------------------------------------------
constexpr int SELF_SMEM = 200 * 1024;
constexpr int SELF_B_OFF = 96 * 1024;
constexpr int SELF_KB = 4;             // 16-byte K blocks of the test (two MMAs)

template <typename T, int NC, bool A_TMEM>
__global__ void __launch_bounds__(128, 1) tc_selftest_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                           float* __restrict__ D, int* __restrict__ err) {
  using Tr = TcT<T>;
  constexpr int KE = Tr::KE;
  constexpr int KC = SELF_KB * KE;
  constexpr int DCOL = 128;            // accumulator columns [128, 128 + 2NC)
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  typename Tr::Bits* sa = reinterpret_cast<typename Tr::Bits*>(smem);
  typename Tr::Bits* sb = reinterpret_cast<typename Tr::Bits*>(smem + SELF_B_OFF);
  if (!A_TMEM) {
    // A (128 x KC, row-major input): row i, K block b at (i / 8) KB 128 + b 128 + (i % 8) 16 bytes
    for (int e = tid; e < 128 * KC; e += 128) {
      const int i = e / KC, k = e % KC;
      const int off = ((i / 8) * SELF_KB * 128 + (k / KE) * 128 + (i % 8) * 16) / (int)sizeof(T) + k % KE;
      sa[off] = Tr::bits(A[e]);
    }
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
  if (warp == 0) tc::tmem_alloc(&tslot, 256);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t lb = (uint32_t)(32 * warp) << 16;
  if (A_TMEM) {
    // row tid of A into TMEM lane tid, columns [0, KC) (TF32) or [0, KC / 2) (BF16 pairs)
    uint32_t r[16];
    if (Tr::SPLIT) {
#pragma unroll
      for (int c = 0; c < 16; ++c) r[c] = __float_as_uint(A[tid * KC + c]);
    } else {
#pragma unroll
      for (int c = 0; c < 16; ++c)
        r[c] = (uint32_t)Tr::bits(A[tid * KC + 2 * c]) | ((uint32_t)Tr::bits(A[tid * KC + 2 * c + 1]) << 16);
    }
    tc::tmem_st16(tmem + lb, r);
    tc::tmem_wait_st();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (tid == 0) {
    const uint32_t abase = tc::smem_u32(smem), bbase = tc::smem_u32(smem + SELF_B_OFF);
    constexpr uint32_t LBO_B = 2 * NC * 16, SBO_B = 128;
    const uint32_t id = tc::idesc(Tr::FMT, 2 * NC, 0, 0);
#pragma unroll
    for (int ks = 0; ks < SELF_KB / 2; ++ks) {
      const uint64_t bd = tc::smem_desc(bbase + ks * 2 * LBO_B, LBO_B, SBO_B);
      if (A_TMEM) {
        tc::mma_ts<Tr::KIND>(tmem + DCOL, tmem + ks * 8, bd, id, ks > 0 ? 1u : 0u);
      } else {
        const uint64_t ad = tc::smem_desc(abase + ks * 2 * 128, 128, SELF_KB * 128);
        tc::mma<Tr::KIND>(tmem + DCOL, ad, bd, id, ks > 0 ? 1u : 0u);
      }
    }
    tc::mma_commit(&bar);
  }
  __syncwarp();
  if (!tc::mbar_wait(&bar, 0u, TC_WAIT) && lane == 0) atomicOr(err, 1);
  tc::tc_fence_after();
  for (int j0 = 0; j0 < 2 * NC; j0 += 16) {
    float d[16];
    tc::tmem_ld16(tmem + lb + (uint32_t)(DCOL + j0), d);
#pragma unroll
    for (int j = 0; j < 16; ++j) D[(32 * warp + lane) * 2 * NC + j0 + j] = d[j];
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, 256);
  }
}

template <typename T, int NC, bool A_TMEM>
int run_selftest(const float* A, const float* B, float* D) {
  constexpr int KC = SELF_KB * TcT<T>::KE;
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
  HM_CUDA_TRY(smem_attr((const void*)tc_selftest_kernel<T, NC, A_TMEM>, SELF_SMEM));
  tc_selftest_kernel<T, NC, A_TMEM><<<1, 128, SELF_SMEM>>>(dA, dB, dD, dE);
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaDeviceSynchronize());
  int e = 0;
  HM_CUDA_TRY(cudaMemcpy(&e, dE, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) return fail(HM_ERR_TIMEOUT, "tensor-core self-test: the MMA did not complete");
  HM_CUDA_TRY(cudaMemcpy(D, dD, sizeof(float) * 128 * 2 * NC, cudaMemcpyDeviceToHost));
  return HM_OK;
}

}  // namespace

int tc_selftest(int kind, int a_src, int nc, const float* A, const float* B, float* D) {
  if (a_src != 0 && a_src != 2) return fail(HM_ERR_ARG, "self-test: a_src 0 (shared memory) or 2 (tensor memory)");
  const bool tm = a_src == 2;
  if (kind == 0) {
    if (nc == 16) return tm ? run_selftest<float, 16, true>(A, B, D) : run_selftest<float, 16, false>(A, B, D);
    if (nc == 64) return tm ? run_selftest<float, 64, true>(A, B, D) : run_selftest<float, 64, false>(A, B, D);
  } else if (kind == 1) {
    if (nc == 16)
      return tm ? run_selftest<__nv_bfloat16, 16, true>(A, B, D) : run_selftest<__nv_bfloat16, 16, false>(A, B, D);
    if (nc == 64)
      return tm ? run_selftest<__nv_bfloat16, 64, true>(A, B, D) : run_selftest<__nv_bfloat16, 64, false>(A, B, D);
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
  HM_CUDA_TRY(h2d_sync(*d, v.data(), sizeof(V) * v.size()));
  return HM_OK;
}

static int build_tc_plan(hm_handle* h, int trans, TcPlan** out) {
  const int eb = elem_bytes(h->storage);
  struct Lf { int64_t li; int64_t zoff; };
  // low-rank leaves in pool order with their z offsets
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
  // ---- phase 2: windows of TC_WR output rows; Z slots window by window,
  // items = the 128-row tiles of a window that some slot covers
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
    const uint32_t zb = (uint32_t)z2.size();
    const int64_t wrows = std::min<int64_t>(TC_WR, n - w * TC_WR);
    bool tile_used[TC_WR / 128] = {false, false, false, false};
    for (int32_t i : per[w]) {
      const Leaf& L = h->leaves[rk[i].li];
      const int64_t npad = col_pad(L.n, eb), mpad = col_pad(L.m, eb);
      const int64_t o0 = trans ? L.col0 : L.row0, o1 = o0 + (trans ? L.n : L.m);
      const int64_t lo = std::max<int64_t>(o0, w * TC_WR), hi = std::min<int64_t>(o1, (w + 1) * TC_WR);
      for (int64_t t = (lo - w * TC_WR) / 128; t * 128 < hi - w * TC_WR; ++t) tile_used[t] = true;
      for (int r = 0; r < L.k; ++r) {
        // F2: A (m x k, stride mpad) for H*x, B (n x k, stride npad) for H'*x
        const int64_t col = trans ? L.off + (int64_t)r * npad : L.off + npad * L.k + (int64_t)r * mpad;
        TcZ2 Z{};
        Z.a_off = col + (lo - o0);
        Z.rlo = (int32_t)(lo - w * TC_WR);
        Z.rhi = (int32_t)(hi - w * TC_WR);
        zpl[fillpos[rk[i].zoff + r]++] = (uint32_t)z2.size();
        z2.push_back(Z);
      }
    }
    const uint32_t ze = (uint32_t)z2.size();
    for (int t = 0; t < TC_WR / 128 && t * 128 < wrows; ++t) {
      if (!tile_used[t]) continue;
      TcItem2 I{};
      I.row0 = (uint32_t)(w * TC_WR + t * 128);
      I.nrows = (uint32_t)std::min<int64_t>(128, wrows - t * 128);
      I.zb = zb;
      I.ze = ze;
      I.toff = (uint32_t)(t * 128);
      it2.push_back(I);
    }
    std::vector<int32_t>().swap(per[w]);
  }
  if (z2.size() > (size_t)UINT32_MAX / 2) { delete P; return fail(HM_ERR_UNSUPPORTED, "too many low-rank terms for the tensor-core plan"); }
  // ---- phase 1: factor columns of F1 grouped by input segment, 128 per tile
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
        TcCol1 Cc{};
        Cc.off = trans ? (uint64_t)(L.off + npad * L.k + (int64_t)r * mpad) : (uint64_t)(L.off + (int64_t)r * npad);
        Cc.zp0 = zp_count[rk[ord1[j]].zoff + r];
        Cc.zp1 = zp_count[rk[ord1[j]].zoff + r + 1];
        col1.push_back(Cc);
      }
      ++j;
    }
    const uint32_t c1 = (uint32_t)col1.size();
    for (uint32_t c = c0; c < c1; c += 128) {
      TcItem1 I{};
      I.col0 = c;
      I.ncol = std::min<uint32_t>(128, c1 - c);
      I.seg0 = (uint32_t)sg.first;
      I.len = (uint32_t)sg.second;
      if (I.len > 0) it1.push_back(I);
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

// The factor magnitudes the converters' split relies on, measured once per
// state of the factor pool.
static int check_pool(hm_handle* h, TcPlan* P) {
  const int eb = elem_bytes(h->storage);
  {
    const int64_t cnt = (int64_t)(h->rk_bytes / (size_t)eb);
    unsigned* d_m = nullptr;
    unsigned mbits = 0;
    cudaError_t e = cudaMalloc(&d_m, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(d_m, 0, sizeof(unsigned));
    if (e == cudaSuccess && cnt > 0) {
      const unsigned g = (unsigned)std::min<int64_t>((cnt + 255) / 256, 148 * 16);
      if (h->storage == HM_F32) pool_maxabs_kernel<float><<<g, 256>>>((const float*)h->d_rk, cnt, d_m);
      else pool_maxabs_kernel<__nv_bfloat16><<<g, 256>>>((const __nv_bfloat16*)h->d_rk, cnt, d_m);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&mbits, d_m, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (d_m) cudaFree(d_m);
    if (e != cudaSuccess) return fail(HM_ERR_CUDA, std::string("tensor-core plan: ") + cudaGetErrorString(e));
    P->usable = mbits <= 0x71800000u;           // 2^100
    P->checked = true;
  }
  return HM_OK;
}

// the factor pool changed (hm_scale): the magnitude check runs again
void tc_factors_changed(hm_handle* h) {
  if (h->tc_fwd) h->tc_fwd->checked = false;
  if (h->tc_bwd) h->tc_bwd->checked = false;
}

// ---------------------------------------------------------------------------
// launch
// ---------------------------------------------------------------------------
template <typename T, int NC>
static int launch_tc(hm_handle* h, TcPlan& P, const double* d_x, double* d_y, int64_t ncols, cudaStream_t st) {
  using Bits = typename TcT<T>::Bits;
  using C = TcCfg<T, NC>;
  constexpr int KE = TcT<T>::KE, KC = TcT<T>::KC;
  const int64_t n = h->n;
  const int64_t nkb = (n + KE + KC) / KE + 2;                   // XT blocks per shifted copy
  const int64_t xt_copy = nkb * 2 * NC * KE;
  const int64_t zkb = (P.nz2 + KC) / KE + 2;                    // Z blocks (with zero padding)
  const size_t xt_bytes = sizeof(Bits) * (size_t)(KE * xt_copy);
  const size_t zt_bytes = sizeof(Bits) * (size_t)(zkb * 2 * NC * KE);
  const size_t need = (xt_bytes + 255) / 256 * 256 + zt_bytes;
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
  Bits* zt = (Bits*)((char*)h->d_tc + (xt_bytes + 255) / 256 * 256);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  HM_CUDA_TRY(smem_attr((const void*)tc_phase1_kernel<T, NC>, C::BYTES));
  HM_CUDA_TRY(smem_attr((const void*)tc_phase2_kernel<T, NC>, C::BYTES));
  // Z padding past the last slot stays zero (its A rows are zero too, and
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
      tc_phase1_kernel<T, NC><<<(unsigned)std::min<int64_t>(nsm, P.nitem1), TC_THREADS, C::BYTES, st>>>(a1);
    }
    if (P.nitem2 > 0) {
      P2Args<T, NC> a2{P.d_item2, P.nitem2, P.d_z2, (const T*)h->d_rk, zt, d_y, n, (int)ncols, cb, h->d_tc_err};
      tc_phase2_kernel<T, NC><<<(unsigned)std::min<int64_t>(nsm, P.nitem2), TC_THREADS, C::BYTES, st>>>(a2);
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

// Builds the plan of a direction on first use and reports whether the
// tensor-core path applies (FP32/BF16 factors, all of them at most 2^100 in
// magnitude); otherwise the caller takes the CUDA-core block kernels.
int tc_prepare(hm_handle* h, int trans, bool* usable) {
  *usable = false;
  if (h->storage != HM_F32 && h->storage != HM_BF16) return HM_OK;
  TcPlan*& P = trans ? h->tc_bwd : h->tc_fwd;
  if (!P) HM_TRY(build_tc_plan(h, trans, &P));
  if (!P->checked) HM_TRY(check_pool(h, P));
  *usable = P->usable;
  return HM_OK;
}

// Y += the low-rank part of H X (H' X) on the tensor cores; the caller has
// written the dense part into Y.
int matvec_multi_tc(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st) {
  if (h->storage != HM_F32 && h->storage != HM_BF16)
    return fail(HM_ERR_UNSUPPORTED, "tensor-core matvec: FP32 or BF16 factors only");
  TcPlan*& P = trans ? h->tc_bwd : h->tc_fwd;
  if (!P) HM_TRY(build_tc_plan(h, trans, &P));
  if (!P->checked) HM_TRY(check_pool(h, P));
  if (!P->usable) return fail(HM_ERR_UNSUPPORTED, "tensor-core matvec: a factor entry exceeds 2^100 or is NaN");
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
