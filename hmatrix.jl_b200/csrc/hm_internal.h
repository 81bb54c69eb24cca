// Internal declarations shared by the translation units of libhmatb200.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/hmatrix_b200.h"

namespace hm {

// ---------------------------------------------------------------------------
// error handling: every entry point returns a status; the message is kept per
// thread and read back with hm_last_error().
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
// Raises a kernel's dynamic shared-memory limit to `bytes` once per (kernel,
// current device); safe to call from several host threads.
cudaError_t smem_attr(const void* kernel, int bytes);

#define HM_CUDA_TRY(expr)                                                      \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess)                                                     \
      return ::hm::fail(HM_ERR_CUDA, std::string(#expr) + ": " +               \
                                         cudaGetErrorString(_e));              \
  } while (0)

// Host -> device copy of pageable memory that has landed when it returns.  A
// pageable cudaMemcpy may return with its DMA still in flight on the legacy
// stream, which the handle's non-blocking streams do not wait for; plans and
// tables uploaded this way are read by kernels on those streams right after.
inline cudaError_t h2d_sync(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  return e != cudaSuccess ? e : cudaStreamSynchronize(cudaStreamLegacy);
}

#define HM_TRY(expr)                                                           \
  do {                                                                         \
    int _s = (expr);                                                           \
    if (_s != HM_OK) return _s;                                                \
  } while (0)

// ---------------------------------------------------------------------------
// kernel description on the device (Hparams.Kernel restricted to an enum)
// ---------------------------------------------------------------------------
struct KernelDesc {
  int kind;        // HM_KERNEL_*
  int dim;         // 1..3
  double p;        // ell or c
  double shift;    // lambda on the global diagonal (only diagonal leaves)
};

// Geometry is column-major n x dim.  The arithmetic order matches the FP64
// oracle exactly (no FMA contraction), so rational kernels are bit-identical
// to the CPU restatement of kernel_full (src/cluster.jl:258-275).
// kernel_eval_xy: k(x, y) for points whose coordinate q is x[q * sx], y[q * sy].
__device__ __forceinline__ double kernel_eval_xy(const KernelDesc& kd, const double* __restrict__ x,
                                                 int64_t sx, const double* __restrict__ y, int64_t sy) {
  double s = 0.0;
  if ((kd.kind == HM_KERNEL_CAUCHY && kd.p != 1.0) || kd.kind == HM_KERNEL_CAUCHY_DP) {
#pragma unroll 3
    for (int q = 0; q < kd.dim; ++q) {
      double d = __ddiv_rn(__dsub_rn(x[q * sx], y[q * sy]), kd.p);
      double t = __dmul_rn(d, d);
      s = (q == 0) ? t : __dadd_rn(s, t);
    }
  } else {
#pragma unroll 3
    for (int q = 0; q < kd.dim; ++q) {
      double d = __dsub_rn(x[q * sx], y[q * sy]);
      double t = __dmul_rn(d, d);
      s = (q == 0) ? t : __dadd_rn(s, t);
    }
  }
  double v;
  if (kd.kind == HM_KERNEL_GAUSS) {
    v = exp(-__ddiv_rn(s, __dmul_rn(__dmul_rn(2.0, kd.p), kd.p)));
  } else if (kd.kind == HM_KERNEL_INVQUAD) {
    v = __ddiv_rn(1.0, __dadd_rn(kd.p, s));
  } else if (kd.kind == HM_KERNEL_CAUCHY_DP) {            // s = |x-y|^2 / p^2
    const double t = __dadd_rn(1.0, s);
    v = __ddiv_rn(__ddiv_rn(__dmul_rn(2.0, s), kd.p), __dmul_rn(t, t));
  } else if (kd.kind == HM_KERNEL_INVQUAD_DP) {
    const double t = __dadd_rn(kd.p, s);
    v = -__ddiv_rn(1.0, __dmul_rn(t, t));
  } else if (kd.kind == HM_KERNEL_GAUSS_DP) {
    const double p3 = __dmul_rn(__dmul_rn(kd.p, kd.p), kd.p);
    v = __dmul_rn(exp(-__ddiv_rn(s, __dmul_rn(__dmul_rn(2.0, kd.p), kd.p))), __ddiv_rn(s, p3));
  } else {
    v = __ddiv_rn(1.0, __dadd_rn(1.0, s));
  }
  return v;
}

__device__ __forceinline__ double kernel_eval(const KernelDesc& kd,
                                              const double* __restrict__ geom,
                                              int64_t n, int64_t i, int64_t j) {
  return kernel_eval_xy(kd, geom + i, n, geom + j, n);
}

// ---------------------------------------------------------------------------
// flattened structure
// ---------------------------------------------------------------------------
enum : int8_t { T_DENSE = 0, T_RK = 1, T_H = 2 };

struct Node {              // block tree node (H, dense or low-rank)
  int8_t type;
  int32_t s, t;            // row / column cluster index
  int32_t child[4];        // 11, 12, 21, 22 for T_H
  int32_t leaf;            // leaf index for T_DENSE / T_RK
};

struct Leaf {
  int8_t type;
  int32_t s, t;            // clusters
  int32_t node;
  int64_t row0, col0;
  int32_t m, n;
  int32_t k;               // rank (low-rank leaves)
  int64_t off;             // element offset in its pool (storage precision)
  int32_t group;           // row group
};

// Matvec plan.  Phase 1 runs one warp per low-rank leaf and computes
// z = F1' x_seg (F1 = B for H*x, A for H'*x) into a z array.  Phase 2 runs one
// CTA per window of MV_WROWS output rows and accumulates y = sum F2 z + dense.
struct __align__(16) P1Desc {          // 32 bytes
  uint64_t off;            // element offset of F1 in the low-rank pool
  uint32_t seg0;           // first input index
  uint32_t len;            // input extent (rows of F1)
  uint32_t stride;         // column stride of F1 (padded length)
  uint32_t zoff;           // offset of this leaf's k values in z
  uint16_t k;
  uint16_t pad0;
  uint32_t pad1;
};
static_assert(sizeof(P1Desc) == 32, "P1Desc must stay 32 bytes");

enum : uint16_t { P2_RK = 1, P2_DENSE = 0, P2_DENSE_T = 2 };
struct __align__(16) P2Desc {          // 32 bytes
  uint64_t off;            // element offset of F2 (low-rank pool) or C (dense pool)
  int32_t row_off;         // first output row relative to the window start
  uint32_t m;              // output extent
  uint32_t ld;             // column stride of F2 / C
  uint32_t aux;            // zoff (low-rank) or first input index (dense)
  uint32_t cnt;            // k (low-rank) or input extent (dense)
  uint16_t type;           // P2_*
  uint16_t pad0;
};
static_assert(sizeof(P2Desc) == 32, "P2Desc must stay 32 bytes");

struct MvWin {
  uint32_t row0, nrows;    // output rows of the window
  uint32_t begin, end;     // P2Desc range
};

constexpr int MV_WROWS = 1024;         // rows per phase-2 window (8 warps x 32 lanes x 4 rows)

struct MvPlan {
  P1Desc* d_p1 = nullptr;
  int64_t np1 = 0;
  P1Desc* d_p1s = nullptr;         // the same descriptors ordered by input segment (multi-RHS phase 1; built on first use)
  uint32_t* d_g1s = nullptr;       // groups of d_p1s sharing a segment (ng1 + 1 starts)
  int64_t ng1 = 0;
  uint32_t* d_t1s = nullptr;       // segment tasks of d_p1s (nt1 + 1 starts)
  int64_t nt1 = 0;
  uint32_t maxlen1 = 0;            // longest segment
  P2Desc* d_p2 = nullptr;
  int64_t np2 = 0;
  MvWin* d_win = nullptr;
  int32_t nwin = 0;
  P2Desc* d_p2d = nullptr;         // the dense descriptors alone, window by window (built on first use)
  MvWin* d_wind = nullptr;         // windows over d_p2d (nwin of them)
  P2Desc* d_p2r = nullptr;         // the low-rank descriptors alone, window by window (built with d_p2d)
  MvWin* d_winr = nullptr;         // windows over d_p2r
  // phase 2 by tree clusters (hm_autotune's phase-2 shape 1; built on first
  // use): a unit is a 128-row chunk of an output cluster that is some leaf's
  // cluster, with exactly the leaves of that cluster; one warp per unit
  bool cl_built = false;
  P2Desc* d_cd = nullptr;          // descriptors, unit by unit (offsets moved to the chunk's first row)
  MvWin* d_cu = nullptr;           // units: rows [row0, row0 + nrows), descriptors [begin, end)
  std::vector<int32_t> cl_level;   // units of tree level i: [cl_level[i], cl_level[i + 1])
};

struct LuState;            // H-LU data (hm_lu.cu)
struct TcPlan;             // tensor-core multi-RHS matvec plan (hm_matvec_tc.cu)

}  // namespace hm

struct hm_handle {
  hm_params prm;
  int64_t n = 0;
  int dim = 1;
  int device = 0;
  cudaStream_t stream = nullptr;
  hm::KernelDesc kd;

  // cluster tree (host)
  std::vector<int64_t> cl_s, cl_e, cl_left, cl_right;
  std::vector<int32_t> cl_depth;

  // block tree and leaves (host)
  std::vector<hm::Node> nodes;
  std::vector<hm::Leaf> leaves;
  int64_t depth = 0;

  // device data
  double* d_geom = nullptr;
  void* d_rk = nullptr;            // low-rank factors, storage precision
  size_t rk_bytes = 0;
  void* d_dense = nullptr;         // dense leaves (FP64 if storage F64 else FP32)
  size_t dense_bytes = 0;
  int storage = HM_F64;
  int kmax = 0;

  hm::MvPlan fwd, bwd;             // matvec plans (H*x, H'*x)
  double* d_z = nullptr;           // phase-1 results, sum of ranks
  int64_t zlen = 0;

  // per-call scratch
  void* d_xs = nullptr;            // aligned shifted copies of the input
  size_t xs_bytes = 0;
  int* d_counter = nullptr;        // work counters
  double* d_io = nullptr;          // staging for host pointers
  size_t io_bytes = 0;
  void* d_xm = nullptr;            // multi-RHS matvec: row-major input block + phase-1 results
  size_t xm_bytes = 0;
  hm::TcPlan* tc_fwd = nullptr;    // tensor-core multi-RHS plans (FP32/BF16 factors), built on first use
  hm::TcPlan* tc_bwd = nullptr;
  void* d_tc = nullptr;            // their X and Z tiles
  size_t tc_bytes = 0;
  int* d_tc_err = nullptr;         // error word of their bounded waits
  void* d_dd = nullptr;            // compensated residual: z as hi + lo
  size_t dd_bytes = 0;
  int32_t* d_piv = nullptr;        // aca2 pivots (row, column) of every step, when kept
  int64_t piv_count = 0;

  struct Tune {                    // launch shapes chosen by hm_autotune (hm_api.cu)
    int p2_split = 4;              // phase-2 CTAs per 1024-row window (2, 4, 8); 1: by tree clusters
    int p1_waves = 1;              // phase-1 grid in resident waves (1, 2, 4)
    int tc_nc[3] = {0, 0, 0};      // tensor-core column block for c <= 16, <= 32, > 32 (0: by c)
    int tuned = 0;
  } tune;
  hm::LuState* lu = nullptr;       // set once factorised
  bool factorized = false;
};

namespace hm {

// element sizes / vector widths of the storage formats
inline int elem_bytes(int storage) { return storage == HM_F64 ? 8 : (storage == HM_F32 ? 4 : 2); }
inline int dense_elem_bytes(int storage) { return storage == HM_F64 ? 8 : 4; }
__host__ __device__ inline int64_t pad_to(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
// padded column length: a multiple of 16 bytes and of 4 elements, so every
// column starts on a 16-byte boundary and 4-row groups never leave a column
__host__ __device__ inline int64_t col_pad_elems(int ebytes) { return 16 / ebytes > 4 ? 16 / ebytes : 4; }
__host__ __device__ inline int64_t col_pad(int64_t len, int ebytes) { return pad_to(len, col_pad_elems(ebytes)); }
__host__ __device__ inline int64_t col_pad_dev(int64_t len, int ebytes) { return pad_to(len, col_pad_elems(ebytes)); }

template <typename T> __device__ __forceinline__ T to_store(double v) { return (T)v; }
template <> __device__ __forceinline__ __nv_bfloat16 to_store<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
template <typename T> __device__ __forceinline__ double from_store(T v) { return (double)v; }
template <> __device__ __forceinline__ double from_store<__nv_bfloat16>(__nv_bfloat16 v) {
  return (double)__bfloat162float(v);
}

// build (hm_build.cu)
int build_handle(hm_handle* h, const double* geom, int64_t ncluster,
                 const int64_t* cl_s, const int64_t* cl_e, const int64_t* cl_left,
                 const int64_t* cl_right, int64_t n_nb, const int64_t* nb_pairs);
int build_matvec_plans(hm_handle* h);
int build_like(hm_handle* h, const hm_handle* ref);
int partition_only(hm_handle* h, int64_t ncl, const int64_t* cl_s, const int64_t* cl_e, const int64_t* cl_left,
                   const int64_t* cl_right, int64_t n_nb, const int64_t* nb_pairs);
int build_mv_descriptors(hm_handle* h, const std::vector<int64_t>& order, int trans);
void free_mv_plan(MvPlan& p);
int leaf_factors_f64(const hm_handle* h, int64_t leaf, double* A, double* B);
int to_dense(const hm_handle* h, double* d_out);   // device output n*n
int apply_shift(hm_handle* h, double lambda);
int apply_scale(hm_handle* h, double u);
int copy_handle(const hm_handle* h, hm_handle** out);
int restore_structure(hm_handle* h);
// leaf-format-changing arithmetic (hm_harith.cu)
int coarsen_handle(const hm_handle* h, hm_handle** out);
int add_handles(const hm_handle* a, const hm_handle* b, double scalar, hm_handle** out);
// file export / import (hm_io.cu)
int save_handle(const hm_handle* h, const char* path, const void* user, int64_t user_bytes);
int load_user(const char* path, void* user, int64_t cap, int64_t* user_bytes);
int load_handle(const char* path, int device, int (*validate)(const hm_params*), hm_handle** out);
void free_handle_data(hm_handle* h);
void lu_describe(const hm_handle* h, int64_t* tiles, int64_t* cap);

// matvec (hm_matvec.cu)
int matvec_device(hm_handle* h, const double* d_x, double* d_y, int trans, cudaStream_t st,
                  cudaEvent_t* ev = nullptr);
// Y = H X (trans 0) or H' X (trans 1) for an n x ncols column-major block,
// factors streamed once per column block (hm_matvec_multi.cu)
int matvec_multi_device(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st,
                        bool simt = false);
// the low-rank part of Y = H X on the tensor cores, added into Y (hm_matvec_tc.cu)
int matvec_multi_tc(hm_handle* h, const double* d_x, double* d_y, int64_t ncols, int trans, cudaStream_t st);
int tc_prepare(hm_handle* h, int trans, bool* usable);
// Splits a plan's window lists into dense-only and low-rank-only lists (once).
int split_p2(MvPlan& P);
void tc_factors_changed(hm_handle* h);
int tc_status(hm_handle* h, cudaStream_t st);
int tc_selftest(int kind, int a_src, int nc, const float* A, const float* B, float* D);
void free_tc_plan(TcPlan*& p);
// r = b - H x (trans: b - H' x) with compensated sums (hm_matvec.cu)
int residual_device(hm_handle* h, const double* d_x, const double* d_b, double* d_r, int trans, cudaStream_t st);
int exact_rows_device(hm_handle* h, const int64_t* d_rows, int64_t nrows,
                      const double* d_x, double* d_y, cudaStream_t st);

// low-rank kernels (hm_lowrank.cu)
int aca_fp_host(const double* A, double* U, double* V, int m, int n, double eps, int rank,
                int* out_rank);

// LU (hm_lu.cu)
int lu_factor(hm_handle* h);
int lu_solve_device(hm_handle* h, const double* d_b, double* d_x, int64_t ncols, int trans, cudaStream_t st);
int lu_solve_refined(hm_handle* h, const double* d_b, double* d_x, int64_t ncols, int trans, double tol,
                     int max_iter, cudaStream_t st, int* iters, double* relres);
int lu_perm(const hm_handle* h, int64_t* P);
int lu_to_dense(const hm_handle* h, double* d_out);
void lu_free(hm_handle* h);
int lu_copy(const hm_handle* src, hm_handle* dst);

}  // namespace hm
