/*
 * hmatrix_b200.h -- C ABI of the B200 (sm_100a) H-matrix hot path.
 *
 * Drop-in boundary for the hot path of Hmatrix.jl: construction with ACA/SVD
 * compression (NewHmat), H-matvec (H*y, H*V, transposed), H-LU (lu / lu!)
 * and the triangular H-solve (H\y).  Every entry point takes plain pointers
 * and sizes, returns an int status (HM_OK == 0) and never aborts; the text of
 * the last error of the calling thread is available from hm_last_error().
 *
 * Index space: exactly as in the reference, vectors live in the
 * cluster-permuted order c.X = Geom[c.P,:] (src/cluster.jl:248-249,
 * test/harithm.jl:9-11).  The caller builds the cluster tree (the reference
 * does it on the host with sklearn, src/cluster.jl:196-256) and passes the
 * permuted geometry plus the flattened tree; the library builds the block
 * partition of src/cluster.jl:48-133 and compresses on the GPU.
 *
 * Pointers are host pointers unless HM_FLAG_DEVICE_PTRS is given, in which
 * case they must be device pointers on the handle's device.
 */
#ifndef HMATRIX_B200_H
#define HMATRIX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HM_OK              0
#define HM_ERR_ARG         1   /* invalid argument or configuration          */
#define HM_ERR_CUDA        2   /* CUDA runtime error                         */
#define HM_ERR_OOM         3   /* device or host allocation failed           */
#define HM_ERR_STATE       4   /* frozen (factorised) / not factorised       */
#define HM_ERR_SINGULAR    5   /* exactly zero pivot in a diagonal leaf      */
#define HM_ERR_RANK        6   /* a rank exceeded the handle's rank capacity */
#define HM_ERR_NONFINITE   7   /* NaN/Inf met where a finite value is needed */
#define HM_ERR_UNSUPPORTED 8   /* valid request outside what is implemented  */
#define HM_ERR_TIMEOUT     9   /* a bounded device wait gave up              */
#define HM_ERR_IO         10   /* a file could not be opened, read or written */

/* ---- kernels (Hparams.Kernel has to be one of these on the device) ----- */
#define HM_KERNEL_CAUCHY   1   /* 1/(1 + |x-y|^2/p^2)      p = kparam (ell)   */
#define HM_KERNEL_INVQUAD  2   /* 1/(p + |x-y|^2)          p = kparam (c)     */
#define HM_KERNEL_GAUSS    3   /* exp(-|x-y|^2/(2 p^2))    p = kparam (ell)   */
/* Derivatives of the kernels above with respect to their parameter p, for the
 * hyper-parameter gradients u'(dH/dp)v (no counterpart in the reference): an
 * H-matrix built with one of these ids compresses dK/dp itself. */
#define HM_KERNEL_CAUCHY_DP   4   /* 2 s/p / (1 + s)^2, s = |x-y|^2/p^2         */
#define HM_KERNEL_INVQUAD_DP  5   /* -1/(p + |x-y|^2)^2                          */
#define HM_KERNEL_GAUSS_DP    6   /* exp(-|x-y|^2/(2 p^2)) |x-y|^2 / p^3         */

/* ---- construction methods (Hparams.ConsMethod) --------------------------- */
#define HM_CONS_ACA2       1   /* partially pivoted ACA, src/hlu.jl:59-111    */
#define HM_CONS_SVD        2   /* dense block + truncated SVD, cluster.jl:99  */
#define HM_CONS_BBFMM      3   /* Chebyshev interpolation, hlu.jl:20-29,113-132;
                                  deps/src/lowrank.cpp:186-222 (1-D and 2-D)   */

/* ---- storage precision of the matvec copy of the factors ----------------- */
#define HM_F64             0
#define HM_F32             1
#define HM_BF16            2   /* BF16 low-rank factors, FP32 dense leaves    */

/* ---- hm_params.build_flags ---------------------------------------------- */
#define HM_BUILD_KEEP_PIVOTS 1   /* aca2: keep every block's pivots for hm_new_like */

/* ---- flags ------------------------------------------------------------- */
#define HM_FLAG_DEVICE_PTRS 1u
#define HM_FLAG_TRANS       2u   /* hm_solve / hm_solve_refined: solve with H' */
#define HM_FLAG_MV_SIMT     4u   /* hm_matvec, several columns, FP32/BF16 factors:
                                    the CUDA-core block kernels instead of the
                                    tensor cores                                */

/* Mirror of the reference's global Params (src/utils.jl:8-24) restricted
 * to the fields the hot path reads, plus the device kernel description. */
typedef struct hm_params {
    int32_t dim;          /* 1..3 spatial dimension of Geom                  */
    int32_t kernel;       /* HM_KERNEL_*                                      */
    double  kparam;       /* kernel parameter (ell or c)                      */
    double  shift;        /* lambda of  H + lambda*I (diagonal of diag. leaves) */
    double  eps_comp;     /* Hparams.εComp  (ACA stop tolerance)              */
    double  eps_trunc;    /* Hparams.εTrunc (relative SVD truncation)         */
    int32_t max_rank;     /* Hparams.MaxRank                                  */
    int32_t max_block;    /* Hparams.MaxBlock (-1 -> n/4)                     */
    int32_t min_block;    /* Hparams.MinBlock                                 */
    int32_t cons_method;  /* HM_CONS_*                                        */
    int32_t aca_force;    /* Hparams.aca_force                                */
    int32_t storage;      /* HM_F64 / HM_F32 / HM_BF16                        */
    int32_t device;       /* CUDA device ordinal                              */
    int32_t rank_cap;     /* capacity of low-rank blocks during H-LU (0: auto) */
    int32_t lu_mode;      /* H-LU schedule: 0 auto, 1 the recursion of lu!,
                             2 tile by tile (needs a level where every block
                             outside the diagonal tiles is one low-rank block) */
    int32_t build_flags;  /* HM_BUILD_* */
    double  eps_trunc_lu; /* truncation tolerance of the recompressions inside
                             H-LU (0: eps_trunc, as in the reference); a looser
                             value gives a cheaper factorisation that
                             hm_solve_refined brings back to full accuracy */
    int32_t row_lo;       /* rows [row_lo, row_hi) of H only (0, 0: all rows):
                             a shard of a row-partitioned H for multi-GPU use.
                             The range must not cut a leaf (cut at clusters of
                             the first admissible level).  H*x of a shard gives
                             its rows and zeros elsewhere, H'*x its share of
                             the sum; hm_lu refuses a shard (HM_ERR_UNSUPPORTED) */
    int32_t row_hi;
} hm_params;

/* info(H) of src/utils.jl:83-110 plus the byte counts used for rooflines. */
typedef struct hm_info_t {
    int64_t n;
    int64_t n_dense;          /* number of dense leaves                        */
    int64_t n_rk;             /* number of low-rank leaves                     */
    int64_t depth;            /* depth of the block tree (root = 1)            */
    double  compress_ratio;   /* stored entries / n^2                          */
    int64_t dense_entries;    /* sum m*n over dense leaves                     */
    int64_t rk_entries;       /* sum k*(m+n) over low-rank leaves              */
    int64_t max_rank;         /* largest rank                                  */
    int64_t pool_bytes;       /* bytes the matvec streams (padded factors)     */
    int64_t matvec_bytes;     /* algorithmic bytes of one single-RHS matvec    */
    int64_t n_row_groups;
    int64_t factorized;       /* 1 after lu!                                   */
    int64_t lu_tiles;         /* after lu!: tiles of the tile schedule (0: the recursion ran) */
    int64_t lu_rank_cap;      /* after lu!: column capacity of the low-rank factors */
    int64_t tune_p2_split;    /* launch shapes of the matvec (hm_autotune): CTAs per
                                 1024-row window of phase 2 (2, 4, 8), or 1 for
                                 phase 2 by tree clusters                          */
    int64_t tune_p1_waves;    /* phase-1 grid in resident waves (1, 2, 4)       */
    int64_t tune_tc_nc[3];    /* tensor-core column block for <= 16, <= 32 and
                                 more columns (0: not tuned, the default rule)    */
    int64_t tuned;            /* 1 after hm_autotune                              */
} hm_info_t;

typedef struct hm_handle hm_handle;

/* Library version (major*10000 + minor*100 + patch). */
int hm_version(void);

/* Copy the last error message of the calling thread into buf (NUL-ended). */
int hm_last_error(char* buf, int64_t len);

/* Fill *p with the reference defaults (src/utils.jl:12-23): εComp=1e-10,
 * MaxRank=16, MaxBlock=-1, MinBlock=64, ConsMethod aca2, εTrunc=1e-10,
 * Cauchy kernel with p=1, dim=1, FP64 storage, device 0. */
int hm_default_params(hm_params* p);

/* c,H = NewHmat()  (src/cluster.jl:36-133).
 *   geom      n*dim doubles, column-major, ALREADY permuted (c.X).
 *   cluster tree: ncluster entries in the pre-order of the reference's
 *   downward pass (ids 1..ncluster -> index 0..ncluster-1):
 *   cl_s[i] 0-based start, cl_e[i] exclusive end, cl_left/cl_right child
 *   index or -1 for a leaf (src/cluster.jl:223-240).
 *   nb_pairs  NULL for the identity adjacency Adj = I (two clusters are
 *   neighbours iff their ranges intersect), else 2*n_nb int64 (i, j) cluster
 *   index pairs for which Neighbors[i+1, j+1] != 0 (src/cluster.jl:140-169). */
int hm_new(const hm_params* p, int64_t n, const double* geom,
           int64_t ncluster, const int64_t* cl_s, const int64_t* cl_e,
           const int64_t* cl_left, const int64_t* cl_right,
           int64_t n_nb, const int64_t* nb_pairs, hm_handle** out);

/* The block partition of NewHmat alone (src/cluster.jl:48-133), computed on
 * the host without a device: for leaf i in the reference's order,
 * out[5i..5i+4] = (type 0 dense / 1 low-rank, row0, col0, m, n); *count
 * receives the number of leaves (out may be NULL to ask for it).  Arguments
 * as for hm_new.  The "svd" route decides its blocks by compressing them and
 * is refused (HM_ERR_UNSUPPORTED).  Used to balance row shards over GPUs by
 * the bytes they will store; no counterpart in the reference. */
int hm_partition(const hm_params* p, int64_t n, int64_t ncluster, const int64_t* cl_s, const int64_t* cl_e,
                 const int64_t* cl_left, const int64_t* cl_right, int64_t n_nb, const int64_t* nb_pairs,
                 int64_t cap, int64_t* out, int64_t* count);

/* A new H-matrix on the structure of `ref` (built with HM_BUILD_KEEP_PIVOTS
 * by the aca2 route): same cluster tree, block partition and ranks, and every
 * low-rank block's cross approximation taken at ref's pivot rows and columns,
 * for the kernel parameter, kernel id and shift of p (the other fields of p
 * must equal ref's).  The factors then depend smoothly on the kernel
 * parameter, so finite differences of anything computed from the H-matrix
 * match its derivative (the adjoint checks of the hyper-parameter
 * gradients).  No counterpart in the reference. */
int hm_new_like(const hm_handle* ref, const hm_params* p, hm_handle** out);

/* free a handle */
int hm_destroy(hm_handle* h);

/* info(H) (src/utils.jl:83-110) and roofline byte counts. */
int hm_info(const hm_handle* h, hm_info_t* out);

/* Leaf list in the order of the reference recursion (children [11 12; 21 22]
 * visited 11,12,21,22; src/cluster.jl:122-127): for leaf i,
 * out[6i..6i+5] = (type 0 dense / 1 low-rank, row0, col0, m, n, rank). */
int hm_leaves(const hm_handle* h, int64_t cap, int64_t* out, int64_t* count);

/* Factors of low-rank leaf `leaf` (index in hm_leaves order) as FP64,
 * A (m x k) and B (n x k) column-major, H_leaf = A*B' (src/cluster.jl:118-120). */
int hm_leaf_factors(const hm_handle* h, int64_t leaf, double* A, double* B);

/* Array(H) / to_fmat (src/utils.jl:162-192): n*n doubles column-major.
 * For a factorised handle this is the packed L\U of lu!. */
int hm_to_dense(const hm_handle* h, double* out, uint32_t flags);

/* H*V and H'*V (src/harithm.jl:317-329, 243-260): Y = H*X (trans=0) or
 * Y = H'*X (trans=1); X, Y are n x ncols column-major doubles.  The device
 * kernels stream the stored factors once per call in the handle's storage
 * precision (several columns: once per block of columns).  FP64 factors
 * accumulate in FP64; FP32 and BF16 factors are multiplied in FP32 (one
 * column) or on the tensor cores (several columns: three TF32 products per
 * term for FP32 factors, two BF16 products for BF16 factors) with FP32 partial
 * sums added in FP64.  stream: a cudaStream_t or NULL for the handle's own
 * stream.  With host pointers the call is synchronous and reports a
 * tensor-core pipeline timeout (HM_ERR_TIMEOUT); hm_status reads it after
 * device-pointer calls. */
int hm_matvec(hm_handle* h, const double* X, double* Y, int64_t ncols,
              int32_t trans, uint32_t flags, void* stream);

/* Autotuner of the matvec launch shapes on this handle's own data: times
 * `calls` matvecs (CUDA events, after two untimed ones) for every phase-2
 * shape (2, 4, 8 CTAs per 1024-row window, or, with FP64/FP32 factors, one
 * warp per 128-row chunk of an output cluster, tree level by tree level) and
 * phase-1 grid (1, 2, 4 resident waves) and keeps the fastest; with ncols > 1
 * and FP32/BF16 factors, also the tensor-core column block (16, 32, 64) for
 * that many columns.  The choice stays with the handle (hm_info reports it).
 * The window shapes give bit-identical results; the cluster shape sums the
 * same products in another order.  times (may be NULL) receives 15 mean
 * milliseconds: [3 a + b] for split (2, 4, 8)[a] and waves (1, 2, 4)[b],
 * [9 + q] for column block (16, 32, 64)[q], [12 + b] for the cluster shape and
 * waves (1, 2, 4)[b] (-1: not tried).  No counterpart in the reference. */
int hm_autotune(hm_handle* h, int64_t ncols, int32_t calls, double* times);

/* Sets the single-column matvec launch shapes by hand (a choice hm_autotune
 * made earlier on the same data, say): p2_split 2, 4 or 8 CTAs per phase-2
 * window, or 1 for phase 2 by tree clusters (not with BF16 factors:
 * HM_ERR_UNSUPPORTED); p1_waves 1, 2 or 4.  Other values: HM_ERR_ARG.  No
 * counterpart in the reference. */
int hm_set_tune(hm_handle* h, int32_t p2_split, int32_t p1_waves);

/* Waits for `stream` (NULL: the handle's stream) and reports, once, whether a
 * bounded wait inside the tensor-core kernels gave up since the last check
 * (HM_ERR_TIMEOUT; the results of that call are not valid).  No counterpart in
 * the reference. */
int hm_status(hm_handle* h, void* stream);

/* Self-test of the tensor-core operand layouts of the multi-RHS matvec, on
 * the current device: D = A B' for A 128 x KC and B 2nc x KC (row-major
 * FP32 host arrays, KC = 16 for kind 0 = TF32, 32 for kind 1 = BF16, whose
 * inputs must be exact BF16 values), B staged as the kernels' X / Z tiles and
 * A either as a K-major shared-memory tile (a_src = 0) or in tensor memory as
 * the kernels' converters write it (a_src = 2); D is 128 x 2nc row-major,
 * nc = 16 or 64.  No counterpart in the reference. */
int hm_tc_selftest(int32_t kind, int32_t a_src, int32_t nc, const float* A, const float* B, float* D);

/* R = B - H*X (trans=0) or B - H'*X (trans=1) for n x ncols column-major
 * blocks, every product and sum carried in twice the FP64 precision (error-free
 * TwoProduct/TwoSum, Ogita-Rump-Oishi 2005): the residual of iterative
 * refinement, exact to the last bits of R even where H*X nearly cancels B.
 * hm_solve_refined uses it; so does the GMRES-based refinement of the host
 * mirror.  The unfactorised H is read (a factorised handle keeps it).  No
 * counterpart in the reference. */
int hm_residual(hm_handle* h, const double* X, const double* B, double* R, int64_t ncols,
                int32_t trans, uint32_t flags, void* stream);

/* One single-RHS matvec on device pointers with CUDA events between its three
 * launches; ms[0..2] = x staging, phase 1 (z = B'x per low-rank leaf), phase 2
 * (y = sum A z + dense).  Profiling aid; no counterpart in the reference. */
int hm_matvec_profile(hm_handle* h, const double* X, double* Y, int32_t trans,
                      void* stream, float* ms);

/* Exact FP64 rows of the kernel matrix times x: y[i] = sum_j K(c.X[rows[i]],
 * c.X[j]) x[j] (+ shift*x[rows[i]]), the dense FullMat oracle for sampled rows. */
int hm_exact_rows(hm_handle* h, const int64_t* rows, int64_t nrows,
                  const double* x, double* y, uint32_t flags, void* stream);

/* H + lambda*I (src/harithm.jl:457-473), in place on h; refused with
 * HM_ERR_STATE on a factorised handle (src/harithm.jl:458-460). */
int hm_add_identity(hm_handle* h, double lambda);

/* u*H (src/harithm.jl:478-498), in place. */
int hm_scale(hm_handle* h, double u);

/* copy(H) (src/utils.jl:130-159) */
int hm_copy(const hm_handle* h, hm_handle** out);

/* coarsening(H) (src/utils.jl:29-59): a new H-matrix in which every dense
 * leaf off the diagonal whose truncated SVD rank (S/S[1] > eps_trunc) is at
 * most MaxRank is stored as that low-rank pair.  HM_ERR_STATE on a
 * factorised handle. */
int hm_coarsen(const hm_handle* h, hm_handle** out);

/* a + scalar*b (hadd / hmat_add!, src/harithm.jl:4-159, 374-420; a - b is
 * scalar = -1) as a new H-matrix, for two H-matrices on the same block
 * partition (leaf formats may differ; the format of a is kept, low-rank sums
 * recompressed with eps_trunc).  Different partitions or storage precisions
 * are refused (HM_ERR_UNSUPPORTED), as is a low-rank sum whose ranks add up
 * to more than 96.  The reference's H*H operator (src/harithm.jl:315) calls
 * itself; its hmul serves lu! and is built inside hm_lu. */
int hm_add(const hm_handle* a, const hm_handle* b, double scalar, hm_handle** out);

/* Export / import of a built (unfactorised) H-matrix: parameters, cluster
 * tree, block tree, geometry and factor pools in one binary file, so that a
 * construction is paid once.  No counterpart in the reference (its REQUIRE
 * lists JLD2, unused).  hm_save refuses a factorised handle (HM_ERR_STATE);
 * `user` (user_bytes, may be 0) is stored alongside for the caller (the host
 * mirror keeps the cluster permutation there).  hm_load rebuilds the handle
 * on `device` after checking every index of the file's structure; a file from
 * another build, a truncated or altered file is refused (HM_ERR_ARG /
 * HM_ERR_IO).  hm_load_user reads only the user block: *user_bytes receives
 * its size, and min(cap, size) bytes are copied to user when it is not NULL. */
int hm_save(const hm_handle* h, const char* path, const void* user, int64_t user_bytes);
int hm_load(const char* path, int32_t device, hm_handle** out);
int hm_load_user(const char* path, void* user, int64_t cap, int64_t* user_bytes);

/* lu!(H) (src/hlu.jl:465-515): factorise in place with pivoting inside each
 * diagonal leaf.  HM_ERR_STATE if already factorised (src/hlu.jl:466-468). */
int hm_lu(hm_handle* h);

/* Row permutation P of a factorised handle (0-based; H[P,:] = L*U). */
int hm_lu_perm(const hm_handle* h, int64_t* P);

/* a\y (src/hlu.jl:553-562) with a factorised handle: X = H^{-1} B for ncols
 * right-hand sides (n x ncols column-major).  With HM_FLAG_TRANS it solves
 * H' X = B (U' then L', then the inverse row permutation), the adjoint that
 * the reference does not have. */
int hm_solve(hm_handle* h, const double* B, double* X, int64_t ncols,
             uint32_t flags, void* stream);

/* H\y with iterative refinement: x = (LU)^{-1} b, then r = b - H x with the
 * compensated H-matvec of hm_residual on the unfactorised H (lu! keeps it),
 * x += (LU)^{-1} r, until
 * max over columns |r|/|b| <= tol or max_iter refinement steps.  *iters and
 * *relres (may be NULL) report the steps taken and the final residual.
 * No counterpart in the reference (its \ has no refinement). */
int hm_solve_refined(hm_handle* h, const double* B, double* X, int64_t ncols,
                     double tol, int32_t max_iter, uint32_t flags, void* stream,
                     int32_t* iters, double* relres);

/* ---- independent problems in one call (no counterpart in the reference,
 * whose Julia code handles one H-matrix at a time).  hs holds `count`
 * distinct handles; each is worked on its own stream by one of `nthreads`
 * host threads (0: min(hardware threads, 16)), so the GPU overlaps the
 * problems.  status (optional, count entries) receives each problem's status;
 * the return value is HM_OK or the first failing problem's status, with
 * hm_last_error naming the problem.  A handle listed twice is an error. */

/* lu!(H) on every handle (src/hlu.jl:465-521 each). */
int hm_batch_lu(hm_handle* const* hs, int64_t count, int32_t nthreads, int32_t* status);

/* H\y on every factorized handle: B[i], X[i] are n_i x ncols column-major
 * (host, or device with HM_FLAG_DEVICE_PTRS); HM_FLAG_TRANS solves with H'. */
int hm_batch_solve(hm_handle* const* hs, int64_t count, const double* const* B, double* const* X,
                   int64_t ncols, uint32_t flags, int32_t nthreads, int32_t* status);

/* hm_solve_refined on every factorized handle; iters and relres (optional,
 * count entries) receive each problem's refinement steps and residual. */
int hm_batch_solve_refined(hm_handle* const* hs, int64_t count, const double* const* B,
                           double* const* X, int64_t ncols, double tol, int32_t max_iter,
                           uint32_t flags, int32_t nthreads, int32_t* status, int32_t* iters,
                           double* relres);

/* H*y on every handle (src/harithm.jl:317-329 each), host or device X[i], Y[i]. */
int hm_batch_matvec(hm_handle* const* hs, int64_t count, const double* const* X, double* const* Y,
                    int64_t ncols, int32_t trans, uint32_t flags, int32_t nthreads, int32_t* status);

/* Drop-in for the reference's native entry point
 * int aca_wrapper(double*, double*, double*, int, int, double, int)
 * (deps/src/ACA_FullyPivoted.cpp:218-236, called from src/hlu.jl:12-13):
 * fully pivoted ACA of the column-major m x n host matrix AA; at most
 * rank+1 columns are written to UU (m x .) and VV (n x .); returns the
 * untruncated rank, or a negative status on error. */
int aca_wrapper(double* AA, double* UU, double* VV, int m, int n,
                double epsilon, int rank);

/* Allocation-free aca_wrapper for callers that cannot call cudaMalloc (their
 * device memory belongs to another allocator's pool, or they cannot afford the
 * synchronisation an allocation implies).  No counterpart in the reference.
 * A (m x n), UU (m x min(m,n,rank+1)) and VV (n x min(m,n,rank+1)) are device
 * pointers on the current device, column-major; the result equals
 * aca_wrapper's and the untruncated rank (at most min(m,n)) is returned
 * (negative status on error).  The residual lives in a fixed device array of
 * 2^18 - 32 doubles shared by all calls: m*n + m + n must not exceed that
 * (HM_ERR_ARG otherwise), calls that overlap on the GPU race, and the first
 * call on a device (which looks the array up) should come before any stream
 * capture.  Each call reads the rank back to the host, so it returns only
 * once `stream` has finished its work.  The looked-up address is kept until
 * the process exits: do not use this entry point on a device across a
 * cudaDeviceReset.  stream: a cudaStream_t or NULL for the legacy default
 * stream. */
int aca_wrapper_noalloc(const double* AA, double* UU, double* VV, int m, int n,
                        double epsilon, int rank, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HMATRIX_B200_H */
