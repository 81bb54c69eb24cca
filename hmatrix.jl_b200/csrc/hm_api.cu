// C ABI of libhmatb200 (declared in include/hmatrix_b200.h).
#include "hm_internal.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <set>
#include <thread>
#include <atomic>

namespace hm {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  // a failed runtime call (an allocation that did not fit, for one) leaves its
  // code as the thread's pending CUDA error; clear it, so that the next
  // entry point's launch check does not report it a second time
  if (code == HM_ERR_OOM || code == HM_ERR_CUDA) (void)cudaGetLastError();
  return code;
}

cudaError_t smem_attr(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({kernel, dev})) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.insert({kernel, dev});
  return e;
}

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int check_params(const hm_params* p) {
  if (!p) return fail(HM_ERR_ARG, "params is NULL");
  if (p->dim < 1 || p->dim > 3) return fail(HM_ERR_ARG, "dim must be 1, 2 or 3");
  if (p->kernel < HM_KERNEL_CAUCHY || p->kernel > HM_KERNEL_GAUSS_DP)
    return fail(HM_ERR_ARG, "unknown kernel id " + std::to_string(p->kernel) +
                                "; Hparams.Kernel must map to HM_KERNEL_*");
  // > 0 for every kernel: 1/(c + |x-y|^2) with c <= 0 is infinite or negative
  // where points meet, and the others divide by their parameter
  if (!(p->kparam > 0.0) || !std::isfinite(p->kparam))
    return fail(HM_ERR_ARG, "kernel parameter must be finite and > 0");
  if (!std::isfinite(p->shift)) return fail(HM_ERR_NONFINITE, "shift is not finite");
  if (p->max_rank < 1 || p->max_rank > 64) return fail(HM_ERR_ARG, "MaxRank must be in [1, 64]");
  if (p->min_block < 1) return fail(HM_ERR_ARG, "MinBlock must be >= 1");
  if (p->cons_method != HM_CONS_ACA2 && p->cons_method != HM_CONS_SVD && p->cons_method != HM_CONS_BBFMM)
    return fail(HM_ERR_ARG, "ConsMethod must be aca2, svd or bbfmm (separate needs user closures)");
  if (p->cons_method == HM_CONS_BBFMM && p->dim > 2)
    return fail(HM_ERR_UNSUPPORTED, "bbfmm construction takes 1-D or 2-D geometry (deps/src/lowrank.cpp:186-222)");
  if (p->storage != HM_F64 && p->storage != HM_F32 && p->storage != HM_BF16)
    return fail(HM_ERR_ARG, "storage must be HM_F64, HM_F32 or HM_BF16");
  if (!(p->eps_trunc >= 0.0) || !(p->eps_comp >= 0.0)) return fail(HM_ERR_ARG, "tolerances must be >= 0");
  return HM_OK;
}

struct IoBuf {
  hm_handle* h;
  double* ptr = nullptr;
  int get(size_t bytes) {
    if (h->io_bytes < bytes) {
      if (h->d_io) cudaFree(h->d_io);
      h->d_io = nullptr;
      h->io_bytes = 0;
      cudaError_t e = cudaMalloc(&h->d_io, bytes);
      if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("staging buffer: ") + cudaGetErrorString(e));
      h->io_bytes = bytes;
    }
    ptr = h->d_io;
    return HM_OK;
  }
};

// Runs fn(i) for i in [0, count) on up to nthreads host threads (the calling
// thread is one of them) and folds the per-problem statuses.
template <typename F>
int run_batch(hm_handle* const* hs, int64_t count, int32_t nthreads, int32_t* status, F fn) {
  if (count < 0 || (count > 0 && !hs)) return fail(HM_ERR_ARG, "invalid batch");
  if (count == 0) return HM_OK;
  {
    std::set<const hm_handle*> seen;
    for (int64_t i = 0; i < count; ++i) {
      if (!hs[i]) return fail(HM_ERR_ARG, "batch entry " + std::to_string(i) + " is NULL");
      if (!seen.insert(hs[i]).second)
        return fail(HM_ERR_ARG, "batch entry " + std::to_string(i) + " repeats a handle");
    }
  }
  const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
  const int64_t T = std::min<int64_t>(nthreads > 0 ? nthreads : std::min<int64_t>(hw, 16), count);
  std::vector<int> st((size_t)count, HM_OK);
  std::vector<std::string> msg((size_t)count);
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const int64_t i = next.fetch_add(1);
      if (i >= count) break;
      st[i] = fn(i);
      if (st[i] != HM_OK) msg[i] = g_last_error;     // this worker's own message
    }
  };
  std::vector<std::thread> th;
  try {
    for (int64_t t = 1; t < T; ++t) th.emplace_back(worker);
  } catch (const std::exception&) {
    // fewer threads than asked: the ones running (and this one) take the rest
  }
  worker();
  for (auto& t : th) t.join();
  int first = HM_OK;
  for (int64_t i = 0; i < count; ++i) {
    if (status) status[i] = st[i];
    if (st[i] != HM_OK && first == HM_OK) {
      first = st[i];
      fail(st[i], "problem " + std::to_string(i) + ": " + msg[i]);
    }
  }
  return first;
}

// Times `calls` launches of fn on the handle's stream (after two untimed
// ones) and returns the mean milliseconds, or a negative value on error.
template <typename F>
float time_calls(hm_handle* h, int calls, F fn) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return -1.f;
  float ms = -1.f;
  bool ok = fn() == HM_OK && fn() == HM_OK;
  if (ok && cudaEventRecord(a, h->stream) == cudaSuccess) {
    for (int i = 0; i < calls && ok; ++i) ok = fn() == HM_OK;
    if (ok && cudaEventRecord(b, h->stream) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess &&
        cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
      ms /= calls;
    else
      ms = -1.f;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms;
}

}  // namespace
}  // namespace hm

using namespace hm;

extern "C" {

int hm_version(void) { return 100; }

int hm_last_error(char* buf, int64_t len) {
  if (!buf || len <= 0) return HM_ERR_ARG;
  std::strncpy(buf, g_last_error.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return HM_OK;
}

int hm_default_params(hm_params* p) {
  if (!p) return fail(HM_ERR_ARG, "params is NULL");
  std::memset(p, 0, sizeof(*p));
  p->dim = 1;
  p->kernel = HM_KERNEL_CAUCHY;
  p->kparam = 1.0;
  p->shift = 0.0;
  p->eps_comp = 1e-10;
  p->eps_trunc = 1e-10;
  p->max_rank = 16;
  p->max_block = -1;
  p->min_block = 64;
  p->cons_method = HM_CONS_ACA2;
  p->aca_force = 0;
  p->storage = HM_F64;
  p->device = 0;
  p->rank_cap = 0;
  return HM_OK;
}

int hm_new(const hm_params* p, int64_t n, const double* geom, int64_t ncluster, const int64_t* cl_s,
           const int64_t* cl_e, const int64_t* cl_left, const int64_t* cl_right, int64_t n_nb,
           const int64_t* nb_pairs, hm_handle** out) {
  if (!out) return fail(HM_ERR_ARG, "out is NULL");
  *out = nullptr;
  HM_TRY(check_params(p));
  if (n < 1 || !geom || ncluster < 1 || !cl_s || !cl_e || !cl_left || !cl_right)
    return fail(HM_ERR_ARG, "invalid geometry or cluster arrays");
  // a NaN or infinite coordinate would make every kernel value of its row and
  // column non-finite; refuse it before anything reaches the device
  for (int64_t i = 0; i < n * (int64_t)p->dim; ++i)
    if (!std::isfinite(geom[i]))
      return fail(HM_ERR_NONFINITE, "geometry: coordinate " + std::to_string(i / n) + " of point " +
                                        std::to_string(i % n) + " is not finite");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(HM_ERR_CUDA, "no CUDA device: the H-matrix path has no CPU fallback");
  if (p->device < 0 || p->device >= ndev) return fail(HM_ERR_ARG, "invalid device ordinal");
  DeviceGuard g(p->device);
  hm_handle* h = new (std::nothrow) hm_handle();
  if (!h) return fail(HM_ERR_OOM, "host allocation");
  h->prm = *p;
  if (h->prm.max_block == -1) h->prm.max_block = (int32_t)(n / 4);   // src/cluster.jl:37-39
  h->n = n;
  h->dim = p->dim;
  h->device = p->device;
  h->storage = p->storage;
  h->kd = KernelDesc{p->kernel, p->dim, p->kparam, p->shift};
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return fail(HM_ERR_CUDA, cudaGetErrorString(e)); }
  int s = build_handle(h, geom, ncluster, cl_s, cl_e, cl_left, cl_right, n_nb, nb_pairs);
  if (s != HM_OK) {
    std::string msg = g_last_error;
    free_handle_data(h);
    cudaStreamDestroy(h->stream);
    delete h;
    return fail(s, msg);
  }
  *out = h;
  return HM_OK;
}

int hm_new_like(const hm_handle* ref, const hm_params* p, hm_handle** out) {
  if (!out || !ref) return fail(HM_ERR_ARG, "NULL argument");
  *out = nullptr;
  HM_TRY(check_params(p));
  if (ref->factorized) return fail(HM_ERR_STATE, "the reference H-matrix is factorised");
  const hm_params& r = ref->prm;
  if (p->dim != r.dim || p->cons_method != HM_CONS_ACA2 || r.cons_method != HM_CONS_ACA2 ||
      p->max_rank != r.max_rank || p->min_block != r.min_block ||
      (p->max_block != r.max_block && !(p->max_block == -1)) || p->storage != r.storage ||
      p->row_lo != r.row_lo || p->row_hi != r.row_hi)
    return fail(HM_ERR_ARG, "hm_new_like: only the kernel, its parameter and the shift may differ from the reference");
  DeviceGuard g(ref->device);
  hm_handle* h = new (std::nothrow) hm_handle();
  if (!h) return fail(HM_ERR_OOM, "host allocation");
  h->prm = *p;
  h->prm.max_block = r.max_block;
  h->prm.device = ref->device;
  h->n = ref->n;
  h->dim = ref->dim;
  h->device = ref->device;
  h->storage = ref->storage;
  h->kd = KernelDesc{p->kernel, p->dim, p->kparam, p->shift};
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return fail(HM_ERR_CUDA, cudaGetErrorString(e)); }
  int s = build_like(h, ref);
  if (s != HM_OK) {
    std::string msg = g_last_error;
    free_handle_data(h);
    cudaStreamDestroy(h->stream);
    delete h;
    return fail(s, msg);
  }
  *out = h;
  return HM_OK;
}

int hm_destroy(hm_handle* h) {
  if (!h) return HM_OK;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  free_handle_data(h);
  cudaStreamDestroy(h->stream);
  delete h;
  return HM_OK;
}

int hm_info(const hm_handle* h, hm_info_t* o) {
  if (!h || !o) return fail(HM_ERR_ARG, "NULL argument");
  std::memset(o, 0, sizeof(*o));
  o->n = h->n;
  o->depth = h->depth;
  double stored = 0.0;
  for (auto& L : h->leaves) {
    if (L.type == T_DENSE) {
      o->n_dense++;
      o->dense_entries += (int64_t)L.m * L.n;
      stored += (double)L.m * L.n;
    } else {
      o->n_rk++;
      o->rk_entries += (int64_t)L.k * (L.m + L.n);
      o->max_rank = std::max<int64_t>(o->max_rank, L.k);
      stored += (double)L.k * (L.m + L.n);
    }
  }
  o->compress_ratio = stored / (double)h->n / (double)h->n;
  o->pool_bytes = (int64_t)(h->rk_bytes + h->dense_bytes);
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  o->matvec_bytes = (int64_t)eb * o->rk_entries + (int64_t)deb * o->dense_entries + 16 * h->n;
  o->n_row_groups = h->fwd.nwin;
  o->factorized = h->factorized ? 1 : 0;
  o->tune_p2_split = h->tune.p2_split;
  o->tune_p1_waves = h->tune.p1_waves;
  for (int b = 0; b < 3; ++b) o->tune_tc_nc[b] = h->tune.tc_nc[b];
  o->tuned = h->tune.tuned;
  if (h->lu) lu_describe(h, &o->lu_tiles, &o->lu_rank_cap);
  return HM_OK;
}

int hm_partition(const hm_params* p, int64_t n, int64_t ncluster, const int64_t* cl_s, const int64_t* cl_e,
                 const int64_t* cl_left, const int64_t* cl_right, int64_t n_nb, const int64_t* nb_pairs,
                 int64_t cap, int64_t* out, int64_t* count) {
  HM_TRY(check_params(p));
  if (!count || n < 1 || ncluster < 1 || !cl_s || !cl_e || !cl_left || !cl_right)
    return fail(HM_ERR_ARG, "invalid cluster arrays");
  hm_handle h;
  h.prm = *p;
  if (h.prm.max_block == -1) h.prm.max_block = (int32_t)(n / 4);   // src/cluster.jl:37-39
  h.n = n;
  h.dim = p->dim;
  HM_TRY(partition_only(&h, ncluster, cl_s, cl_e, cl_left, cl_right, n_nb, nb_pairs));
  *count = (int64_t)h.leaves.size();
  if (!out) return HM_OK;
  if (cap < *count) return fail(HM_ERR_ARG, "leaf buffer too small");
  for (size_t i = 0; i < h.leaves.size(); ++i) {
    const Leaf& L = h.leaves[i];
    int64_t* o = out + 5 * i;
    o[0] = L.type == T_DENSE ? 0 : 1;
    o[1] = L.row0; o[2] = L.col0; o[3] = L.m; o[4] = L.n;
  }
  return HM_OK;
}

int hm_leaves(const hm_handle* h, int64_t cap, int64_t* out, int64_t* count) {
  if (!h || !count) return fail(HM_ERR_ARG, "NULL argument");
  *count = (int64_t)h->leaves.size();
  if (!out) return HM_OK;
  if (cap < *count) return fail(HM_ERR_ARG, "leaf buffer too small");
  for (size_t i = 0; i < h->leaves.size(); ++i) {
    const Leaf& L = h->leaves[i];
    int64_t* o = out + 6 * i;
    o[0] = L.type == T_DENSE ? 0 : 1;
    o[1] = L.row0; o[2] = L.col0; o[3] = L.m; o[4] = L.n; o[5] = L.k;
  }
  return HM_OK;
}

int hm_leaf_factors(const hm_handle* h, int64_t leaf, double* A, double* B) {
  if (!h || !A || !B) return fail(HM_ERR_ARG, "NULL argument");
  if (leaf < 0 || leaf >= (int64_t)h->leaves.size()) return fail(HM_ERR_ARG, "leaf index out of range");
  if (h->factorized) return fail(HM_ERR_STATE, "factors of a factorised handle are held by the LU state");
  DeviceGuard g(h->device);
  return leaf_factors_f64(h, leaf, A, B);
}

int hm_to_dense(const hm_handle* h, double* out, uint32_t flags) {
  if (!h || !out) return fail(HM_ERR_ARG, "NULL argument");
  DeviceGuard g(h->device);
  const size_t bytes = sizeof(double) * (size_t)h->n * (size_t)h->n;
  double* d = out;
  if (!(flags & HM_FLAG_DEVICE_PTRS)) {
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return fail(HM_ERR_OOM, "to_dense buffer");
  }
  int s = h->factorized ? lu_to_dense(h, d) : to_dense(h, d);
  if (s == HM_OK && !(flags & HM_FLAG_DEVICE_PTRS)) {
    cudaError_t e = cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) s = fail(HM_ERR_CUDA, cudaGetErrorString(e));
  }
  if (!(flags & HM_FLAG_DEVICE_PTRS)) cudaFree(d);
  return s;
}

int hm_matvec(hm_handle* h, const double* X, double* Y, int64_t ncols, int32_t trans, uint32_t flags, void* stream) {
  if (!h || !X || !Y || ncols < 0) return fail(HM_ERR_ARG, "invalid argument");
  if (h->factorized) return fail(HM_ERR_STATE, "H is factorised; the matvec reads the unfactorised H");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  const int64_t n = h->n;
  // one column: the single-vector kernels; a block: every factor streamed once per column block
  // (FP32/BF16 factors: on the tensor cores unless HM_FLAG_MV_SIMT)
  const bool simt = (flags & HM_FLAG_MV_SIMT) != 0;
  auto run = [&](const double* dx, double* dy) -> int {
    if (ncols == 1) return matvec_device(h, dx, dy, trans ? 1 : 0, st);
    return matvec_multi_device(h, dx, dy, ncols, trans ? 1 : 0, st, simt);
  };
  if (ncols == 0) return HM_OK;
  if (flags & HM_FLAG_DEVICE_PTRS) return run(X, Y);
  IoBuf io{h};
  HM_TRY(io.get(sizeof(double) * 2 * n * ncols));
  HM_CUDA_TRY(cudaMemcpyAsync(io.ptr, X, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, st));
  HM_TRY(run(io.ptr, io.ptr + n * ncols));
  HM_CUDA_TRY(cudaMemcpyAsync(Y, io.ptr + n * ncols, sizeof(double) * n * ncols, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  return tc_status(h, st);
}

int hm_residual(hm_handle* h, const double* X, const double* B, double* R, int64_t ncols, int32_t trans,
                uint32_t flags, void* stream) {
  if (!h || !X || !B || !R || ncols < 0) return fail(HM_ERR_ARG, "invalid argument");
  if (h->factorized && !h->lu) return fail(HM_ERR_STATE, "H is factorised");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  const int64_t n = h->n;
  if (ncols == 0) return HM_OK;
  auto run = [&](const double* dx, const double* db, double* dr) -> int {
    for (int64_t q = 0; q < ncols; ++q) HM_TRY(residual_device(h, dx + q * n, db + q * n, dr + q * n, trans ? 1 : 0, st));
    return HM_OK;
  };
  if (flags & HM_FLAG_DEVICE_PTRS) return run(X, B, R);
  IoBuf io{h};
  HM_TRY(io.get(sizeof(double) * 3 * n * ncols));
  HM_CUDA_TRY(cudaMemcpyAsync(io.ptr, X, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, st));
  HM_CUDA_TRY(cudaMemcpyAsync(io.ptr + n * ncols, B, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, st));
  HM_TRY(run(io.ptr, io.ptr + n * ncols, io.ptr + 2 * n * ncols));
  HM_CUDA_TRY(cudaMemcpyAsync(R, io.ptr + 2 * n * ncols, sizeof(double) * n * ncols, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  return HM_OK;
}

int hm_tc_selftest(int32_t kind, int32_t a_src, int32_t nc, const float* A, const float* B, float* D) {
  if (!A || !B || !D) return fail(HM_ERR_ARG, "invalid argument");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HM_ERR_CUDA, "no CUDA device");
  return tc_selftest(kind, a_src, nc, A, B, D);
}

int hm_autotune(hm_handle* h, int64_t ncols, int32_t calls, double* times) {
  if (!h || ncols < 1 || calls < 1) return fail(HM_ERR_ARG, "invalid argument");
  if (h->factorized) return fail(HM_ERR_STATE, "H is factorised");
  DeviceGuard g(h->device);
  const int64_t n = h->n;
  double* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, sizeof(double) * 2 * (size_t)n * (size_t)ncols);
  if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("autotune buffers: ") + cudaGetErrorString(e));
  struct Free { double* p; ~Free() { cudaFree(p); } } fr{buf};
  HM_CUDA_TRY(cudaMemsetAsync(buf, 0, sizeof(double) * (size_t)n * (size_t)ncols, h->stream));
  double* x = buf;
  double* y = buf + n * ncols;
  // single right-hand side: phase-2 split x phase-1 waves
  float best = -1.f;
  hm_handle::Tune keep = h->tune;
  const int splits[3] = {2, 4, 8}, waves[3] = {1, 2, 4};
  if (times)
    for (int i = 0; i < 15; ++i) times[i] = -1.0;
  auto try_shape = [&](int split, int b, int slot) -> int {
    h->tune.p2_split = split;
    h->tune.p1_waves = waves[b];
    const float ms = time_calls(h, calls, [&] { return matvec_device(h, x, y, 0, h->stream); });
    if (ms < 0) { h->tune = keep; return fail(HM_ERR_CUDA, "autotune: a timed matvec failed"); }
    if (times) times[slot] = ms;
    if (best < 0 || ms < best) { best = ms; keep.p2_split = split; keep.p1_waves = waves[b]; }
    return HM_OK;
  };
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) HM_TRY(try_shape(splits[a], b, 3 * a + b));
  // phase 2 by tree clusters (FP64 and FP32 factors; BF16 factors have their own phase 2)
  if (h->storage != HM_BF16)
    for (int b = 0; b < 3; ++b) HM_TRY(try_shape(1, b, 12 + b));
  h->tune = keep;
  // several columns on the tensor cores: the column block
  if (ncols > 1 && (h->storage == HM_F32 || h->storage == HM_BF16)) {
    const int bucket = ncols <= 16 ? 0 : (ncols <= 32 ? 1 : 2);
    float bm = -1.f;
    int bnc = 0;
    const int ncs[3] = {16, 32, 64};
    for (int q = 0; q < 3; ++q) {
      const int nc = ncs[q];
      if ((bucket == 0 && nc > 16) || (bucket == 1 && nc > 32)) continue;
      h->tune.tc_nc[bucket] = nc;
      const float ms = time_calls(h, calls, [&] { return matvec_multi_device(h, x, y, ncols, 0, h->stream); });
      if (ms < 0) { h->tune.tc_nc[bucket] = 0; return fail(HM_ERR_CUDA, "autotune: a timed block product failed"); }
      if (times) times[9 + q] = ms;
      if (bm < 0 || ms < bm) { bm = ms; bnc = nc; }
    }
    h->tune.tc_nc[bucket] = bnc;
    HM_TRY(tc_status(h, h->stream));
  }
  h->tune.tuned = 1;
  return HM_OK;
}

int hm_set_tune(hm_handle* h, int32_t p2_split, int32_t p1_waves) {
  if (!h) return fail(HM_ERR_ARG, "invalid argument");
  if (p2_split != 1 && p2_split != 2 && p2_split != 4 && p2_split != 8)
    return fail(HM_ERR_ARG, "phase-2 shape must be 1, 2, 4 or 8");
  if (p1_waves != 1 && p1_waves != 2 && p1_waves != 4) return fail(HM_ERR_ARG, "phase-1 waves must be 1, 2 or 4");
  if (p2_split == 1 && h->storage == HM_BF16)
    return fail(HM_ERR_UNSUPPORTED, "phase 2 by tree clusters needs FP64 or FP32 factors");
  h->tune.p2_split = p2_split;
  h->tune.p1_waves = p1_waves;
  return HM_OK;
}

int hm_status(hm_handle* h, void* stream) {
  if (!h) return fail(HM_ERR_ARG, "invalid argument");
  DeviceGuard g(h->device);
  return tc_status(h, stream ? (cudaStream_t)stream : h->stream);
}

int hm_matvec_profile(hm_handle* h, const double* X, double* Y, int32_t trans, void* stream, float* ms) {
  if (!h || !X || !Y || !ms) return fail(HM_ERR_ARG, "invalid argument");
  if (h->factorized) return fail(HM_ERR_STATE, "H is factorised");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  cudaEvent_t ev[4];
  for (int i = 0; i < 4; ++i) HM_CUDA_TRY(cudaEventCreate(&ev[i]));
  int s = matvec_device(h, X, Y, trans ? 1 : 0, st, ev);
  if (s == HM_OK) {
    HM_CUDA_TRY(cudaEventSynchronize(ev[3]));
    for (int i = 0; i < 3; ++i) HM_CUDA_TRY(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
  }
  for (int i = 0; i < 4; ++i) cudaEventDestroy(ev[i]);
  return s;
}

int hm_exact_rows(hm_handle* h, const int64_t* rows, int64_t nrows, const double* x, double* y, uint32_t flags,
                  void* stream) {
  if (!h || !rows || !x || !y || nrows < 0) return fail(HM_ERR_ARG, "invalid argument");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  if (flags & HM_FLAG_DEVICE_PTRS) return exact_rows_device(h, rows, nrows, x, y, st);
  for (int64_t i = 0; i < nrows; ++i)
    if (rows[i] < 0 || rows[i] >= h->n) return fail(HM_ERR_ARG, "row index out of range");
  int64_t* dr = nullptr;
  double *dx = nullptr, *dy = nullptr;
  HM_CUDA_TRY(cudaMalloc(&dr, 8 * std::max<int64_t>(nrows, 1)));
  HM_CUDA_TRY(cudaMalloc(&dx, 8 * h->n));
  HM_CUDA_TRY(cudaMalloc(&dy, 8 * std::max<int64_t>(nrows, 1)));
  HM_CUDA_TRY(cudaMemcpyAsync(dr, rows, 8 * nrows, cudaMemcpyHostToDevice, st));
  HM_CUDA_TRY(cudaMemcpyAsync(dx, x, 8 * h->n, cudaMemcpyHostToDevice, st));
  int s = exact_rows_device(h, dr, nrows, dx, dy, st);
  if (s == HM_OK) HM_CUDA_TRY(cudaMemcpyAsync(y, dy, 8 * nrows, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  cudaFree(dr); cudaFree(dx); cudaFree(dy);
  return s;
}

int hm_add_identity(hm_handle* h, double lambda) {
  if (!h) return fail(HM_ERR_ARG, "NULL handle");
  if (h->factorized) return fail(HM_ERR_STATE, "Hmatrix is frozen after factorization");
  DeviceGuard g(h->device);
  return apply_shift(h, lambda);
}

int hm_scale(hm_handle* h, double u) {
  if (!h) return fail(HM_ERR_ARG, "NULL handle");
  if (h->factorized) return fail(HM_ERR_STATE, "Hmatrix is frozen after factorization");
  DeviceGuard g(h->device);
  tc_factors_changed(h);
  return apply_scale(h, u);
}

int hm_copy(const hm_handle* h, hm_handle** out) {
  if (!h || !out) return fail(HM_ERR_ARG, "NULL argument");
  DeviceGuard g(h->device);
  return copy_handle(h, out);
}

int hm_coarsen(const hm_handle* h, hm_handle** out) {
  if (!h || !out) return fail(HM_ERR_ARG, "NULL argument");
  *out = nullptr;
  DeviceGuard g(h->device);
  return coarsen_handle(h, out);
}

int hm_add(const hm_handle* a, const hm_handle* b, double scalar, hm_handle** out) {
  if (!a || !b || !out) return fail(HM_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (a->device != b->device) return fail(HM_ERR_UNSUPPORTED, "hadd: the H-matrices live on different devices");
  DeviceGuard g(a->device);
  return add_handles(a, b, scalar, out);
}

int hm_save(const hm_handle* h, const char* path, const void* user, int64_t user_bytes) {
  if (!h || !path) return fail(HM_ERR_ARG, "NULL argument");
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  return save_handle(h, path, user, user_bytes);
}

int hm_load(const char* path, int32_t device, hm_handle** out) {
  if (!path || !out) return fail(HM_ERR_ARG, "NULL argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(HM_ERR_CUDA, "no CUDA device: the H-matrix path has no CPU fallback");
  if (device < 0 || device >= ndev) return fail(HM_ERR_ARG, "invalid device ordinal");
  DeviceGuard g(device);
  try {
    return load_handle(path, device, check_params, out);
  } catch (const std::bad_alloc&) {
    return fail(HM_ERR_OOM, "load: host allocation");
  }
}

int hm_load_user(const char* path, void* user, int64_t cap, int64_t* user_bytes) {
  if (!path) return fail(HM_ERR_ARG, "NULL argument");
  return load_user(path, user, cap, user_bytes);
}

int hm_lu(hm_handle* h) {
  if (!h) return fail(HM_ERR_ARG, "NULL handle");
  if (h->factorized) return fail(HM_ERR_STATE, "H-matrix H is already factorized; reuse factorization");
  if (h->prm.row_hi > h->prm.row_lo) return fail(HM_ERR_UNSUPPORTED, "lu! of a row shard of H");
  DeviceGuard g(h->device);
  return lu_factor(h);
}

int hm_lu_perm(const hm_handle* h, int64_t* P) {
  if (!h || !P) return fail(HM_ERR_ARG, "NULL argument");
  if (!h->factorized) return fail(HM_ERR_STATE, "a has not been factorized");
  return lu_perm(h, P);
}

int hm_solve(hm_handle* h, const double* B, double* X, int64_t ncols, uint32_t flags, void* stream) {
  if (!h || !B || !X || ncols < 0) return fail(HM_ERR_ARG, "invalid argument");
  if (!h->factorized) return fail(HM_ERR_STATE, "a has not been factorized");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  const int64_t n = h->n;
  const int trans = (flags & HM_FLAG_TRANS) ? 1 : 0;
  if (flags & HM_FLAG_DEVICE_PTRS) return lu_solve_device(h, B, X, ncols, trans, st);
  IoBuf io{h};
  HM_TRY(io.get(sizeof(double) * 2 * n * std::max<int64_t>(ncols, 1)));
  HM_CUDA_TRY(cudaMemcpyAsync(io.ptr, B, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, st));
  HM_TRY(lu_solve_device(h, io.ptr, io.ptr + n * ncols, ncols, trans, st));
  HM_CUDA_TRY(cudaMemcpyAsync(X, io.ptr + n * ncols, sizeof(double) * n * ncols, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  return HM_OK;
}

int hm_solve_refined(hm_handle* h, const double* B, double* X, int64_t ncols, double tol, int32_t max_iter,
                     uint32_t flags, void* stream, int32_t* iters, double* relres) {
  if (!h || !B || !X || ncols < 0 || max_iter < 0) return fail(HM_ERR_ARG, "invalid argument");
  if (!h->factorized) return fail(HM_ERR_STATE, "a has not been factorized");
  DeviceGuard g(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  const int64_t n = h->n;
  const int trans = (flags & HM_FLAG_TRANS) ? 1 : 0;
  int it = 0;
  double rr = 0.0;
  int s;
  if (flags & HM_FLAG_DEVICE_PTRS) {
    s = lu_solve_refined(h, B, X, ncols, trans, tol, max_iter, st, &it, &rr);
  } else {
    double* d = nullptr;
    HM_CUDA_TRY(cudaMallocAsync(&d, sizeof(double) * 2 * n * std::max<int64_t>(ncols, 1), st));
    HM_CUDA_TRY(cudaMemcpyAsync(d, B, sizeof(double) * n * ncols, cudaMemcpyHostToDevice, st));
    s = lu_solve_refined(h, d, d + n * ncols, ncols, trans, tol, max_iter, st, &it, &rr);
    if (s == HM_OK)
      HM_CUDA_TRY(cudaMemcpyAsync(X, d + n * ncols, sizeof(double) * n * ncols, cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(d, st);
    HM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (iters) *iters = it;
  if (relres) *relres = rr;
  return s;
}

int hm_batch_lu(hm_handle* const* hs, int64_t count, int32_t nthreads, int32_t* status) {
  return run_batch(hs, count, nthreads, status, [&](int64_t i) { return hm_lu(hs[i]); });
}

int hm_batch_solve(hm_handle* const* hs, int64_t count, const double* const* B, double* const* X,
                   int64_t ncols, uint32_t flags, int32_t nthreads, int32_t* status) {
  if (count > 0 && (!B || !X)) return fail(HM_ERR_ARG, "NULL B or X");
  return run_batch(hs, count, nthreads, status,
                   [&](int64_t i) { return hm_solve(hs[i], B[i], X[i], ncols, flags, nullptr); });
}

int hm_batch_solve_refined(hm_handle* const* hs, int64_t count, const double* const* B,
                           double* const* X, int64_t ncols, double tol, int32_t max_iter,
                           uint32_t flags, int32_t nthreads, int32_t* status, int32_t* iters,
                           double* relres) {
  if (count > 0 && (!B || !X)) return fail(HM_ERR_ARG, "NULL B or X");
  return run_batch(hs, count, nthreads, status, [&](int64_t i) {
    return hm_solve_refined(hs[i], B[i], X[i], ncols, tol, max_iter, flags, nullptr,
                            iters ? iters + i : nullptr, relres ? relres + i : nullptr);
  });
}

int hm_batch_matvec(hm_handle* const* hs, int64_t count, const double* const* X, double* const* Y,
                    int64_t ncols, int32_t trans, uint32_t flags, int32_t nthreads, int32_t* status) {
  if (count > 0 && (!X || !Y)) return fail(HM_ERR_ARG, "NULL X or Y");
  return run_batch(hs, count, nthreads, status,
                   [&](int64_t i) { return hm_matvec(hs[i], X[i], Y[i], ncols, trans, flags, nullptr); });
}

int aca_wrapper(double* AA, double* UU, double* VV, int m, int n, double epsilon, int rank) {
  if (!AA || !UU || !VV || m <= 0 || n <= 0 || rank < 0) {
    fail(HM_ERR_ARG, "aca_wrapper: invalid argument");
    return -HM_ERR_ARG;
  }
  int r = 0;
  int s = aca_fp_host(AA, UU, VV, m, n, epsilon, rank, &r);
  return s == HM_OK ? r : -s;
}

}  // extern "C"
