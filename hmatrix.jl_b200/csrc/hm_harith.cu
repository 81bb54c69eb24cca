// Whole-H-matrix arithmetic that changes leaf formats: coarsening
// (src/utils.jl:29-59) and the public H + H (hadd / hmat_add!,
// src/harithm.jl:4-159, 374-420).  Both produce a new handle on the same
// cluster and block trees: the leaf formats and ranks are decided in a first
// pass on the device, the pools are laid out for them, and a second pass
// recomputes each changed leaf straight into the new pools (so the scratch
// stays bounded for any n).
//
// Device pieces: form_kernel builds FP64 blocks alpha0*t0 + alpha1*t1 from
// dense or low-rank terms of either handle; compression is the fully pivoted
// ACA + QR/Jacobi-SVD core of the "svd" construction route; pack kernels write
// FP64 results in the storage precision and padded layout of the new pools;
// copy_blocks_kernel moves the leaves that do not change.
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace hm {

namespace {

struct Term {
  int32_t type;       // -1 none, T_DENSE, T_RK
  int32_t k;
  int32_t src;        // 0: first handle's pools, 1: second handle's
  int32_t pad;
  int64_t off;        // element offset of the leaf in its pool
  double alpha;
};

struct FormJob {
  Term t[2];
  int32_t m, n;
  int64_t out;        // double offset of the m x n result (ld m) in the scratch
};

template <typename T, typename TD>
__device__ __forceinline__ double term_value(const Term& t, int m, int n, int i, int j, const T* rk,
                                             const TD* dn) {
  const int eb = (int)sizeof(T), deb = (int)sizeof(TD);
  if (t.type == T_DENSE) return (double)dn[t.off + i + (int64_t)j * col_pad_dev(m, deb)];
  const int64_t npad = col_pad_dev(n, eb), mpad = col_pad_dev(m, eb);
  const T* B = rk + t.off;
  const T* A = B + npad * t.k;
  double v = 0.0;
  for (int q = 0; q < t.k; ++q) v = fma(from_store<T>(A[i + q * mpad]), from_store<T>(B[j + q * npad]), v);
  return v;
}

// out = alpha0 * t0 (+ alpha1 * t1 as fma); |out|_F^2 and sum|out| per job
template <typename T, typename TD>
__global__ void __launch_bounds__(256) form_kernel(const FormJob* __restrict__ jobs, const T* rk0, const TD* dn0,
                                                   const T* rk1, const TD* dn1, double* __restrict__ scratch,
                                                   double* __restrict__ fro2, double* __restrict__ sabs) {
  __shared__ double red[32];
  const FormJob J = jobs[blockIdx.x];
  double s2 = 0.0, s1 = 0.0;
  for (int64_t e = threadIdx.x; e < (int64_t)J.m * J.n; e += blockDim.x) {
    const int i = (int)(e % J.m), j = (int)(e / J.m);
    const Term& a = J.t[0];
    double v = term_value<T, TD>(a, J.m, J.n, i, j, a.src ? rk1 : rk0, a.src ? dn1 : dn0);
    if (a.alpha != 1.0) v *= a.alpha;
    if (J.t[1].type >= 0) {
      const Term& b = J.t[1];
      v = fma(b.alpha, term_value<T, TD>(b, J.m, J.n, i, j, b.src ? rk1 : rk0, b.src ? dn1 : dn0), v);
    }
    scratch[J.out + e] = v;
    s2 = fma(v, v, s2);
    s1 += fabs(v);
  }
  s2 = block_sum(s2, red);
  s1 = block_sum(s1, red);
  if (threadIdx.x == 0) { fro2[blockIdx.x] = s2; sabs[blockIdx.x] = s1; }
}

// [A1, alpha*A2] and [B1, B2] of two low-rank leaves in FP64 (ld m, n)
struct CatJob {
  int64_t off1, off2;     // leaf offsets in the first / second handle's pool
  int32_t m, n, k1, k2;
  double alpha;
  int64_t outA, outB;     // double offsets in the scratch
};

template <typename T>
__global__ void __launch_bounds__(256) cat_kernel(const CatJob* __restrict__ jobs, const T* rk0, const T* rk1,
                                                  double* __restrict__ scratch) {
  const CatJob J = jobs[blockIdx.x];
  const int eb = (int)sizeof(T);
  const int64_t npad = col_pad_dev(J.n, eb), mpad = col_pad_dev(J.m, eb);
  const int k = J.k1 + J.k2;
  for (int64_t e = threadIdx.x; e < (int64_t)(J.m + J.n) * k; e += blockDim.x) {
    const bool isA = e < (int64_t)J.m * k;
    const int64_t e2 = isA ? e : e - (int64_t)J.m * k;
    const int len = isA ? J.m : J.n;
    const int i = (int)(e2 % len), q = (int)(e2 / len);
    const bool second = q >= J.k1;
    const int qq = second ? q - J.k1 : q;
    const int kk = second ? J.k2 : J.k1;
    const T* B = (second ? rk1 + J.off2 : rk0 + J.off1);
    double v = isA ? from_store<T>(B[npad * kk + i + (int64_t)qq * mpad]) : from_store<T>(B[i + (int64_t)qq * npad]);
    if (isA && second) v *= J.alpha;
    scratch[(isA ? J.outA : J.outB) + e2] = v;
  }
}

// FP64 factors (A m x k ld lda, B n x k ld ldb) or a dense block (C, ld m)
// written into a pool in its storage precision and padded layout
struct PackJob {
  int64_t A, B;           // double offsets in the scratch (A: C for a dense block)
  int32_t m, n, k, lda, ldb, dense;
  int64_t dst;            // element offset of the leaf in the new pool
};

template <typename T, typename TD>
__global__ void __launch_bounds__(256) pack_kernel(const PackJob* __restrict__ jobs, const double* __restrict__ s,
                                                   T* __restrict__ rk, TD* __restrict__ dn) {
  const PackJob J = jobs[blockIdx.x];
  if (J.dense) {
    const int64_t ld = col_pad_dev(J.m, (int)sizeof(TD));
    for (int64_t e = threadIdx.x; e < ld * J.n; e += blockDim.x) {
      const int i = (int)(e % ld), j = (int)(e / ld);
      dn[J.dst + e] = (TD)(i < J.m ? s[J.A + i + (int64_t)j * J.m] : 0.0);
    }
    return;
  }
  const int eb = (int)sizeof(T);
  const int64_t npad = col_pad_dev(J.n, eb), mpad = col_pad_dev(J.m, eb);
  for (int64_t e = threadIdx.x; e < (npad + mpad) * J.k; e += blockDim.x) {
    double v;
    if (e < npad * J.k) {
      const int j = (int)(e % npad), q = (int)(e / npad);
      v = j < J.n ? s[J.B + j + (int64_t)q * J.ldb] : 0.0;
    } else {
      const int64_t e2 = e - npad * J.k;
      const int i = (int)(e2 % mpad), q = (int)(e2 / mpad);
      v = i < J.m ? s[J.A + i + (int64_t)q * J.lda] : 0.0;
    }
    rk[J.dst + e] = to_store<T>(v);
  }
}

struct CopyJob {
  const uint4* src;
  uint4* dst;
  int64_t n16;            // 16-byte words
};

__global__ void __launch_bounds__(256) copy_blocks_kernel(const CopyJob* __restrict__ jobs) {
  const CopyJob J = jobs[blockIdx.x];
  for (int64_t e = threadIdx.x; e < J.n16; e += blockDim.x) J.dst[e] = J.src[e];
}

template <typename V>
int upload(const std::vector<V>& v, V** d, cudaStream_t st) {
  *d = nullptr;
  if (v.empty()) return HM_OK;
  HM_CUDA_TRY(cudaMallocAsync((void**)d, sizeof(V) * v.size(), st));
  HM_CUDA_TRY(cudaMemcpyAsync(*d, v.data(), sizeof(V) * v.size(), cudaMemcpyHostToDevice, st));
  return HM_OK;
}

int64_t rk_elems(const Leaf& L, int eb) {
  return pad_to((col_pad(L.n, eb) + col_pad(L.m, eb)) * L.k, 64 / eb);
}
int64_t dense_elems(const Leaf& L, int deb) { return pad_to(col_pad(L.m, deb) * L.n, 64 / deb); }

// ---------------------------------------------------------------------------
// Compression of FP64 blocks already in the scratch (the "svd" route's
// compress, src/hlu.jl:159-190): fully pivoted ACA down to a residual far
// below eps_trunc * s_1, then the QR+SVD core truncated at eps_trunc.
// Per block: C (m x n) at c, work space U (m x cap), V (n x cap), outA, outB.
// ranks[i] = k, or -1 when the ACA did not converge within RCORE_MAX terms.
// ---------------------------------------------------------------------------
struct Blk {
  int64_t c, u, v, a, b;
  int32_t m, n;
};

int compress_blocks(const std::vector<Blk>& bl, const std::vector<double>& fro2, double* scr, double eps_trunc,
                    std::vector<int32_t>& ranks, cudaStream_t st) {
  const int nb = (int)bl.size();
  ranks.assign(nb, -1);
  if (nb == 0) return HM_OK;
  const int cap = RCORE_MAX;
  int32_t* d_i = nullptr;
  int* d_flags = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void**)&d_i, sizeof(int32_t) * 3 * nb, st));
  HM_CUDA_TRY(cudaMallocAsync((void**)&d_flags, sizeof(int), st));
  HM_CUDA_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int), st));
  std::vector<AcaFpJob> fj(nb);
  for (int i = 0; i < nb; ++i) {
    const double fro = std::sqrt(fro2[i]);
    double tau = 1e-3 * eps_trunc * fro / std::sqrt((double)std::min(bl[i].m, bl[i].n));
    tau = std::max(tau, 64.0 * 2.220446049250313e-16 * fro);
    AcaFpJob J{};
    J.R = scr + bl[i].c; J.U = scr + bl[i].u; J.V = scr + bl[i].v;
    J.m = bl[i].m; J.n = bl[i].n; J.cap = cap; J.min_rank = 1; J.eps = tau;
    J.rank = d_i + i; J.status = d_i + nb + i;
    fj[i] = J;
  }
  AcaFpJob* d_fj = nullptr;
  HM_TRY(upload(fj, &d_fj, st));
  HM_TRY(launch_aca_fp(d_fj, nb, st));
  std::vector<int32_t> rr(2 * nb);
  HM_CUDA_TRY(cudaMemcpyAsync(rr.data(), d_i, sizeof(int32_t) * 2 * nb, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<CoreJob> cj;
  std::vector<int> idx;
  int rmax = 1;
  for (int i = 0; i < nb; ++i) {
    if (rr[nb + i] == 2) return fail(HM_ERR_NONFINITE, "non-finite block during compression");
    if (rr[nb + i] == 1) continue;                       // not low-rank within the core capacity
    CoreJob J{};
    J.A = scr + bl[i].u; J.B = scr + bl[i].v; J.outA = scr + bl[i].a; J.outB = scr + bl[i].b;
    J.m = bl[i].m; J.n = bl[i].n; J.r = rr[i]; J.lda = bl[i].m; J.ldb = bl[i].n; J.ldoa = bl[i].m;
    J.ldob = bl[i].n; J.kcap = cap; J.zero_test = 0; J.rank = d_i + 2 * nb + (int32_t)cj.size();
    cj.push_back(J);
    idx.push_back(i);
    rmax = std::max(rmax, (int)rr[i]);
  }
  if (!cj.empty()) {
    CoreJob* d_cj = nullptr;
    HM_TRY(upload(cj, &d_cj, st));
    HM_TRY(launch_core_recompress(d_cj, (int)cj.size(), rmax, eps_trunc, d_flags, st));
    std::vector<int32_t> kk(cj.size());
    HM_CUDA_TRY(cudaMemcpyAsync(kk.data(), d_i + 2 * nb, sizeof(int32_t) * cj.size(), cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
    HM_CUDA_TRY(cudaFreeAsync(d_cj, st));
    for (size_t q = 0; q < cj.size(); ++q) ranks[idx[q]] = kk[q];
  }
  HM_CUDA_TRY(cudaFreeAsync(d_fj, st));
  HM_CUDA_TRY(cudaFreeAsync(d_i, st));
  HM_CUDA_TRY(cudaFreeAsync(d_flags, st));
  return HM_OK;
}

// A handle with h's trees and the given leaf formats and ranks; pools laid out
// (uninitialised), matvec plans built.
int clone_layout(const hm_handle* h, const std::vector<int8_t>& type, const std::vector<int32_t>& rank,
                 hm_handle** out) {
  hm_handle* c = new hm_handle();
  c->prm = h->prm; c->n = h->n; c->dim = h->dim; c->device = h->device; c->kd = h->kd;
  c->cl_s = h->cl_s; c->cl_e = h->cl_e; c->cl_left = h->cl_left; c->cl_right = h->cl_right;
  c->cl_depth = h->cl_depth; c->nodes = h->nodes; c->leaves = h->leaves; c->depth = h->depth;
  c->storage = h->storage;
  for (size_t i = 0; i < c->leaves.size(); ++i) {
    Leaf& L = c->leaves[i];
    L.type = type[i];
    L.k = type[i] == T_RK ? rank[i] : 0;
    c->nodes[L.node].type = type[i];
  }
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return fail(HM_ERR_CUDA, cudaGetErrorString(e)); }
  int s = HM_OK;
  if (cudaMalloc((void**)&c->d_geom, sizeof(double) * h->n * h->dim) != cudaSuccess)
    s = fail(HM_ERR_OOM, "geometry copy");
  if (s == HM_OK && cudaMemcpy(c->d_geom, h->d_geom, sizeof(double) * h->n * h->dim, cudaMemcpyDeviceToDevice) !=
                        cudaSuccess)
    s = fail(HM_ERR_CUDA, "geometry copy");
  if (s == HM_OK) s = build_matvec_plans(c);
  // the pools are zeroed on c's stream; the callers fill them on another one
  if (s == HM_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) s = fail(HM_ERR_CUDA, "layout");
  if (s != HM_OK) {
    free_handle_data(c);
    cudaStreamDestroy(c->stream);
    delete c;
    return s;
  }
  *out = c;
  return HM_OK;
}

void destroy(hm_handle* c) {
  if (!c) return;
  cudaStreamSynchronize(c->stream);
  free_handle_data(c);
  cudaStreamDestroy(c->stream);
  delete c;
}

// leaves that keep their format and rank: one block copy each
int copy_unchanged(const hm_handle* src, hm_handle* dst, const std::vector<int64_t>& which, cudaStream_t st) {
  if (which.empty()) return HM_OK;
  const int eb = elem_bytes(src->storage), deb = dense_elem_bytes(src->storage);
  std::vector<CopyJob> jobs;
  for (int64_t i : which) {
    const Leaf& a = src->leaves[i];
    const Leaf& b = dst->leaves[i];
    const bool rk = a.type == T_RK;
    const int64_t bytes = rk ? rk_elems(a, eb) * eb : dense_elems(a, deb) * deb;
    if (bytes == 0) continue;
    const char* s = (const char*)(rk ? src->d_rk : src->d_dense) + a.off * (rk ? eb : deb);
    char* d = (char*)(rk ? dst->d_rk : dst->d_dense) + b.off * (rk ? eb : deb);
    jobs.push_back(CopyJob{(const uint4*)s, (uint4*)d, bytes / 16});
  }
  for (size_t b0 = 0; b0 < jobs.size(); b0 += 65535) {
    std::vector<CopyJob> part(jobs.begin() + b0, jobs.begin() + std::min(jobs.size(), b0 + 65535));
    CopyJob* dj = nullptr;
    HM_TRY(upload(part, &dj, st));
    copy_blocks_kernel<<<(unsigned)part.size(), 256, 0, st>>>(dj);
    HM_CUDA_TRY(cudaGetLastError());
    HM_CUDA_TRY(cudaFreeAsync(dj, st));
  }
  return HM_OK;
}

template <typename T, typename TD>
int launch_form(const std::vector<FormJob>& jobs, const hm_handle* h0, const hm_handle* h1, double* scr,
                double* d_f2, double* d_sa, cudaStream_t st) {
  FormJob* dj = nullptr;
  HM_TRY(upload(jobs, &dj, st));
  form_kernel<T, TD><<<(unsigned)jobs.size(), 256, 0, st>>>(
      dj, (const T*)h0->d_rk, (const TD*)h0->d_dense, (const T*)(h1 ? h1->d_rk : nullptr),
      (const TD*)(h1 ? h1->d_dense : nullptr), scr, d_f2, d_sa);
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaFreeAsync(dj, st));
  return HM_OK;
}

int form(const std::vector<FormJob>& jobs, const hm_handle* h0, const hm_handle* h1, double* scr,
         std::vector<double>& fro2, std::vector<double>& sabs, cudaStream_t st) {
  const size_t nb = jobs.size();
  fro2.assign(nb, 0.0);
  sabs.assign(nb, 0.0);
  if (nb == 0) return HM_OK;
  double* d = nullptr;
  HM_CUDA_TRY(cudaMallocAsync((void**)&d, sizeof(double) * 2 * nb, st));
  int s;
  switch (h0->storage) {
    case HM_F64: s = launch_form<double, double>(jobs, h0, h1, scr, d, d + nb, st); break;
    case HM_F32: s = launch_form<float, float>(jobs, h0, h1, scr, d, d + nb, st); break;
    default: s = launch_form<__nv_bfloat16, float>(jobs, h0, h1, scr, d, d + nb, st);
  }
  if (s != HM_OK) return s;
  HM_CUDA_TRY(cudaMemcpyAsync(fro2.data(), d, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaMemcpyAsync(sabs.data(), d + nb, sizeof(double) * nb, cudaMemcpyDeviceToHost, st));
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  HM_CUDA_TRY(cudaFreeAsync(d, st));
  return HM_OK;
}

int pack(const std::vector<PackJob>& jobs, const double* scr, hm_handle* c, cudaStream_t st) {
  if (jobs.empty()) return HM_OK;
  PackJob* dj = nullptr;
  HM_TRY(upload(jobs, &dj, st));
  switch (c->storage) {
    case HM_F64:
      pack_kernel<double, double><<<(unsigned)jobs.size(), 256, 0, st>>>(dj, scr, (double*)c->d_rk,
                                                                          (double*)c->d_dense);
      break;
    case HM_F32:
      pack_kernel<float, float><<<(unsigned)jobs.size(), 256, 0, st>>>(dj, scr, (float*)c->d_rk, (float*)c->d_dense);
      break;
    default:
      pack_kernel<__nv_bfloat16, float><<<(unsigned)jobs.size(), 256, 0, st>>>(dj, scr, (__nv_bfloat16*)c->d_rk,
                                                                                (float*)c->d_dense);
  }
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaFreeAsync(dj, st));
  return HM_OK;
}

template <typename T>
int launch_cat(const std::vector<CatJob>& jobs, const hm_handle* a, const hm_handle* b, double* scr,
               cudaStream_t st) {
  CatJob* dj = nullptr;
  HM_TRY(upload(jobs, &dj, st));
  cat_kernel<T><<<(unsigned)jobs.size(), 256, 0, st>>>(dj, (const T*)a->d_rk, (const T*)b->d_rk, scr);
  HM_CUDA_TRY(cudaGetLastError());
  HM_CUDA_TRY(cudaFreeAsync(dj, st));
  return HM_OK;
}

int cat(const std::vector<CatJob>& jobs, const hm_handle* a, const hm_handle* b, double* scr, cudaStream_t st) {
  if (jobs.empty()) return HM_OK;
  switch (a->storage) {
    case HM_F64: return launch_cat<double>(jobs, a, b, scr, st);
    case HM_F32: return launch_cat<float>(jobs, a, b, scr, st);
    default: return launch_cat<__nv_bfloat16>(jobs, a, b, scr, st);
  }
}

constexpr int64_t kScratch = (int64_t)1 << 27;      // doubles (1 GiB) of FP64 scratch a chunk

// one chunk of the scratch
struct Scratch {
  double* p = nullptr;
  cudaStream_t st = nullptr;
  ~Scratch() { if (p) cudaFreeAsync(p, st); }
};

}  // namespace

// ---------------------------------------------------------------------------
// coarsening (src/utils.jl:29-59): every dense leaf off the diagonal (row and
// column clusters differ) whose truncated SVD rank k = findlast(S/S[1] >
// eps_trunc) is at most MaxRank becomes a rank-k leaf A = U_k, B = V_k S_k.
// A block whose Frobenius norm is zero stays dense (the reference divides by
// S[1] = 0 there and fails).
// ---------------------------------------------------------------------------
int coarsen_handle(const hm_handle* h, hm_handle** out) {
  if (h->factorized || h->lu) return fail(HM_ERR_STATE, "coarsening: the handle is factorised");
  cudaStream_t st = h->stream;
  HM_CUDA_TRY(cudaStreamSynchronize(st));
  const int cap = RCORE_MAX;
  std::vector<int64_t> cand;
  for (int64_t i = 0; i < (int64_t)h->leaves.size(); ++i) {
    const Leaf& L = h->leaves[i];
    if (L.type == T_DENSE && !(L.row0 == L.col0 && L.m == L.n)) cand.push_back(i);
  }
  // chunks of candidates whose blocks and work space fit the scratch
  std::vector<std::pair<size_t, size_t>> chunks;
  {
    size_t b0 = 0;
    int64_t used = 0;
    for (size_t q = 0; q < cand.size(); ++q) {
      const Leaf& L = h->leaves[cand[q]];
      const int64_t need = (int64_t)L.m * L.n + 2 * (int64_t)(L.m + L.n) * cap + 128;
      if (q > b0 && used + need > kScratch) { chunks.push_back({b0, q}); b0 = q; used = 0; }
      used += need;
    }
    if (b0 < cand.size()) chunks.push_back({b0, cand.size()});
  }
  Scratch S;
  S.st = st;
  HM_CUDA_TRY(cudaMallocAsync((void**)&S.p, sizeof(double) * kScratch, st));
  std::vector<int8_t> type(h->leaves.size());
  std::vector<int32_t> rank(h->leaves.size(), 0);
  for (size_t i = 0; i < h->leaves.size(); ++i) { type[i] = h->leaves[i].type; rank[i] = h->leaves[i].k; }

  // per chunk: FP64 blocks, compression; pass 0 decides, pass 1 writes
  auto run_chunk = [&](size_t b0, size_t b1, std::vector<Blk>& bl, std::vector<int32_t>& kk) -> int {
    std::vector<FormJob> fj;
    bl.clear();
    int64_t o = 0;
    for (size_t q = b0; q < b1; ++q) {
      const Leaf& L = h->leaves[cand[q]];
      Blk B{};
      B.m = L.m; B.n = L.n;
      B.c = o; o += pad_to((int64_t)L.m * L.n, 16);
      B.u = o; o += pad_to((int64_t)L.m * cap, 16);
      B.v = o; o += pad_to((int64_t)L.n * cap, 16);
      bl.push_back(B);
      FormJob J{};
      J.t[0] = Term{T_DENSE, 0, 0, 0, L.off, 1.0};
      J.t[1].type = -1;
      J.m = L.m; J.n = L.n; J.out = B.c;
      fj.push_back(J);
    }
    for (auto& B : bl) {
      B.a = o; o += pad_to((int64_t)B.m * cap, 16);
      B.b = o; o += pad_to((int64_t)B.n * cap, 16);
    }
    if (o > kScratch) return fail(HM_ERR_OOM, "coarsening: a block exceeds the scratch");
    std::vector<double> f2, sa;
    HM_TRY(form(fj, h, nullptr, S.p, f2, sa, st));
    HM_TRY(compress_blocks(bl, f2, S.p, h->prm.eps_trunc, kk, st));
    for (size_t q = 0; q < kk.size(); ++q)
      if (!(f2[q] > 0.0)) kk[q] = -1;                  // zero block: stays dense
    return HM_OK;
  };

  std::vector<Blk> bl;
  std::vector<int32_t> kk;
  std::vector<int32_t> decided(cand.size(), -1);
  for (auto& c : chunks) {
    HM_TRY(run_chunk(c.first, c.second, bl, kk));
    for (size_t q = 0; q < kk.size(); ++q)
      if (kk[q] >= 1 && kk[q] <= h->prm.max_rank) decided[c.first + q] = kk[q];
  }
  std::vector<int64_t> keep;
  std::vector<char> conv(h->leaves.size(), 0);
  for (size_t q = 0; q < cand.size(); ++q)
    if (decided[q] > 0) {
      type[cand[q]] = T_RK;
      rank[cand[q]] = decided[q];
      conv[cand[q]] = 1;
    }
  for (int64_t i = 0; i < (int64_t)h->leaves.size(); ++i)
    if (!conv[i]) keep.push_back(i);
  hm_handle* c = nullptr;
  HM_TRY(clone_layout(h, type, rank, &c));
  int s = copy_unchanged(h, c, keep, st);
  for (size_t ci = 0; ci < chunks.size() && s == HM_OK; ++ci) {
    bool any = false;
    for (size_t q = chunks[ci].first; q < chunks[ci].second; ++q) any = any || decided[q] > 0;
    if (!any) continue;
    s = run_chunk(chunks[ci].first, chunks[ci].second, bl, kk);
    std::vector<PackJob> pj;
    for (size_t q = 0; q < kk.size() && s == HM_OK; ++q) {
      const size_t g = chunks[ci].first + q;
      if (decided[g] <= 0) continue;
      if (kk[q] != decided[g]) s = fail(HM_ERR_CUDA, "coarsening: write pass disagrees with the rank pass");
      const Blk& B = bl[q];
      pj.push_back(PackJob{B.a, B.b, B.m, B.n, kk[q], B.m, B.n, 0, c->leaves[cand[g]].off});
    }
    if (s == HM_OK) s = pack(pj, S.p, c, st);
  }
  if (s == HM_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(HM_ERR_CUDA, "coarsening");
  if (s != HM_OK) { destroy(c); return s; }
  *out = c;
  return HM_OK;
}

// ---------------------------------------------------------------------------
// a + scalar * b (hadd / hmat_add!, src/harithm.jl:4-159, 374-420) for two
// H-matrices on the same block partition (same leaves, formats may differ),
// the format of a preserved:
//   a dense:            C_a + scalar * (C_b or A_b B_b')               (axpy / gemm!)
//   a low-rank, b dense: compress(A_a B_a' + scalar * C_b)             (hmat_full_add!)
//   a, b low-rank:      QR of [A_a, scalar A_b] and [B_a, B_b], compress of
//                       R_A R_B' (rkmat_add!); a rank-0 a or b leaves a as is.
// compress applies its zero test (sum|W| < 1e-5 -> one zero column).
// ---------------------------------------------------------------------------
int add_handles(const hm_handle* a, const hm_handle* b, double scalar, hm_handle** out) {
  if (a->factorized || a->lu || b->factorized || b->lu) return fail(HM_ERR_STATE, "hadd: a handle is factorised");
  if (a->n != b->n || a->leaves.size() != b->leaves.size())
    return fail(HM_ERR_UNSUPPORTED, "hadd: the two H-matrices have different block partitions");
  if (a->storage != b->storage) return fail(HM_ERR_UNSUPPORTED, "hadd: the two H-matrices use different storage");
  for (size_t i = 0; i < a->leaves.size(); ++i) {
    const Leaf &x = a->leaves[i], &y = b->leaves[i];
    if (x.row0 != y.row0 || x.col0 != y.col0 || x.m != y.m || x.n != y.n)
      return fail(HM_ERR_UNSUPPORTED, "hadd: the two H-matrices have different block partitions");
  }
  cudaStream_t st = a->stream;
  HM_CUDA_TRY(cudaStreamSynchronize(a->stream));
  HM_CUDA_TRY(cudaStreamSynchronize(b->stream));
  const int cap = RCORE_MAX;
  const size_t nl = a->leaves.size();
  // kinds: 0 dense result, 1 compress(rk + dense), 2 rk + rk core, 3 keep a's block
  std::vector<int> kind(nl);
  for (size_t i = 0; i < nl; ++i) {
    const Leaf &x = a->leaves[i], &y = b->leaves[i];
    if (x.type == T_DENSE) kind[i] = 0;
    else if (y.type == T_DENSE) kind[i] = 1;
    else if (x.k == 0 || y.k == 0) kind[i] = 3;
    else {
      if (x.k + y.k > RCORE_MAX)
        return fail(HM_ERR_UNSUPPORTED, "hadd: summed rank " + std::to_string(x.k + y.k) + " above " +
                                            std::to_string(RCORE_MAX));
      kind[i] = 2;
    }
  }
  // chunks of leaves by scratch need
  auto need = [&](size_t i) -> int64_t {
    const Leaf& x = a->leaves[i];
    const int64_t m = x.m, n = x.n;
    if (kind[i] == 0) return m * n + 16;
    if (kind[i] == 1) return m * n + 2 * (m + n) * cap + 64;
    if (kind[i] == 2) return 2 * (m + n) * (int64_t)(x.k + b->leaves[i].k) + 64;
    return 0;
  };
  std::vector<std::pair<size_t, size_t>> chunks;
  {
    size_t b0 = 0;
    int64_t used = 0;
    for (size_t i = 0; i < nl; ++i) {
      if (i > b0 && used + need(i) > kScratch) { chunks.push_back({b0, i}); b0 = i; used = 0; }
      used += need(i);
    }
    if (b0 < nl) chunks.push_back({b0, nl});
  }
  Scratch S;
  S.st = st;
  HM_CUDA_TRY(cudaMallocAsync((void**)&S.p, sizeof(double) * kScratch, st));
  // per chunk: form / cat / compress; results (rank, FP64 offsets) per leaf
  struct Res { int32_t k; int64_t A, B; int32_t lda, ldb; };
  auto run_chunk = [&](size_t b0, size_t b1, std::vector<Res>& res) -> int {
    res.assign(b1 - b0, Res{0, 0, 0, 0, 0});
    std::vector<FormJob> fj;
    std::vector<size_t> fidx;
    std::vector<Blk> bl;          // kind 1 blocks for compress_blocks
    std::vector<size_t> bidx;
    std::vector<CatJob> cj;
    std::vector<size_t> cidx;
    int64_t o = 0;
    for (size_t i = b0; i < b1; ++i) {
      const Leaf &x = a->leaves[i], &y = b->leaves[i];
      if (kind[i] == 0) {
        FormJob J{};
        J.t[0] = Term{T_DENSE, 0, 0, 0, x.off, 1.0};
        J.t[1] = Term{y.type, y.k, 1, 0, y.off, scalar};
        if (y.type == T_RK && y.k == 0) J.t[1].type = -1;
        J.m = x.m; J.n = x.n; J.out = o;
        res[i - b0] = Res{0, o, 0, x.m, 0};
        o += pad_to((int64_t)x.m * x.n, 16);
        fj.push_back(J);
        fidx.push_back(i);
      } else if (kind[i] == 1) {
        Blk B{};
        B.m = x.m; B.n = x.n;
        B.c = o; o += pad_to((int64_t)x.m * x.n, 16);
        B.u = o; o += pad_to((int64_t)x.m * cap, 16);
        B.v = o; o += pad_to((int64_t)x.n * cap, 16);
        B.a = o; o += pad_to((int64_t)x.m * cap, 16);
        B.b = o; o += pad_to((int64_t)x.n * cap, 16);
        FormJob J{};
        J.t[0] = Term{T_RK, x.k, 0, 0, x.off, 1.0};
        J.t[1] = Term{T_DENSE, 0, 1, 0, y.off, scalar};
        J.m = x.m; J.n = x.n; J.out = B.c;
        fj.push_back(J);
        fidx.push_back(i);
        bl.push_back(B);
        bidx.push_back(i);
      } else if (kind[i] == 2) {
        const int k = x.k + y.k;
        CatJob C{x.off, y.off, x.m, x.n, x.k, y.k, scalar, o, o + pad_to((int64_t)x.m * k, 16)};
        o += pad_to((int64_t)x.m * k, 16) + pad_to((int64_t)x.n * k, 16);
        Blk B{};
        B.m = x.m; B.n = x.n; B.u = C.outA; B.v = C.outB;
        B.a = o; o += pad_to((int64_t)x.m * k, 16);
        B.b = o; o += pad_to((int64_t)x.n * k, 16);
        cj.push_back(C);
        cidx.push_back(i);
        res[i - b0] = Res{k, B.a, B.b, x.m, x.n};
      }
    }
    if (o > kScratch) return fail(HM_ERR_OOM, "hadd: a block exceeds the scratch");
    std::vector<double> f2, sa;
    HM_TRY(form(fj, a, b, S.p, f2, sa, st));
    // compress(rk + dense) with its zero test
    std::vector<double> bf2;
    std::vector<Blk> bl2;
    std::vector<size_t> bidx2;
    for (size_t q = 0, p = 0; q < fidx.size(); ++q) {
      if (kind[fidx[q]] != 1) continue;
      const size_t i = bidx[p];
      const Blk& B = bl[p++];
      if (sa[q] < 1e-5) { res[i - b0] = Res{-2, 0, 0, 0, 0}; continue; }   // one zero column
      bl2.push_back(B);
      bf2.push_back(f2[q]);
      bidx2.push_back(i);
    }
    std::vector<int32_t> kk;
    HM_TRY(compress_blocks(bl2, bf2, S.p, a->prm.eps_trunc, kk, st));
    for (size_t q = 0; q < bl2.size(); ++q) {
      if (kk[q] < 0) return fail(HM_ERR_UNSUPPORTED, "hadd: a block sum is not low-rank within the core capacity");
      res[bidx2[q] - b0] = Res{kk[q], bl2[q].a, bl2[q].b, bl2[q].m, bl2[q].n};
    }
    // rk + rk: concatenated factors, QR + SVD core with compress's zero test
    if (!cj.empty()) {
      HM_TRY(cat(cj, a, b, S.p, st));
      std::vector<CoreJob> core;
      int32_t* d_k = nullptr;
      int* d_flags = nullptr;
      HM_CUDA_TRY(cudaMallocAsync((void**)&d_k, sizeof(int32_t) * cj.size(), st));
      HM_CUDA_TRY(cudaMallocAsync((void**)&d_flags, sizeof(int), st));
      HM_CUDA_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int), st));
      int rmax = 1;
      for (size_t q = 0; q < cj.size(); ++q) {
        const Res& R = res[cidx[q] - b0];
        const int k = R.k;
        CoreJob J{};
        J.A = S.p + cj[q].outA; J.B = S.p + cj[q].outB; J.outA = S.p + R.A; J.outB = S.p + R.B;
        J.m = cj[q].m; J.n = cj[q].n; J.r = k; J.lda = cj[q].m; J.ldb = cj[q].n; J.ldoa = cj[q].m;
        J.ldob = cj[q].n; J.kcap = k; J.zero_test = 1; J.rank = d_k + q;
        core.push_back(J);
        rmax = std::max(rmax, k);
      }
      CoreJob* d_core = nullptr;
      HM_TRY(upload(core, &d_core, st));
      HM_TRY(launch_core_recompress(d_core, (int)core.size(), rmax, a->prm.eps_trunc, d_flags, st));
      std::vector<int32_t> ks(cj.size());
      int flags = 0;
      HM_CUDA_TRY(cudaMemcpyAsync(ks.data(), d_k, sizeof(int32_t) * cj.size(), cudaMemcpyDeviceToHost, st));
      HM_CUDA_TRY(cudaMemcpyAsync(&flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st));
      HM_CUDA_TRY(cudaStreamSynchronize(st));
      HM_CUDA_TRY(cudaFreeAsync(d_core, st));
      HM_CUDA_TRY(cudaFreeAsync(d_k, st));
      HM_CUDA_TRY(cudaFreeAsync(d_flags, st));
      if (flags & 2) return fail(HM_ERR_NONFINITE, "hadd: non-finite recompression");
      for (size_t q = 0; q < cj.size(); ++q) res[cidx[q] - b0].k = ks[q];
    }
    return HM_OK;
  };

  // pass 0: formats and ranks
  std::vector<int8_t> type(nl);
  std::vector<int32_t> rank(nl, 0);
  std::vector<Res> res;
  for (auto& c : chunks) {
    HM_TRY(run_chunk(c.first, c.second, res));
    for (size_t i = c.first; i < c.second; ++i) {
      const Res& R = res[i - c.first];
      type[i] = a->leaves[i].type;
      if (kind[i] == 3) rank[i] = a->leaves[i].k;
      else if (kind[i] == 1 || kind[i] == 2) rank[i] = R.k == -2 ? 1 : R.k;
    }
  }
  hm_handle* c = nullptr;
  HM_TRY(clone_layout(a, type, rank, &c));
  std::vector<int64_t> keep;
  for (size_t i = 0; i < nl; ++i)
    if (kind[i] == 3) keep.push_back((int64_t)i);
  int s = copy_unchanged(a, c, keep, st);
  // pass 1: recompute each chunk and write it
  for (size_t ci = 0; ci < chunks.size() && s == HM_OK; ++ci) {
    const size_t b0 = chunks[ci].first, b1 = chunks[ci].second;
    s = run_chunk(b0, b1, res);
    std::vector<PackJob> pj;
    std::vector<int64_t> zero_rk;
    for (size_t i = b0; i < b1 && s == HM_OK; ++i) {
      const Res& R = res[i - b0];
      const Leaf& L = c->leaves[i];
      if (kind[i] == 0) {
        pj.push_back(PackJob{R.A, 0, L.m, L.n, 0, L.m, 0, 1, L.off});
      } else if (kind[i] == 1 || kind[i] == 2) {
        const int k = R.k == -2 ? 1 : R.k;
        if (k != rank[i]) { s = fail(HM_ERR_CUDA, "hadd: write pass disagrees with the rank pass"); break; }
        if (R.k == -2) zero_rk.push_back((int64_t)i);
        else pj.push_back(PackJob{R.A, R.B, L.m, L.n, k, R.lda, R.ldb, 0, L.off});
      }
    }
    if (s == HM_OK) s = pack(pj, S.p, c, st);
    // compress's zero test: one zero column (the pool block is zeroed)
    for (int64_t i : zero_rk) {
      if (s != HM_OK) break;
      const Leaf& L = c->leaves[i];
      const int eb = elem_bytes(c->storage);
      if (cudaMemsetAsync((char*)c->d_rk + L.off * eb, 0, rk_elems(L, eb) * eb, st) != cudaSuccess)
        s = fail(HM_ERR_CUDA, "hadd: zero block");
    }
  }
  if (s == HM_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(HM_ERR_CUDA, "hadd");
  if (s != HM_OK) { destroy(c); return s; }
  *out = c;
  return HM_OK;
}

}  // namespace hm
