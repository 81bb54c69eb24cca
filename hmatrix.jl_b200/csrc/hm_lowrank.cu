// Batched low-rank kernels for sm_100a: aca2, fully pivoted ACA and the
// QR + one-sided-Jacobi-SVD recompression core.
#include "hm_lowrank.cuh"
#include "hm_core.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace hm {

// ===========================================================================
// aca2 (src/hlu.jl:59-111), one warp per block.  Deterministic pivots: the
// first row, then the arg-max of |a_r| over unused rows (the reference draws
// a random unused row inside its "patience" loop, hlu.jl:72-85).  Up to R
// terms; stops after the first term with |a_r||b_r|/(|a_1||b_1|) <= eps
// (kept) or on an exactly zero pivot (dropped).
// ===========================================================================
struct AcaJob {
  int64_t row0, col0;
  int32_t m, n;
  int64_t off;      // element offset of the leaf in the low-rank pool
};

// Pivots: piv (2 R entries a job: row tau_r, column sigma_r of step r) is
// written when pmode == 1 and read when pmode == 2.  A replay (write pass
// only) takes the recorded rows and columns and runs exactly ranks[job]
// steps with no stopping test, so that the factors of a nearby kernel come
// from the same cross approximation and vary smoothly with its parameter.
template <typename T>
__global__ void __launch_bounds__(128) aca2_kernel(
    KernelDesc kd, const double* __restrict__ geom, int64_t ng, const AcaJob* __restrict__ jobs,
    int64_t njobs, int R, double eps_comp, double* __restrict__ scratch, int mcap, int ncap,
    int32_t* __restrict__ ranks, T* __restrict__ pool, int write, int32_t* __restrict__ piv, int pmode) {
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double* SA = scratch + gwarp * (int64_t)R * (mcap + ncap);   // A: R columns of mcap
  double* SB = SA + (int64_t)R * mcap;                         // B: R columns of ncap

  for (int64_t job = gwarp; job < njobs; job += nwarps) {
    const AcaJob J = jobs[job];
    const int m = J.m, n = J.n;
    int tau = 0;
    uint64_t used = 0;          // bit q of lane l: row l + 32q is used
    double na0 = 1.0, nb0 = 1.0;
    int rank = R;
    int32_t* jp = piv ? piv + job * 2 * (int64_t)R : nullptr;
    const int rmax = pmode == 2 ? min(ranks[job], R) : R;
    if (pmode == 2) rank = rmax;
    for (int r = 0; r < rmax; ++r) {
      if (pmode == 2) tau = jp[2 * r];
      // residual row tau (src/hlu.jl:73-77)
      double best = -1.0, bval = 0.0, nB = 0.0;
      int64_t bidx = INT64_MAX;
      for (int j = lane; j < n; j += 32) {
        double v = kernel_eval(kd, geom, ng, J.row0 + tau, J.col0 + j);
        if (r > 0) {
          double s = 0.0;
          for (int q = 0; q < r; ++q) s = fma(SB[(int64_t)q * ncap + j], SA[(int64_t)q * mcap + tau], s);
          v = v - s;
        }
        SB[(int64_t)r * ncap + j] = v;
        nB = fma(v, v, nB);
        double a = fabs(v);
        if (a > best) { best = a; bidx = j; bval = v; }
      }
      warp_argmax(best, bidx, bval);
      nB = warp_sum(nB);
      __syncwarp();
      const int sigma = pmode == 2 ? jp[2 * r + 1] : (int)bidx;
      const double delta = pmode == 2 ? SB[(int64_t)r * ncap + sigma] : bval;
      if (!(delta != 0.0)) { rank = r; break; }      // delta == 0 (src/hlu.jl:87-89)
      if (pmode == 1 && lane == 0) { jp[2 * r] = tau; jp[2 * r + 1] = sigma; }
      if ((tau & 31) == lane) used |= 1ull << (tau >> 5);
      __syncwarp();
      // residual column sigma, new a_r (src/hlu.jl:93-98)
      double nA = 0.0, best2 = -1.0, v2 = 0.0;
      int64_t idx2 = INT64_MAX;
      for (int i = lane; i < m; i += 32) {
        double v = kernel_eval(kd, geom, ng, J.row0 + i, J.col0 + sigma);
        if (r > 0) {
          double s = 0.0;
          for (int q = 0; q < r; ++q) s = fma(SA[(int64_t)q * mcap + i], SB[(int64_t)q * ncap + sigma], s);
          v = v - s;
        }
        v = v / delta;
        SA[(int64_t)r * mcap + i] = v;
        nA = fma(v, v, nA);
        if (!((used >> (i >> 5)) & 1ull)) {
          double a = fabs(v);
          if (a > best2) { best2 = a; idx2 = i; v2 = v; }
        }
      }
      warp_argmax(best2, idx2, v2);
      nA = warp_sum(nA);
      __syncwarp();
      const double na = sqrt(nA), nb = sqrt(nB);
      if (r == 0) { na0 = na; nb0 = nb; }
      if (pmode == 2) continue;                          // replay: the recorded steps, no stopping test
      if (idx2 == INT64_MAX) { rank = r + 1; break; }   // no unused row left
      tau = (int)idx2;
      const double eps = na * nb / na0 / nb0;           // src/hlu.jl:104
      if (eps <= eps_comp) { rank = r + 1; break; }
    }
    if (!write) {
      if (lane == 0) ranks[job] = rank;
    } else {
      const int eb = (int)sizeof(T);
      const int64_t npad = col_pad_dev(n, eb), mpad = col_pad_dev(m, eb);
      T* Bout = pool + J.off;
      T* Aout = Bout + npad * rank;
      for (int q = 0; q < rank; ++q) {
        for (int j = lane; j < npad; j += 32) Bout[q * npad + j] = to_store<T>(j < n ? SB[(int64_t)q * ncap + j] : 0.0);
        for (int i = lane; i < mpad; i += 32) Aout[q * mpad + i] = to_store<T>(i < m ? SA[(int64_t)q * mcap + i] : 0.0);
      }
      if (lane == 0 && ranks[job] != rank) ranks[job] = -1 - rank;   // must match the rank pass
    }
    __syncwarp();
  }
}

static int aca2_launch(hm_handle* h, const std::vector<int64_t>& rk_leaf, int write,
                       std::vector<int32_t>* ranks_out, int pmode) {
  const int64_t nj = (int64_t)rk_leaf.size();
  if (nj == 0) { if (ranks_out) ranks_out->clear(); return HM_OK; }
  std::vector<AcaJob> jobs(nj);
  int mcap = 1, ncap = 1;
  for (int64_t i = 0; i < nj; ++i) {
    const Leaf& L = h->leaves[rk_leaf[i]];
    jobs[i] = AcaJob{L.row0, L.col0, L.m, L.n, L.off};
    mcap = std::max(mcap, L.m);
    ncap = std::max(ncap, L.n);
  }
  if (mcap > ACA_MAX_EXTENT || ncap > ACA_MAX_EXTENT)
    return fail(HM_ERR_UNSUPPORTED, "aca2 block larger than " + std::to_string(ACA_MAX_EXTENT));
  const int R = std::max(1, h->prm.max_rank);   // aca2(..., MaxRank-1): up to MaxRank terms
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  int64_t per_warp = (int64_t)R * (mcap + ncap) * 8;
  int64_t nwarps = std::min<int64_t>((int64_t)nsm * 32, std::max<int64_t>(4, (int64_t)(1ll << 30) / per_warp));
  nwarps = std::min<int64_t>(nwarps, (nj + 3) / 4 * 4);
  nwarps = std::max<int64_t>(4, nwarps / 4 * 4);
  double* scratch = nullptr;
  AcaJob* dj = nullptr;
  int32_t* dr = nullptr;
  HM_CUDA_TRY(cudaMalloc(&scratch, per_warp * nwarps));
  HM_CUDA_TRY(cudaMalloc(&dj, sizeof(AcaJob) * nj));
  HM_CUDA_TRY(cudaMalloc(&dr, sizeof(int32_t) * nj));
  HM_CUDA_TRY(cudaMemcpyAsync(dj, jobs.data(), sizeof(AcaJob) * nj, cudaMemcpyHostToDevice, h->stream));
  if (write) {
    std::vector<int32_t> kk(nj);
    for (int64_t i = 0; i < nj; ++i) kk[i] = h->leaves[rk_leaf[i]].k;
    HM_CUDA_TRY(cudaMemcpyAsync(dr, kk.data(), sizeof(int32_t) * nj, cudaMemcpyHostToDevice, h->stream));
  }
  unsigned grid = (unsigned)(nwarps / 4);
  switch (write ? h->storage : HM_F64) {
    case HM_F64:
      aca2_kernel<double><<<grid, 128, 0, h->stream>>>(h->kd, h->d_geom, h->n, dj, nj, R, h->prm.eps_comp,
                                                      scratch, mcap, ncap, dr, (double*)h->d_rk, write, h->d_piv, pmode);
      break;
    case HM_F32:
      aca2_kernel<float><<<grid, 128, 0, h->stream>>>(h->kd, h->d_geom, h->n, dj, nj, R, h->prm.eps_comp,
                                                     scratch, mcap, ncap, dr, (float*)h->d_rk, write, h->d_piv, pmode);
      break;
    default:
      aca2_kernel<__nv_bfloat16><<<grid, 128, 0, h->stream>>>(h->kd, h->d_geom, h->n, dj, nj, R,
                                                             h->prm.eps_comp, scratch, mcap, ncap, dr,
                                                             (__nv_bfloat16*)h->d_rk, write, h->d_piv, pmode);
  }
  HM_CUDA_TRY(cudaGetLastError());
  std::vector<int32_t> ranks(nj);
  HM_CUDA_TRY(cudaMemcpyAsync(ranks.data(), dr, sizeof(int32_t) * nj, cudaMemcpyDeviceToHost, h->stream));
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  cudaFree(scratch);
  cudaFree(dj);
  cudaFree(dr);
  if (write) {
    for (int64_t i = 0; i < nj; ++i)
      if (ranks[i] < 0) return fail(HM_ERR_CUDA, "aca2 write pass disagrees with the rank pass");
  } else {
    for (int64_t i = 0; i < nj; ++i)
      if (ranks[i] < 0 || ranks[i] > R) return fail(HM_ERR_CUDA, "aca2 produced an invalid rank");
  }
  if (ranks_out) ranks_out->swap(ranks);
  return HM_OK;
}

int aca2_ranks(hm_handle* h, const std::vector<int64_t>& rk_leaf, std::vector<int32_t>& ranks) {
  return aca2_launch(h, rk_leaf, 0, &ranks, 0);
}
// the write pass records the pivots when the handle keeps them (d_piv set
// before, replay = false) or replays them (replay = true)
int aca2_write(hm_handle* h, const std::vector<int64_t>& rk_leaf, bool replay) {
  return aca2_launch(h, rk_leaf, 1, nullptr, h->d_piv ? (replay ? 2 : 1) : 0);
}

// ===========================================================================
// Fully pivoted ACA (deps/src/ACA_FullyPivoted.cpp:9-151), one CTA per
// block.  R (m x n, ld m) is the residual, updated in place; U/V receive up
// to `cap` columns.  Pivot: largest |R| with the smallest column-major index
// (Eigen's per-column then overall maxCoeff).  Loop condition of line 60:
// (rank < min(m,n) && |R|_F > eps && |R|_F > machine eps) || rank < min_rank.
// status: 0 converged, 1 stopped at `cap` terms, 2 non-finite norm.
// ===========================================================================
__device__ void aca_fp_body(const AcaFpJob& J) {
  __shared__ double red[32];
  __shared__ double s_a[32];
  __shared__ int64_t s_i[32];
  __shared__ double s_v[32];
  __shared__ int64_t s_sel;
  __shared__ double s_max;
  const int m = J.m, n = J.n;
  const int64_t mn = (int64_t)m * n;
  const int maxr = min(m, n);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double meps = 2.220446049250313e-16;
  int rank = 0, status = 0;
  double* ucol = nullptr;
  double* vcol = nullptr;

  double eps = J.eps;
  for (;;) {
    // pass over R: update with the previous term, then arg-max and norm
    double best = -1.0, bval = 0.0, ss = 0.0, sa = 0.0;
    int64_t bidx = INT64_MAX;
    for (int64_t e = threadIdx.x; e < mn; e += blockDim.x) {
      double v = J.R[e];
      if (ucol) {
        const int i = (int)(e % m), j = (int)(e / m);
        v = v - ucol[i] * vcol[j];
        J.R[e] = v;
      }
      ss = fma(v, v, ss);
      sa += fabs(v);
      double a = fabs(v);
      if (a > best) { best = a; bidx = e; bval = v; }
    }
    if (J.rel_mode && !ucol) {
      // compress() semantics (src/hlu.jl:163-167): an absolutely tiny block is
      // rank-1 zeros; otherwise stop far below eps_trunc * s_1
      const double sabs = block_sum(sa, red);
      const double fro = sqrt(block_sum(ss, red));
      if (sabs < 1e-5) { status = 3; break; }
      eps = fmax(1e-3 * J.eps_trunc * fro / sqrt((double)min(m, n)), 64.0 * meps * fro);
    }
    warp_argmax(best, bidx, bval);
    __syncthreads();
    if (lane == 0) { s_a[w] = best; s_i[w] = bidx; s_v[w] = bval; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = s_a[0]; int64_t bi = s_i[0]; double bv = s_v[0];
      for (int q = 1; q < nw; ++q)
        if (s_a[q] > b || (s_a[q] == b && s_i[q] < bi)) { b = s_a[q]; bi = s_i[q]; bv = s_v[q]; }
      s_sel = bi; s_max = bv;
    }
    const double Rnorm = sqrt(block_sum(ss, red));   // contains a __syncthreads
    const int64_t sel = s_sel;
    const double Max = s_max;
    if (isnan(Rnorm)) { status = 2; break; }
    if (!((rank < maxr && Rnorm > eps && Rnorm > meps) || rank < J.min_rank)) break;
    if (rank >= J.cap) { status = 1; break; }
    const int sel_row = (int)(sel % m), sel_col = (int)(sel / m);
    ucol = J.U + (int64_t)rank * m;
    vcol = J.V + (int64_t)rank * n;
    if (fabs(Max) > meps && !isnan(Max)) {
      const double gamma = 1.0 / Max;
      for (int i = threadIdx.x; i < m; i += blockDim.x) ucol[i] = gamma * J.R[i + (int64_t)sel_col * m];
      for (int j = threadIdx.x; j < n; j += blockDim.x) vcol[j] = J.R[sel_row + (int64_t)j * m];
    } else {
      for (int i = threadIdx.x; i < m; i += blockDim.x) ucol[i] = (i == rank) ? 1.0 : 0.0;
      for (int j = threadIdx.x; j < n; j += blockDim.x) vcol[j] = 0.0;
    }
    __syncthreads();
    ++rank;
  }
  if (threadIdx.x == 0) { *J.rank = rank; *J.status = status; }
}

__global__ void __launch_bounds__(512) aca_fp_kernel(const AcaFpJob* __restrict__ jobs) {
  aca_fp_body(jobs[blockIdx.x]);
}

__global__ void __launch_bounds__(512) aca_fp_one_kernel(AcaFpJob J) { aca_fp_body(J); }

int launch_aca_fp(const AcaFpJob* d_jobs, int njobs, cudaStream_t st) {
  if (njobs <= 0) return HM_OK;
  aca_fp_kernel<<<njobs, 512, 0, st>>>(d_jobs);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

int launch_aca_fp_one(const AcaFpJob& J, cudaStream_t st) {
  aca_fp_one_kernel<<<1, 512, 0, st>>>(J);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

// JAC8: the H-LU's recompressions (8 lanes per Jacobi pair, parallel ordering);
// construction and H + H keep the block-wide rounds
template <bool JAC8>
__global__ void __launch_bounds__(256) core_recompress_kernel(const CoreJob* __restrict__ jobs, int rmax,
                                                              double eps_trunc, int* __restrict__ flags) {
  const CoreJob& J = jobs[blockIdx.x];
  core_body_t<double, JAC8>(J, J.A, J.B, rmax, eps_trunc, flags);
}

__global__ void __launch_bounds__(256) core_recompress_one_kernel(CoreJob J, int rmax, double eps_trunc,
                                                                  int* __restrict__ flags) {
  core_body(J, rmax, eps_trunc, flags);
}

int launch_core_one(const CoreJob& J, double eps_trunc, int* d_flags, cudaStream_t st) {
  const size_t smem = (size_t)3 * RCORE_MAX * RCORE_MAX * sizeof(double);
  HM_CUDA_TRY(smem_attr((const void*)core_recompress_one_kernel, (int)smem));
  core_recompress_one_kernel<<<1, 256, smem, st>>>(J, RCORE_MAX, eps_trunc, d_flags);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

int launch_core_recompress(const CoreJob* d_jobs, int njobs, int rmax, double eps_trunc, int* d_flags,
                           cudaStream_t st, bool jac8) {
  if (njobs == 0) return HM_OK;
  if (rmax > RCORE_MAX) return fail(HM_ERR_UNSUPPORTED, "recompression core above " + std::to_string(RCORE_MAX));
  rmax = std::max(rmax, 1);
  size_t smem = (size_t)3 * rmax * rmax * sizeof(double);
  const void* kfn = jac8 ? (const void*)core_recompress_kernel<true> : (const void*)core_recompress_kernel<false>;
  HM_CUDA_TRY(smem_attr(kfn, (int)((size_t)3 * RCORE_MAX * RCORE_MAX * sizeof(double))));
  // small cores: 2 warps per job, so that many jobs share an SM
  const int nt = rmax <= 32 ? 64 : 256;
  if (jac8) core_recompress_kernel<true><<<njobs, nt, smem, st>>>(d_jobs, rmax, eps_trunc, d_flags);
  else core_recompress_kernel<false><<<njobs, nt, smem, st>>>(d_jobs, rmax, eps_trunc, d_flags);
  HM_CUDA_TRY(cudaGetLastError());
  return HM_OK;
}

// ===========================================================================
// "svd" route candidates (src/cluster.jl:99-107): dense block, compress,
// low-rank iff rank <= MaxRank.  compress (src/hlu.jl:159-190) is realised
// as a fully pivoted ACA down to a residual far below eps_trunc*s_1 followed
// by the exact QR+SVD of its core, which yields the truncated SVD of the
// block up to that residual.
// ===========================================================================
__global__ void dense_block_kernel(KernelDesc kd, const double* __restrict__ geom, int64_t ng,
                                   const int64_t* __restrict__ r0, const int64_t* __restrict__ c0,
                                   const int32_t* __restrict__ mm, const int32_t* __restrict__ nn,
                                   const int64_t* __restrict__ off, double* __restrict__ out,
                                   double* __restrict__ fro2, double* __restrict__ sabs) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  const int m = mm[b], n = nn[b];
  double* C = out + off[b];
  double s2 = 0.0, s1 = 0.0;
  for (int64_t e = threadIdx.x; e < (int64_t)m * n; e += blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    double v = kernel_eval(kd, geom, ng, r0[b] + i, c0[b] + j);
    C[e] = v;
    s2 = fma(v, v, s2);
    s1 += fabs(v);
  }
  s2 = block_sum(s2, red);
  s1 = block_sum(s1, red);
  if (threadIdx.x == 0) { fro2[b] = s2; sabs[b] = s1; }
}

int svd_compress_candidates(hm_handle* h, const std::vector<int64_t>& r0, const std::vector<int64_t>& c0,
                            const std::vector<int32_t>& mm, const std::vector<int32_t>& nn,
                            std::vector<int32_t>& ranks, SvdCandidateStore& store,
                            const std::vector<int32_t>& nodes) {
  const int64_t nc = (int64_t)r0.size();
  ranks.assign(nc, 0);
  const int cap = RCORE_MAX;
  const double eps_trunc = h->prm.eps_trunc;
  // chunk the candidates so that the dense blocks stay below ~2 GB
  int64_t b0 = 0;
  while (b0 < nc) {
    int64_t b1 = b0, elems = 0;
    while (b1 < nc && (b1 == b0 || elems + (int64_t)mm[b1] * nn[b1] < (1ll << 28))) {
      elems += (int64_t)mm[b1] * nn[b1] + (int64_t)(mm[b1] + nn[b1]) * cap * 2;
      ++b1;
    }
    const int64_t nb = b1 - b0;
    std::vector<int64_t> offC(nb), offU(nb), offV(nb), offA(nb), offB(nb);
    int64_t tot = 0;
    for (int64_t i = 0; i < nb; ++i) {
      const int64_t m = mm[b0 + i], n = nn[b0 + i];
      offC[i] = tot; tot += pad_to(m * n, 32);
      offU[i] = tot; tot += pad_to(m * cap, 32);
      offV[i] = tot; tot += pad_to(n * cap, 32);
      offA[i] = tot; tot += pad_to(m * cap, 32);
      offB[i] = tot; tot += pad_to(n * cap, 32);
    }
    double* buf = nullptr;
    HM_CUDA_TRY(cudaMalloc(&buf, sizeof(double) * tot));
    int64_t *d_r0 = nullptr, *d_c0 = nullptr, *d_off = nullptr;
    int32_t *d_m = nullptr, *d_n = nullptr, *d_rank = nullptr, *d_stat = nullptr;
    double *d_f2 = nullptr, *d_sa = nullptr;
    int* d_flags = nullptr;
    HM_CUDA_TRY(cudaMalloc(&d_r0, 8 * nb)); HM_CUDA_TRY(cudaMalloc(&d_c0, 8 * nb));
    HM_CUDA_TRY(cudaMalloc(&d_off, 8 * nb)); HM_CUDA_TRY(cudaMalloc(&d_m, 4 * nb));
    HM_CUDA_TRY(cudaMalloc(&d_n, 4 * nb)); HM_CUDA_TRY(cudaMalloc(&d_rank, 4 * nb * 2));
    HM_CUDA_TRY(cudaMalloc(&d_stat, 4 * nb)); HM_CUDA_TRY(cudaMalloc(&d_f2, 8 * nb));
    HM_CUDA_TRY(cudaMalloc(&d_sa, 8 * nb)); HM_CUDA_TRY(cudaMalloc(&d_flags, 4));
    HM_CUDA_TRY(cudaMemsetAsync(d_flags, 0, 4, h->stream));
    cudaStream_t st = h->stream;
    HM_CUDA_TRY(cudaMemcpyAsync(d_r0, r0.data() + b0, 8 * nb, cudaMemcpyHostToDevice, st));
    HM_CUDA_TRY(cudaMemcpyAsync(d_c0, c0.data() + b0, 8 * nb, cudaMemcpyHostToDevice, st));
    HM_CUDA_TRY(cudaMemcpyAsync(d_off, offC.data(), 8 * nb, cudaMemcpyHostToDevice, st));
    HM_CUDA_TRY(cudaMemcpyAsync(d_m, mm.data() + b0, 4 * nb, cudaMemcpyHostToDevice, st));
    HM_CUDA_TRY(cudaMemcpyAsync(d_n, nn.data() + b0, 4 * nb, cudaMemcpyHostToDevice, st));
    dense_block_kernel<<<(unsigned)nb, 256, 0, st>>>(h->kd, h->d_geom, h->n, d_r0, d_c0, d_m, d_n, d_off,
                                                     buf, d_f2, d_sa);
    HM_CUDA_TRY(cudaGetLastError());
    std::vector<double> fro2(nb), sabs(nb);
    HM_CUDA_TRY(cudaMemcpyAsync(fro2.data(), d_f2, 8 * nb, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaMemcpyAsync(sabs.data(), d_sa, 8 * nb, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
    // fully pivoted ACA to tau = 1e-3 * eps_trunc * |C|_F / sqrt(min(m,n)) (<= 1e-3 eps_trunc s_1)
    std::vector<AcaFpJob> fj(nb);
    for (int64_t i = 0; i < nb; ++i) {
      const int m = mm[b0 + i], n = nn[b0 + i];
      const double fro = sqrt(fro2[i]);
      double tau = 1e-3 * eps_trunc * fro / sqrt((double)std::min(m, n));
      tau = std::max(tau, 64.0 * 2.220446049250313e-16 * fro);
      AcaFpJob J{};
      J.R = buf + offC[i]; J.U = buf + offU[i]; J.V = buf + offV[i]; J.m = m; J.n = n; J.cap = cap;
      J.min_rank = 1; J.eps = tau; J.rank = d_rank + i; J.status = d_stat + i;
      fj[i] = J;
    }
    AcaFpJob* d_fj = nullptr;
    HM_CUDA_TRY(cudaMalloc(&d_fj, sizeof(AcaFpJob) * nb));
    HM_CUDA_TRY(cudaMemcpyAsync(d_fj, fj.data(), sizeof(AcaFpJob) * nb, cudaMemcpyHostToDevice, st));
    aca_fp_kernel<<<(unsigned)nb, 512, 0, st>>>(d_fj);
    HM_CUDA_TRY(cudaGetLastError());
    std::vector<int32_t> rr(nb), stt(nb);
    HM_CUDA_TRY(cudaMemcpyAsync(rr.data(), d_rank, 4 * nb, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaMemcpyAsync(stt.data(), d_stat, 4 * nb, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
    // QR + SVD of the ACA cores for the blocks that converged
    std::vector<CoreJob> cj;
    std::vector<int64_t> cj_idx;
    int rmax = 1;
    for (int64_t i = 0; i < nb; ++i) {
      if (stt[i] == 2) return fail(HM_ERR_NONFINITE, "non-finite kernel block during compression");
      const int m = mm[b0 + i], n = nn[b0 + i];
      if (sabs[i] < 1e-5) { ranks[b0 + i] = 1; continue; }       // compress() zero test
      if (stt[i] == 1) { ranks[b0 + i] = 1 << 30; continue; }    // not low-rank within the core cap
      CoreJob J{};
      J.A = buf + offU[i]; J.B = buf + offV[i]; J.outA = buf + offA[i]; J.outB = buf + offB[i];
      J.m = m; J.n = n; J.r = rr[i]; J.lda = m; J.ldb = n; J.ldoa = m; J.ldob = n; J.kcap = cap;
      J.zero_test = 0; J.rank = d_rank + nb + (int32_t)cj.size();
      cj.push_back(J);
      cj_idx.push_back(i);
      rmax = std::max(rmax, (int)rr[i]);
    }
    CoreJob* d_cj = nullptr;
    std::vector<int32_t> kk(cj.size());
    if (!cj.empty()) {
      HM_CUDA_TRY(cudaMalloc(&d_cj, sizeof(CoreJob) * cj.size()));
      HM_CUDA_TRY(cudaMemcpyAsync(d_cj, cj.data(), sizeof(CoreJob) * cj.size(), cudaMemcpyHostToDevice, st));
      HM_TRY(launch_core_recompress(d_cj, (int)cj.size(), rmax, eps_trunc, d_flags, st));
      HM_CUDA_TRY(cudaMemcpyAsync(kk.data(), d_rank + nb, 4 * cj.size(), cudaMemcpyDeviceToHost, st));
      HM_CUDA_TRY(cudaStreamSynchronize(st));
    }
    for (size_t q = 0; q < cj.size(); ++q) ranks[b0 + cj_idx[q]] = kk[q];
    // keep the factors of the blocks that become low-rank
    for (int64_t i = 0; i < nb; ++i) {
      const int k = ranks[b0 + i];
      if (k > h->prm.max_rank) continue;
      const int m = mm[b0 + i], n = nn[b0 + i];
      SvdCandidateStore::F f;
      f.m = m; f.n = n; f.k = k;
      f.A.assign((size_t)m * k, 0.0);
      f.B.assign((size_t)n * k, 0.0);
      if (sabs[i] >= 1e-5 && k > 0) {
        HM_CUDA_TRY(cudaMemcpy(f.A.data(), buf + offA[i], 8 * (size_t)m * k, cudaMemcpyDeviceToHost));
        HM_CUDA_TRY(cudaMemcpy(f.B.data(), buf + offB[i], 8 * (size_t)n * k, cudaMemcpyDeviceToHost));
      }
      store.by_node[nodes[b0 + i]] = std::move(f);
    }
    cudaFree(buf); cudaFree(d_r0); cudaFree(d_c0); cudaFree(d_off); cudaFree(d_m); cudaFree(d_n);
    cudaFree(d_rank); cudaFree(d_stat); cudaFree(d_f2); cudaFree(d_sa); cudaFree(d_flags);
    cudaFree(d_fj); if (d_cj) cudaFree(d_cj);
    b0 = b1;
  }
  return HM_OK;
}

// pack FP64 host factors into the pool (storage precision, padded layout)
__global__ void pack_rk_kernel(const double* __restrict__ A, const double* __restrict__ B, int m, int n, int k,
                               int64_t npad, int64_t mpad, int storage, void* pool, int64_t off) {
  const int64_t tot = (npad + mpad) * k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    double v;
    if (e < npad * k) {
      const int64_t j = e % npad, q = e / npad;
      v = j < n ? B[j + q * n] : 0.0;
    } else {
      const int64_t e2 = e - npad * k;
      const int64_t i = e2 % mpad, q = e2 / mpad;
      v = i < m ? A[i + q * m] : 0.0;
    }
    if (storage == HM_F64) ((double*)pool)[off + e] = v;
    else if (storage == HM_F32) ((float*)pool)[off + e] = (float)v;
    else ((__nv_bfloat16*)pool)[off + e] = __double2bfloat16(v);
  }
}

int SvdCandidateStore::write_pool(hm_handle* h, const std::vector<int64_t>& rk_leaf) const {
  const int eb = elem_bytes(h->storage);
  double* dA = nullptr;
  struct Guard {
    double** p;
    ~Guard() { if (*p) cudaFree(*p); }
  } guard{&dA};
  size_t cap = 0;
  for (int64_t li : rk_leaf) {
    const Leaf& L = h->leaves[li];
    auto it = by_node.find(L.node);
    if (it == by_node.end()) return fail(HM_ERR_CUDA, "missing factors of an svd-route leaf");
    const F& f = it->second;
    if (f.k == 0) continue;
    size_t need = (f.A.size() + f.B.size()) * sizeof(double);
    if (need > cap) {
      if (dA) cudaFree(dA);
      dA = nullptr;
      HM_CUDA_TRY(cudaMalloc(&dA, need));
      cap = need;
    }
    HM_CUDA_TRY(cudaMemcpyAsync(dA, f.A.data(), f.A.size() * 8, cudaMemcpyHostToDevice, h->stream));
    HM_CUDA_TRY(cudaMemcpyAsync(dA + f.A.size(), f.B.data(), f.B.size() * 8, cudaMemcpyHostToDevice, h->stream));
    pack_rk_kernel<<<64, 256, 0, h->stream>>>(dA, dA + f.A.size(), f.m, f.n, f.k, col_pad(f.n, eb),
                                              col_pad(f.m, eb), h->storage, h->d_rk, L.off);
    HM_CUDA_TRY(cudaGetLastError());
    HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  }
  return HM_OK;
}

// ===========================================================================
// aca_wrapper drop-in: fully pivoted ACA of a host matrix (rank 0 branch).
// ===========================================================================
int aca_fp_host(const double* A, double* U, double* V, int m, int n, double eps, int rank, int* out_rank) {
  if (m <= 0 || n <= 0) return fail(HM_ERR_ARG, "aca_wrapper: empty matrix");
  const int cap = std::min(m, n);
  double *dR = nullptr, *dU = nullptr, *dV = nullptr;
  int32_t* dk = nullptr;
  AcaFpJob* dj = nullptr;
  // every return below, early error returns included, frees what was allocated
  struct Guard {
    void** p[5];
    ~Guard() { for (void** q : p) if (*q) cudaFree(*q); }
  } guard{{(void**)&dR, (void**)&dU, (void**)&dV, (void**)&dk, (void**)&dj}};
  HM_CUDA_TRY(cudaMalloc(&dR, 8ull * m * n));
  HM_CUDA_TRY(cudaMalloc(&dU, 8ull * m * cap));
  HM_CUDA_TRY(cudaMalloc(&dV, 8ull * n * cap));
  HM_CUDA_TRY(cudaMalloc(&dk, 8));
  HM_CUDA_TRY(cudaMalloc(&dj, sizeof(AcaFpJob)));
  HM_CUDA_TRY(cudaMemcpy(dR, A, 8ull * m * n, cudaMemcpyHostToDevice));
  AcaFpJob j{};
  j.R = dR; j.U = dU; j.V = dV; j.m = m; j.n = n; j.cap = cap; j.min_rank = 1; j.eps = eps;
  j.rank = dk; j.status = dk + 1;
  HM_CUDA_TRY(cudaMemcpy(dj, &j, sizeof(j), cudaMemcpyHostToDevice));
  aca_fp_kernel<<<1, 512>>>(dj);
  HM_CUDA_TRY(cudaGetLastError());
  int32_t res[2];
  HM_CUDA_TRY(cudaMemcpy(res, dk, 8, cudaMemcpyDeviceToHost));
  int r = res[0];
  const int M = std::min(r, rank + 1);
  if (res[1] == 2) {
    // NaN residual: identity fallback of ACA_FullyPivoted.cpp:122-147
    if (m < n) {
      r = m;
      std::vector<double> hA(A, A + (size_t)m * n);
      const int Mf = std::min(r, rank + 1);
      for (int c = 0; c < Mf; ++c)
        for (int i = 0; i < m; ++i) U[i + (size_t)c * m] = (i == c) ? 1.0 : 0.0;
      for (int c = 0; c < Mf; ++c)
        for (int jx = 0; jx < n; ++jx) V[jx + (size_t)c * n] = hA[c + (size_t)jx * m];
    } else {
      r = n;
      const int Mf = std::min(r, rank + 1);
      std::memcpy(U, A, sizeof(double) * (size_t)m * Mf);
      for (int c = 0; c < Mf; ++c)
        for (int jx = 0; jx < n; ++jx) V[jx + (size_t)c * n] = (jx == c) ? 1.0 : 0.0;
    }
  } else if (M > 0) {
    HM_CUDA_TRY(cudaMemcpy(U, dU, 8ull * m * M, cudaMemcpyDeviceToHost));
    HM_CUDA_TRY(cudaMemcpy(V, dV, 8ull * n * M, cudaMemcpyDeviceToHost));
  }
  *out_rank = r;
  return HM_OK;
}

}  // namespace hm
