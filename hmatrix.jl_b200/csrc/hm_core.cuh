// Recompression core shared by the construction and the H-LU kernels (one
// CTA per job): CGS2 QR of the two tall factors, SVD of the small core by
// one-sided Jacobi, truncation, and the products that form the new factors.
// The tall factors may live in global or shared memory.
#pragma once
#include "hm_lowrank.cuh"

namespace hm {

// ===========================================================================
// Recompression core (K3): CGS2 QR of A and B in place, W = R_A R_B^T, one
// sided Jacobi SVD of W, truncation k = #{s_i/s_1 > eps_trunc}, and
// A' = Q_A U_k, B' = Q_B V_k S_k.  One CTA per job; smem 3*rmax^2 doubles.
// ===========================================================================
// Columns [0, j0) are already orthonormal and their block of Rm is set by the
// caller (cgs2_qr zeroes the rest of Rm first).
template <typename TS>
static __device__ void cgs2_qr(TS* X, int len, int ld, int r, TS* Rm /* r x r, col-major */,
                        TS* proj /* r */, double* red, int j0 = 0) {
  for (int e = threadIdx.x; e < r * r; e += blockDim.x)
    if (!(e % r < j0 && e / r < j0)) Rm[e] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = j0; j < r; ++j) {
    TS* xj = X + (int64_t)j * ld;
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = w; i < j; i += nw) {
        const TS* qi = X + (int64_t)i * ld;
        TS s = 0;
        for (int t = lane; t < len; t += 32) s = fma(qi[t], xj[t], s);
        s = warp_sum(s);
        if (lane == 0) proj[i] = s;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < len; t += blockDim.x) {
        TS s = 0;
        for (int i = 0; i < j; ++i) s = fma(X[t + (int64_t)i * ld], proj[i], s);
        xj[t] -= s;
      }
      if (threadIdx.x < j) Rm[threadIdx.x + j * r] += proj[threadIdx.x];
      // after the second pass no barrier: the norm reads only this thread's
      // rows, and proj is rewritten only after the norm's barrier
      if (pass == 0) __syncthreads();
    }
    TS ss = 0;
    for (int t = threadIdx.x; t < len; t += blockDim.x) ss = fma(xj[t], xj[t], ss);
    // block_sum without its leading barrier: red was last read before the
    // previous column's closing barrier
    double sd = warp_sum((double)ss);
    if (lane == 0) red[w] = sd;
    __syncthreads();
    sd = 0.0;
    for (int q = 0; q < ((blockDim.x + 31) >> 5); ++q) sd += red[q];
    const TS nrm = sqrt((TS)sd);
    const TS inv = nrm > (TS)0 ? (TS)1 / nrm : (TS)0;
    for (int t = threadIdx.x; t < len; t += blockDim.x) xj[t] *= inv;
    if (threadIdx.x == 0) Rm[j + j * r] = nrm;
    __syncthreads();
  }
}

static __device__ void zero_cols(double* X, int len, int64_t ld, int c0, int c1) {
  for (int c = c0; c < c1; ++c)
    for (int i = threadIdx.x; i < len; i += blockDim.x) X[i + (int64_t)c * ld] = 0.0;
}

// TS: the working precision (double; float for a loose truncation, where
// FP32 Gram-Schmidt and Jacobi keep far more accuracy than the truncation
// discards).  A, B: the tall factors (in TS), J's other fields as for
// core_body; the new factors are written in FP64.
// JAC8 (the H-LU tile kernel): Jacobi rounds with 8 lanes per column pair, so
// a round's pairs run at once instead of one after another per warp, and the
// singular values ordered by a parallel rank count instead of one thread's
// selection sort.  The rotations and the order are the same; only the order
// of the sums in the dot products differs.
template <typename TS, bool JAC8 = false>
static __device__ void core_body_t(const CoreJob& J, TS* __restrict__ JA, TS* __restrict__ JB, int rmax,
                                   double eps_trunc, int* __restrict__ flags) {
  extern __shared__ double sm_raw[];
  TS* sm = reinterpret_cast<TS*>(sm_raw);
  __shared__ double red[32];
  __shared__ TS proj[RCORE_MAX];
  __shared__ TS sig[RCORE_MAX];
  __shared__ int ord[RCORE_MAX];
  __shared__ int s_rot;
  __shared__ int s_k;
  int r = J.r_dev ? *J.r_dev : J.r;
  TS* b0 = sm;                           // R_A, later V (Jacobi right vectors)
  TS* b1 = sm + rmax * rmax;             // R_B, later U-coefficients
  TS* b2 = sm + 2 * rmax * rmax;         // W, later V-coefficients
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int pre = J.pre_status ? *J.pre_status : 0;
  if (pre != 0 || r > rmax) {
    // pre == 3: compress() of an absolutely tiny block -> rank-1 zeros;
    // otherwise the input could not be reduced (not converged / too large)
    if (threadIdx.x == 0 && pre != 3) atomicOr(flags, pre == 2 ? 2 : 1);
    zero_cols(J.outA, J.m, J.ldoa, 0, J.kcap);
    zero_cols(J.outB, J.n, J.ldob, 0, J.kcap);
    if (threadIdx.x == 0) *J.rank = (pre == 3) ? 1 : 0;
    return;
  }
  // zero_fill writes zeros up to zlim only: beyond it the columns are zero
  const int zlim = J.known_zero ? min(max(J.zero_from, 0), J.kcap) : J.kcap;
  if (r == 0) {
    if (J.zero_fill) {
      zero_cols(J.outA, J.m, J.ldoa, 0, zlim);
      zero_cols(J.outB, J.n, J.ldob, 0, zlim);
    }
    if (threadIdx.x == 0) *J.rank = 0;
    return;
  }
  const int ok = min(J.ortho_k, r);
  if (ok > 0) {
    // A's leading columns are orthonormal: R_A = I there.  B's are orthogonal:
    // normalise them, R_B = diag(norms).
    for (int e = threadIdx.x; e < ok * ok; e += blockDim.x) {
      const int i = e % ok, j = e / ok;
      b0[i + j * r] = (i == j) ? 1.0 : 0.0;
      b1[i + j * r] = 0.0;
    }
    for (int j = w; j < ok; j += nw) {
      TS s = 0;
      for (int t = lane; t < J.n; t += 32) s = fma(JB[t + (int64_t)j * J.ldb], JB[t + (int64_t)j * J.ldb], s);
      s = warp_sum(s);
      if (lane == 0) proj[j] = sqrt(s);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < J.n * ok; e += blockDim.x) {
      const int t = e % J.n, j = e / J.n;
      const TS nj = proj[j];
      JB[t + (int64_t)j * J.ldb] = nj > (TS)0 ? JB[t + (int64_t)j * J.ldb] / nj : (TS)0;
    }
    if (threadIdx.x < ok) b1[threadIdx.x + threadIdx.x * r] = proj[threadIdx.x];
    __syncthreads();
  }
  cgs2_qr(JA, J.m, J.lda, r, b0, proj, red, ok);
  cgs2_qr(JB, J.n, J.ldb, r, b1, proj, red, ok);
  // W = R_A R_B^T  (r x r, column-major, ld r)
  double sabs = 0.0;
  for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
    const int i = e % r, j = e / r;
    TS s = 0;
    for (int q = max(i, j); q < r; ++q) s = fma(b0[i + q * r], b1[j + q * r], s);
    b2[e] = s;
    sabs += fabs((double)s);
  }
  sabs = block_sum(sabs, red);
  bool nonfinite = !isfinite(sabs);
  if (J.zero_test && sabs < 1e-5) {
    // compress(): an (absolutely) tiny core becomes rank-1 zeros (src/hlu.jl:163-167)
    const int kz = J.zero_fill ? max(zlim, 1) : 1;
    zero_cols(J.outA, J.m, J.ldoa, 0, kz);
    zero_cols(J.outB, J.n, J.ldob, 0, kz);
    if (threadIdx.x == 0) *J.rank = 1;
    return;
  }
  // V = I
  for (int e = threadIdx.x; e < r * r; e += blockDim.x) b0[e] = (e % r == e / r) ? (TS)1 : (TS)0;
  __syncthreads();
  // one-sided Jacobi on the columns of W, round-robin pairing.  A pair is
  // rotated while its cosine exceeds thr; the truncation only needs the
  // singular values far below eps_trunc, so thr follows it (at least 1e-15)
  const int rr = (r + 1) & ~1;
  const TS thr = (TS)fmax(sizeof(TS) == 8 ? 1e-15 : 1e-7, 1e-3 * eps_trunc);
  for (int sweep = 0; sweep < 60; ++sweep) {
    if (threadIdx.x == 0) s_rot = 0;
    __syncthreads();
    for (int round = 0; round < rr - 1; ++round) {
      // tournament pairing: position 0 fixed, others rotate
      auto posv = [&](int q) { return q == 0 ? 0 : 1 + (q - 1 + round) % (rr - 1); };
      if constexpr (JAC8) {
        // 8 lanes per pair (4 pairs a warp at once, rows strided by 8): a
        // round's pairs run concurrently instead of one after another per warp
        const int sg = lane >> 3, sl = lane & 7;
        for (int base = w * 4; base < rr / 2; base += nw * 4) {
          const int pidx = base + sg;
          int p = 0, q = 0;
          bool act = pidx < rr / 2;
          if (act) {
            p = posv(pidx); q = posv(rr - 1 - pidx);
            if (p > q) { int t = p; p = q; q = t; }
            act = q < r;
          }
          TS* wp = b2 + p * r;
          TS* wq = b2 + q * r;
          TS al = 0, be = 0, ga = 0;
          if (act)
            for (int t = sl; t < r; t += 8) {
              al = fma(wp[t], wp[t], al);
              be = fma(wq[t], wq[t], be);
              ga = fma(wp[t], wq[t], ga);
            }
#pragma unroll
          for (int o = 4; o > 0; o >>= 1) {
            al += __shfl_xor_sync(0xffffffffu, al, o);
            be += __shfl_xor_sync(0xffffffffu, be, o);
            ga += __shfl_xor_sync(0xffffffffu, ga, o);
          }
          if (act && ga != (TS)0 && fabs(ga) > thr * sqrt(al * be)) {
            const TS zeta = (be - al) / ((TS)2 * ga);
            const TS t = (zeta >= (TS)0 ? (TS)1 : (TS)-1) / (fabs(zeta) + sqrt((TS)1 + zeta * zeta));
            const TS c = (TS)1 / sqrt((TS)1 + t * t), s = c * t;
            TS* vp = b0 + p * r;
            TS* vq = b0 + q * r;
            for (int t2 = sl; t2 < r; t2 += 8) {
              const TS x = wp[t2], y = wq[t2];
              wp[t2] = c * x - s * y;
              wq[t2] = s * x + c * y;
              const TS u = vp[t2], v = vq[t2];
              vp[t2] = c * u - s * v;
              vq[t2] = s * u + c * v;
            }
            if (sl == 0) atomicAdd(&s_rot, 1);
          }
        }
      } else {
      for (int pidx = w; pidx < rr / 2; pidx += nw) {
        int p = posv(pidx), q = posv(rr - 1 - pidx);
        if (p > q) { int t = p; p = q; q = t; }
        if (q >= r) continue;
        TS* wp = b2 + p * r;
        TS* wq = b2 + q * r;
        TS al = 0, be = 0, ga = 0;
        for (int t = lane; t < r; t += 32) {
          al = fma(wp[t], wp[t], al);
          be = fma(wq[t], wq[t], be);
          ga = fma(wp[t], wq[t], ga);
        }
        al = warp_sum(al); be = warp_sum(be); ga = warp_sum(ga);
        if (ga != (TS)0 && fabs(ga) > thr * sqrt(al * be)) {
          const TS zeta = (be - al) / ((TS)2 * ga);
          const TS t = (zeta >= (TS)0 ? (TS)1 : (TS)-1) / (fabs(zeta) + sqrt((TS)1 + zeta * zeta));
          const TS c = (TS)1 / sqrt((TS)1 + t * t), s = c * t;
          TS* vp = b0 + p * r;
          TS* vq = b0 + q * r;
          for (int t2 = lane; t2 < r; t2 += 32) {
            const TS x = wp[t2], y = wq[t2];
            wp[t2] = c * x - s * y;
            wq[t2] = s * x + c * y;
            const TS u = vp[t2], v = vq[t2];
            vp[t2] = c * u - s * v;
            vq[t2] = s * u + c * v;
          }
          if (lane == 0) atomicAdd(&s_rot, 1);
        }
      }
      }
      __syncthreads();
    }
    if (s_rot == 0) break;
    __syncthreads();
  }
  // singular values = column norms of W; sort descending
  for (int j = w; j < r; j += nw) {
    TS s = 0;
    for (int t = lane; t < r; t += 32) s = fma(b2[t + j * r], b2[t + j * r], s);
    s = warp_sum(s);
    if (lane == 0) sig[j] = sqrt(s);
  }
  __syncthreads();
  if constexpr (JAC8) {
    // the same stable descending order in parallel (r <= RCORE_MAX < 128
    // threads): column j goes to the place of the values above it and of the
    // equal values before it; ord starts as the identity, so every entry
    // stays a valid column even if a non-finite value breaks the order.  k:
    // on the sorted values the findlast below is the count of ratios > eps.
    if ((int)threadIdx.x < r) ord[threadIdx.x] = threadIdx.x;
    __syncthreads();
    if ((int)threadIdx.x < r) {
      const TS sj = sig[threadIdx.x];
      int pos = 0;
      for (int c = 0; c < r; ++c) pos += (sig[c] > sj) || (sig[c] == sj && c < (int)threadIdx.x);
      if (pos < r) ord[pos] = threadIdx.x;
    }
    __syncthreads();
    const double s1 = sig[ord[0]];
    const int kc = __syncthreads_count((int)threadIdx.x < r && (double)sig[threadIdx.x] / s1 > eps_trunc);
    if (threadIdx.x == 0) s_k = (s1 > 0.0) ? kc : 0;
  } else if (threadIdx.x == 0) {
    for (int j = 0; j < r; ++j) ord[j] = j;
    for (int a = 0; a < r; ++a) {             // stable selection sort, descending
      int b = a;
      for (int c = a + 1; c < r; ++c)
        if (sig[ord[c]] > sig[ord[b]]) b = c;
      int t = ord[b];
      for (int c = b; c > a; --c) ord[c] = ord[c - 1];
      ord[a] = t;
    }
    const double s1 = sig[ord[0]];
    int k = 0;
    for (int j = 0; j < r; ++j)
      if ((double)sig[ord[j]] / s1 > eps_trunc) k = j + 1;   // findlast(S/S[1] .> εTrunc)
    if (!(s1 > 0.0)) k = 0;
    s_k = k;
  }
  __syncthreads();
  int k = s_k;
  if (k > J.kcap) {
    if (threadIdx.x == 0) atomicOr(flags, 1);
    k = J.kcap;
  }
  if (nonfinite && threadIdx.x == 0) atomicOr(flags, 2);
  // coefficients: CU[j][c] = W[j, ord c] / s ; CV[j][c] = V[j, ord c] * s
  for (int e = threadIdx.x; e < r * k; e += blockDim.x) {
    const int j = e % r, c = e / r;
    const int o = ord[c];
    const TS s = sig[o];
    b1[e] = s > (TS)0 ? b2[j + o * r] / s : (TS)0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < r * k; e += blockDim.x) {
    const int j = e % r, c = e / r;
    const int o = ord[c];
    b2[e] = b0[j + o * r] * sig[o];
  }
  __syncthreads();
  // (column, row) loops without a division per element; the same sums
  for (int c = 0; c < k; ++c)
    for (int i = threadIdx.x; i < J.m; i += blockDim.x) {
      TS s = 0;
      for (int j = 0; j < r; ++j) s = fma(JA[i + (int64_t)j * J.lda], b1[j + c * r], s);
      J.outA[i + (int64_t)c * J.ldoa] = (double)s;
    }
  for (int c = 0; c < k; ++c)
    for (int i = threadIdx.x; i < J.n; i += blockDim.x) {
      TS s = 0;
      for (int j = 0; j < r; ++j) s = fma(JB[i + (int64_t)j * J.ldb], b2[j + c * r], s);
      J.outB[i + (int64_t)c * J.ldob] = (double)s;
    }
  if (J.zero_fill && k < zlim) {
    zero_cols(J.outA, J.m, J.ldoa, k, zlim);
    zero_cols(J.outB, J.n, J.ldob, k, zlim);
  }
  if (threadIdx.x == 0) *J.rank = k;
}

static __device__ void core_body(const CoreJob& J, int rmax, double eps_trunc, int* __restrict__ flags) {
  core_body_t<double>(J, J.A, J.B, rmax, eps_trunc, flags);
}


}  // namespace hm
