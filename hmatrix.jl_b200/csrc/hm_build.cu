// Construction of an H-matrix on the device: the block partition of
// src/cluster.jl:48-133 on the host, then batched GPU compression
// (aca2, src/hlu.jl:59-111; or dense block + truncated SVD, src/hlu.jl:159-190)
// and dense-leaf generation (kernel_full, src/cluster.jl:258-275).
#include "hm_internal.h"
#include "hm_lowrank.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_set>

namespace hm {

// ---------------------------------------------------------------------------
// dense leaf generation (K1): C[i,j] = K(x_{row0+i}, x_{col0+j}) (+ shift on
// the global diagonal), written column-major with a 16-byte padded column.
// ---------------------------------------------------------------------------
struct DenseJob {
  int64_t row0, col0;
  int32_t m, n;
  int64_t off;      // element offset in the dense pool
  int32_t ld;       // padded column length
  int32_t pad;
};

template <typename TD>
__global__ void dense_leaf_kernel(KernelDesc kd, const double* __restrict__ geom, int64_t ng,
                                  const DenseJob* __restrict__ jobs, TD* __restrict__ pool) {
  const DenseJob J = jobs[blockIdx.x];
  const int64_t total = (int64_t)J.ld * J.n;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
    int i = (int)(e % J.ld);
    int j = (int)(e / J.ld);
    double v = 0.0;
    if (i < J.m) {
      int64_t gi = J.row0 + i, gj = J.col0 + j;
      v = kernel_eval(kd, geom, ng, gi, gj);
      if (gi == gj) v = __dadd_rn(v, kd.shift);
    }
    pool[J.off + e] = (TD)v;
  }
}

// ---------------------------------------------------------------------------
// host-side partition (src/cluster.jl:48-133)
// ---------------------------------------------------------------------------
namespace {

struct NbSet {
  bool identity = true;
  int64_t ncl = 0;
  std::unordered_set<uint64_t> pairs;
  bool neighbours(const hm_handle* h, int32_t s, int32_t t) const {
    if (identity) return !(h->cl_e[s] <= h->cl_s[t] || h->cl_e[t] <= h->cl_s[s]);
    return pairs.count((uint64_t)s * (uint64_t)ncl + (uint64_t)t) != 0;
  }
};

inline bool is_leaf_cluster(const hm_handle* h, int32_t c) { return h->cl_left[c] < 0; }
inline int64_t csize(const hm_handle* h, int32_t c) { return h->cl_e[c] - h->cl_s[c]; }

int validate_tree(hm_handle* h, int64_t ncl) {
  if (ncl < 1) return fail(HM_ERR_ARG, "empty cluster tree");
  if (h->cl_s[0] != 0 || h->cl_e[0] != h->n)
    return fail(HM_ERR_ARG, "cluster 0 must be the root covering [0, n)");
  h->cl_depth.assign(ncl, -1);
  h->cl_depth[0] = 0;
  for (int64_t c = 0; c < ncl; ++c) {
    int64_t l = h->cl_left[c], r = h->cl_right[c];
    if (h->cl_s[c] < 0 || h->cl_e[c] > h->n || h->cl_s[c] >= h->cl_e[c])
      return fail(HM_ERR_ARG, "cluster " + std::to_string(c) + " has an empty or invalid range");
    if ((l < 0) != (r < 0)) return fail(HM_ERR_ARG, "cluster with a single child");
    if (l >= 0) {
      if (l <= c || r <= c || l >= ncl || r >= ncl)
        return fail(HM_ERR_ARG, "children must follow their parent in pre-order");
      if (h->cl_s[l] != h->cl_s[c] || h->cl_e[l] != h->cl_s[r] || h->cl_e[r] != h->cl_e[c])
        return fail(HM_ERR_ARG, "children of cluster " + std::to_string(c) +
                                    " do not split its range into [left | right]");
      h->cl_depth[l] = h->cl_depth[c] + 1;
      h->cl_depth[r] = h->cl_depth[c] + 1;
    }
  }
  for (int64_t c = 0; c < ncl; ++c)
    if (h->cl_depth[c] < 0) return fail(HM_ERR_ARG, "cluster tree is not connected");
  return HM_OK;
}

// Classify a block (src/cluster.jl:60-111).  Returns T_DENSE, T_H, T_RK or -1
// when the block is a low-rank candidate whose type the "svd" route decides.
int classify(const hm_handle* h, const NbSet& nb, int32_t s, int32_t t) {
  const hm_params& p = h->prm;
  int64_t m = csize(h, s), n = csize(h, t);
  if (m <= p.min_block || n <= p.min_block || is_leaf_cluster(h, s) || is_leaf_cluster(h, t))
    return T_DENSE;
  if (m > p.max_block || n > p.max_block) return T_H;
  if (h->cl_s[s] == h->cl_s[t] && h->cl_e[s] == h->cl_e[t]) return T_H;  // s == t
  // aca2 and bbfmm: admissible iff not neighbours (cluster.jl:68-75, 86-97)
  if (p.cons_method == HM_CONS_ACA2 || p.cons_method == HM_CONS_BBFMM) return nb.neighbours(h, s, t) ? T_H : T_RK;
  return -1;
}

void enumerate_leaves(hm_handle* h) {
  // depth-first, children 11, 12, 21, 22: the order of helper() in __c1
  h->leaves.clear();
  std::vector<std::pair<int32_t, int32_t>> st;  // node, depth
  st.push_back({0, 1});
  h->depth = 0;
  while (!st.empty()) {
    auto [id, d] = st.back();
    st.pop_back();
    Node& nd = h->nodes[id];
    if (nd.type == T_H) {
      for (int c = 3; c >= 0; --c) st.push_back({nd.child[c], d + 1});
    } else {
      h->depth = std::max<int64_t>(h->depth, d);
      Leaf L{};
      L.type = nd.type;
      L.s = nd.s;
      L.t = nd.t;
      L.node = id;
      L.row0 = h->cl_s[nd.s];
      L.col0 = h->cl_s[nd.t];
      L.m = (int32_t)csize(h, nd.s);
      L.n = (int32_t)csize(h, nd.t);
      L.k = 0;
      L.off = 0;
      nd.leaf = (int32_t)h->leaves.size();
      h->leaves.push_back(L);
    }
  }
}

int make_nbset(int64_t ncl, int64_t n_nb, const int64_t* nb_pairs, NbSet& nb) {
  nb.ncl = ncl;
  if (nb_pairs != nullptr) {
    nb.identity = false;
    nb.pairs.reserve((size_t)n_nb * 2);
    for (int64_t i = 0; i < n_nb; ++i) {
      int64_t a = nb_pairs[2 * i], b = nb_pairs[2 * i + 1];
      if (a < 0 || b < 0 || a >= ncl || b >= ncl) return fail(HM_ERR_ARG, "neighbour pair out of range");
      nb.pairs.insert((uint64_t)a * (uint64_t)ncl + (uint64_t)b);
    }
  }
  return HM_OK;
}

// The block tree level by level (src/cluster.jl:48-133), then the leaves in
// the reference's order.  decide(undecided) settles the "svd" route's
// candidates (their type needs a compression); the other routes have none.
template <typename Decide>
int partition_levels(hm_handle* h, const NbSet& nb, Decide decide) {
  h->nodes.clear();
  h->nodes.push_back(Node{T_H, 0, 0, {-1, -1, -1, -1}, -1});
  std::vector<int32_t> level{0};
  while (!level.empty()) {
    std::vector<int32_t> undecided;
    for (int32_t id : level) {
      int ty = classify(h, nb, h->nodes[id].s, h->nodes[id].t);
      if (ty < 0) undecided.push_back(id);
      else h->nodes[id].type = (int8_t)ty;
    }
    if (!undecided.empty()) HM_TRY(decide(undecided));
    std::vector<int32_t> next;
    for (int32_t id : level) {
      if (h->nodes[id].type != T_H) continue;
      int32_t s = h->nodes[id].s, t = h->nodes[id].t;
      int32_t sl = (int32_t)h->cl_left[s], sr = (int32_t)h->cl_right[s];
      int32_t tl = (int32_t)h->cl_left[t], tr = (int32_t)h->cl_right[t];
      int32_t cs[4][2] = {{sl, tl}, {sl, tr}, {sr, tl}, {sr, tr}};
      for (int c = 0; c < 4; ++c) {
        int32_t cid = (int32_t)h->nodes.size();
        h->nodes.push_back(Node{T_H, cs[c][0], cs[c][1], {-1, -1, -1, -1}, -1});
        h->nodes[id].child[c] = cid;
        next.push_back(cid);
      }
    }
    level.swap(next);
  }
  enumerate_leaves(h);
  return HM_OK;
}

template <typename T>
int upload(T** dptr, const std::vector<T>& v, cudaStream_t st) {
  if (v.empty()) { *dptr = nullptr; return HM_OK; }
  HM_CUDA_TRY(cudaMalloc((void**)dptr, v.size() * sizeof(T)));
  HM_CUDA_TRY(cudaMemcpyAsync(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return HM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// storage of one low-rank leaf in the pool: B (n x k, column stride pad(n))
// followed by A (m x k, column stride pad(m)); both start on 64-byte
// boundaries.  H_leaf = A * B'.
// ---------------------------------------------------------------------------
static inline int64_t rk_block_elems(int64_t m, int64_t n, int64_t k, int eb) {
  return pad_to((col_pad(n, eb) + col_pad(m, eb)) * k, 64 / eb);
}
static inline int64_t dense_block_elems(int64_t m, int64_t n, int eb) {
  return pad_to(col_pad(m, eb) * n, 64 / eb);
}

int build_handle(hm_handle* h, const double* geom, int64_t ncl, const int64_t* cl_s,
                 const int64_t* cl_e, const int64_t* cl_left, const int64_t* cl_right,
                 int64_t n_nb, const int64_t* nb_pairs) {
  hm_params& p = h->prm;
  const int64_t n = h->n;
  h->cl_s.assign(cl_s, cl_s + ncl);
  h->cl_e.assign(cl_e, cl_e + ncl);
  h->cl_left.assign(cl_left, cl_left + ncl);
  h->cl_right.assign(cl_right, cl_right + ncl);
  HM_TRY(validate_tree(h, ncl));

  NbSet nb;
  HM_TRY(make_nbset(ncl, n_nb, nb_pairs, nb));

  HM_CUDA_TRY(cudaMalloc((void**)&h->d_geom, sizeof(double) * n * h->dim));
  HM_CUDA_TRY(cudaMemcpyAsync(h->d_geom, geom, sizeof(double) * n * h->dim, cudaMemcpyHostToDevice,
                              h->stream));

  // ---- partition, level by level ------------------------------------------
  SvdCandidateStore svd_store;   // factors of "svd"-route low-rank leaves
  HM_TRY(partition_levels(h, nb, [&](const std::vector<int32_t>& undecided) -> int {
    // "svd" route: dense block + compress + (rank <= MaxRank) (cluster.jl:99-107)
    std::vector<int64_t> r0, c0;
    std::vector<int32_t> mm, nn;
    for (int32_t id : undecided) {
      r0.push_back(h->cl_s[h->nodes[id].s]);
      c0.push_back(h->cl_s[h->nodes[id].t]);
      mm.push_back((int32_t)csize(h, h->nodes[id].s));
      nn.push_back((int32_t)csize(h, h->nodes[id].t));
    }
    std::vector<int32_t> ranks;
    HM_TRY(svd_compress_candidates(h, r0, c0, mm, nn, ranks, svd_store, undecided));
    for (size_t i = 0; i < undecided.size(); ++i)
      h->nodes[undecided[i]].type = (ranks[i] <= p.max_rank) ? T_RK : T_H;
    return HM_OK;
  }));

  // ---- a shard: only the leaves of rows [row_lo, row_hi) ------------------
  if (p.row_hi > p.row_lo) {
    if (p.row_lo < 0 || p.row_hi > n) return fail(HM_ERR_ARG, "row range outside [0, n)");
    std::vector<Leaf> keep;
    for (auto& L : h->leaves) {
      const int64_t a = L.row0, b = L.row0 + L.m;
      if (a >= p.row_lo && b <= p.row_hi) {
        h->nodes[L.node].leaf = (int32_t)keep.size();
        keep.push_back(L);
      } else if (b > p.row_lo && a < p.row_hi) {
        return fail(HM_ERR_ARG, "row range [" + std::to_string(p.row_lo) + ", " + std::to_string(p.row_hi) +
                                    ") cuts the rows [" + std::to_string(a) + ", " + std::to_string(b) +
                                    ") of a leaf");
      } else {
        h->nodes[L.node].leaf = -1;
      }
    }
    h->leaves.swap(keep);
  } else if (p.row_lo != 0 || p.row_hi != 0) {
    return fail(HM_ERR_ARG, "row range must satisfy row_lo < row_hi (or both 0)");
  }

  // ---- ranks of the low-rank leaves ---------------------------------------
  std::vector<int64_t> rk_leaf;     // leaf indices of low-rank leaves
  for (int64_t i = 0; i < (int64_t)h->leaves.size(); ++i)
    if (h->leaves[i].type == T_RK) rk_leaf.push_back(i);

  if (p.cons_method == HM_CONS_ACA2) {
    if (p.max_block > ACA_MAX_EXTENT)
      return fail(HM_ERR_UNSUPPORTED, "aca2 on the device supports MaxBlock <= " +
                                          std::to_string(ACA_MAX_EXTENT));
    std::vector<int32_t> ranks;
    HM_TRY(aca2_ranks(h, rk_leaf, ranks));
    for (size_t i = 0; i < rk_leaf.size(); ++i) h->leaves[rk_leaf[i]].k = ranks[i];
  } else if (p.cons_method == HM_CONS_BBFMM) {
    for (int64_t li : rk_leaf)
      h->leaves[li].k = bbfmm_rank(h->leaves[li].m, h->leaves[li].n, (int)h->dim, p.max_rank);
  } else {
    for (int64_t li : rk_leaf) {
      int32_t node = h->leaves[li].node;
      h->leaves[li].k = svd_store.rank_of(node);
    }
  }

  // ---- matvec layout: pools ordered by row group -----------------------------
  HM_TRY(build_matvec_plans(h));
  if (p.cons_method == HM_CONS_ACA2 && (p.build_flags & HM_BUILD_KEEP_PIVOTS)) {
    h->piv_count = (int64_t)rk_leaf.size() * 2 * std::max(1, p.max_rank);
    if (h->piv_count) {
      cudaError_t e = cudaMalloc(&h->d_piv, sizeof(int32_t) * h->piv_count);
      if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("aca2 pivots: ") + cudaGetErrorString(e));
    }
  }
  return fill_pools(h, rk_leaf, false, &svd_store);
}

// Dense leaves and low-rank factors into the laid-out pools.  replay: the
// aca2 factors from the pivots in h->d_piv (hm_new_like).
int fill_pools(hm_handle* h, const std::vector<int64_t>& rk_leaf, bool replay, const SvdCandidateStore* svd_store) {
  const hm_params& p = h->prm;
  const int64_t n = h->n;
  const int deb = dense_elem_bytes(h->storage);
  {
    std::vector<DenseJob> jobs;
    for (auto& L : h->leaves)
      if (L.type == T_DENSE)
        jobs.push_back(DenseJob{L.row0, L.col0, L.m, L.n, L.off, (int32_t)col_pad(L.m, deb), 0});
    if (!jobs.empty()) {
      DenseJob* dj = nullptr;
      HM_TRY(upload(&dj, jobs, h->stream));
      for (size_t b0 = 0; b0 < jobs.size(); b0 += 1u << 30) {
        unsigned nb_ = (unsigned)std::min<size_t>(jobs.size() - b0, 1u << 30);
        if (h->storage == HM_F64)
          dense_leaf_kernel<double><<<nb_, 256, 0, h->stream>>>(h->kd, h->d_geom, n, dj + b0,
                                                                 (double*)h->d_dense);
        else
          dense_leaf_kernel<float><<<nb_, 256, 0, h->stream>>>(h->kd, h->d_geom, n, dj + b0,
                                                                (float*)h->d_dense);
      }
      HM_CUDA_TRY(cudaGetLastError());
      HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
      cudaFree(dj);
    }
  }
  if (p.cons_method == HM_CONS_ACA2) {
    HM_TRY(aca2_write(h, rk_leaf, replay));
  } else if (p.cons_method == HM_CONS_BBFMM) {
    HM_TRY(bbfmm_write(h, rk_leaf));
  } else {
    if (!svd_store) return fail(HM_ERR_UNSUPPORTED, "svd-route factors are not kept");
    HM_TRY(svd_store->write_pool(h, rk_leaf));
  }
  HM_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return HM_OK;
}

// A new H-matrix of the kernel and shift in h->prm on the structure of ref:
// same cluster tree, block partition, ranks and aca2 pivots (hm_new_like).
int build_like(hm_handle* h, const hm_handle* ref) {
  if (!ref->d_piv) return fail(HM_ERR_STATE, "the reference H-matrix kept no aca2 pivots (HM_BUILD_KEEP_PIVOTS)");
  h->cl_s = ref->cl_s; h->cl_e = ref->cl_e; h->cl_left = ref->cl_left; h->cl_right = ref->cl_right;
  h->cl_depth = ref->cl_depth; h->nodes = ref->nodes; h->leaves = ref->leaves; h->depth = ref->depth;
  HM_CUDA_TRY(cudaMalloc((void**)&h->d_geom, sizeof(double) * h->n * h->dim));
  HM_CUDA_TRY(cudaMemcpyAsync(h->d_geom, ref->d_geom, sizeof(double) * h->n * h->dim, cudaMemcpyDeviceToDevice,
                              h->stream));
  h->piv_count = ref->piv_count;
  cudaError_t e = cudaMalloc(&h->d_piv, sizeof(int32_t) * h->piv_count);
  if (e != cudaSuccess) return fail(HM_ERR_OOM, std::string("aca2 pivots: ") + cudaGetErrorString(e));
  HM_CUDA_TRY(cudaMemcpyAsync(h->d_piv, ref->d_piv, sizeof(int32_t) * h->piv_count, cudaMemcpyDeviceToDevice,
                              h->stream));
  std::vector<int64_t> rk_leaf;
  for (int64_t i = 0; i < (int64_t)h->leaves.size(); ++i)
    if (h->leaves[i].type == T_RK) rk_leaf.push_back(i);
  HM_TRY(build_matvec_plans(h));
  return fill_pools(h, rk_leaf, true, nullptr);
}

// The leaves of the block partition alone, on the host (no device is used):
// the aca2 and bbfmm routes decide every block from the tree and the
// adjacency; the svd route needs a compression per candidate and is refused.
int partition_only(hm_handle* h, int64_t ncl, const int64_t* cl_s, const int64_t* cl_e, const int64_t* cl_left,
                   const int64_t* cl_right, int64_t n_nb, const int64_t* nb_pairs) {
  h->cl_s.assign(cl_s, cl_s + ncl);
  h->cl_e.assign(cl_e, cl_e + ncl);
  h->cl_left.assign(cl_left, cl_left + ncl);
  h->cl_right.assign(cl_right, cl_right + ncl);
  HM_TRY(validate_tree(h, ncl));
  NbSet nb;
  HM_TRY(make_nbset(ncl, n_nb, nb_pairs, nb));
  return partition_levels(h, nb, [](const std::vector<int32_t>&) -> int {
    return fail(HM_ERR_UNSUPPORTED, "the svd route decides its blocks by compressing them on the device");
  });
}

// ---------------------------------------------------------------------------
// matvec plans.  Phase 1 (per low-rank leaf) computes z = B' x_seg into a
// z array; phase 2 (per window of MV_WROWS output rows) accumulates
// y = sum A z + sum C x_seg.  The forward plan uses the pools in row-group
// order; the transposed plan reads the same data with A and B swapped.
// ---------------------------------------------------------------------------
int build_matvec_plans(hm_handle* h) {
  const int eb = elem_bytes(h->storage), deb = dense_elem_bytes(h->storage);
  const int64_t ncl = (int64_t)h->cl_s.size();

  // row groups: coarsest cluster that is the row cluster of some leaf
  std::vector<char> is_row(ncl, 0);
  for (auto& L : h->leaves) is_row[L.s] = 1;
  std::vector<int32_t> grp(ncl, -1);
  std::vector<int32_t> group_cluster;
  for (int64_t c = 0; c < ncl; ++c) {      // pre-order: parents before children
    if (grp[c] < 0 && is_row[c]) {
      grp[c] = (int32_t)group_cluster.size();
      group_cluster.push_back((int32_t)c);
    }
    if (h->cl_left[c] >= 0) {
      grp[h->cl_left[c]] = grp[c];
      grp[h->cl_right[c]] = grp[c];
    }
  }
  // groups sorted by their first row
  std::vector<int32_t> gorder(group_cluster.size());
  std::iota(gorder.begin(), gorder.end(), 0);
  std::sort(gorder.begin(), gorder.end(), [&](int32_t a, int32_t b) {
    return h->cl_s[group_cluster[a]] < h->cl_s[group_cluster[b]];
  });
  std::vector<int32_t> grank(group_cluster.size());
  for (size_t i = 0; i < gorder.size(); ++i) grank[gorder[i]] = (int32_t)i;
  for (auto& L : h->leaves) L.group = grank[grp[L.s]];

  // leaf order in the pools: by group, then leaf order
  std::vector<int64_t> order(h->leaves.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return h->leaves[a].group < h->leaves[b].group;
  });
  int64_t rk_off = 0, dn_off = 0;
  h->kmax = 0;
  for (int64_t li : order) {
    Leaf& L = h->leaves[li];
    if (L.type == T_RK) {
      L.off = rk_off;
      rk_off += rk_block_elems(L.m, L.n, L.k, eb);
      h->kmax = std::max(h->kmax, L.k);
    } else {
      L.off = dn_off;
      dn_off += dense_block_elems(L.m, L.n, deb);
    }
  }
  if (h->kmax > MV_KMAX) return fail(HM_ERR_UNSUPPORTED, "rank above " + std::to_string(MV_KMAX));
  h->rk_bytes = (size_t)rk_off * eb;
  h->dense_bytes = (size_t)dn_off * deb;
  if (h->d_rk) cudaFree(h->d_rk);
  if (h->d_dense) cudaFree(h->d_dense);
  h->d_rk = h->d_dense = nullptr;
  if (h->rk_bytes) {
    cudaError_t e = cudaMalloc(&h->d_rk, h->rk_bytes);
    if (e != cudaSuccess) return fail(HM_ERR_OOM, "low-rank pool of " + std::to_string(h->rk_bytes) + " bytes: " + cudaGetErrorString(e));
    HM_CUDA_TRY(cudaMemsetAsync(h->d_rk, 0, h->rk_bytes, h->stream));
  }
  if (h->dense_bytes) {
    cudaError_t e = cudaMalloc(&h->d_dense, h->dense_bytes);
    if (e != cudaSuccess) return fail(HM_ERR_OOM, "dense pool of " + std::to_string(h->dense_bytes) + " bytes: " + cudaGetErrorString(e));
  }
  HM_TRY(build_mv_descriptors(h, order, /*trans=*/0));
  HM_TRY(build_mv_descriptors(h, order, /*trans=*/1));
  // phase-2 shape until hm_autotune: row windows when every leaf starts on a
  // 64-row boundary (bisection of 2^k points), where a window's leaves tile it
  // in aligned pieces; otherwise (KMeans trees, other sizes) by tree clusters,
  // which keeps every load aligned and every lane busy whatever the
  // boundaries (BF16 factors have their own phase 2)
  if (!h->tune.tuned) {
    bool aligned = true;
    for (const Leaf& L : h->leaves) aligned = aligned && (L.row0 % 64 == 0) && (L.col0 % 64 == 0);
    h->tune.p2_split = (aligned || h->storage == HM_BF16) ? 4 : 1;
  }
  return HM_OK;
}

// A handle read back from a file: the cluster tree, block tree and leaf list
// are checked before anything is derived from them (every index in range,
// every leaf inside the matrix and on its own clusters, node and leaf lists
// pointing at each other), then the pools and matvec plans are laid out as
// construction lays them out.
int restore_structure(hm_handle* h) {
  const int64_t ncl = (int64_t)h->cl_s.size();
  if ((int64_t)h->cl_e.size() != ncl || (int64_t)h->cl_left.size() != ncl || (int64_t)h->cl_right.size() != ncl)
    return fail(HM_ERR_ARG, "file: inconsistent cluster arrays");
  HM_TRY(validate_tree(h, ncl));
  const int64_t nn = (int64_t)h->nodes.size(), nl = (int64_t)h->leaves.size();
  if (nn < 1 || nn > ((int64_t)1 << 31) || nl > nn) return fail(HM_ERR_ARG, "file: invalid block tree size");
  for (int64_t i = 0; i < nn; ++i) {
    const Node& d = h->nodes[i];
    if (d.s < 0 || d.s >= ncl || d.t < 0 || d.t >= ncl) return fail(HM_ERR_ARG, "file: node cluster out of range");
    if (d.type == T_H) {
      for (int c = 0; c < 4; ++c)
        if (d.child[c] <= i || d.child[c] >= nn) return fail(HM_ERR_ARG, "file: node child out of range");
    } else if (d.type == T_DENSE || d.type == T_RK) {
      if (d.leaf >= nl || (d.leaf >= 0 && h->leaves[d.leaf].node != i))
        return fail(HM_ERR_ARG, "file: node and leaf lists disagree");
    } else {
      return fail(HM_ERR_ARG, "file: invalid node type");
    }
  }
  for (int64_t i = 0; i < nl; ++i) {
    const Leaf& L = h->leaves[i];
    if (L.node < 0 || L.node >= nn || h->nodes[L.node].leaf != i || h->nodes[L.node].type != L.type)
      return fail(HM_ERR_ARG, "file: leaf " + std::to_string(i) + " does not match its node");
    if (L.s != h->nodes[L.node].s || L.t != h->nodes[L.node].t)
      return fail(HM_ERR_ARG, "file: leaf clusters differ from its node's");
    if (L.row0 != h->cl_s[L.s] || L.col0 != h->cl_s[L.t] || L.m != csize(h, L.s) || L.n != csize(h, L.t))
      return fail(HM_ERR_ARG, "file: leaf extent differs from its clusters");
    if (L.type == T_RK ? (L.k < 0 || L.k > MV_KMAX) : L.k != 0)
      return fail(HM_ERR_ARG, "file: invalid leaf rank");
  }
  return build_matvec_plans(h);
}

void free_handle_data(hm_handle* h) {
  auto fr = [](void* p) { if (p) cudaFree(p); };
  fr(h->d_geom);
  fr(h->d_rk);
  fr(h->d_dense);
  fr(h->d_xs);
  fr(h->d_counter);
  fr(h->d_io);
  fr(h->d_z);
  fr(h->d_xm);
  fr(h->d_tc);
  fr(h->d_tc_err);
  fr(h->d_piv);
  fr(h->d_dd);
  h->d_dd = nullptr;
  h->dd_bytes = 0;
  h->d_piv = nullptr;
  h->piv_count = 0;
  free_tc_plan(h->tc_fwd);
  free_tc_plan(h->tc_bwd);
  h->d_tc = nullptr;
  h->d_tc_err = nullptr;
  h->tc_bytes = 0;
  free_mv_plan(h->fwd);
  free_mv_plan(h->bwd);
  h->d_geom = nullptr;
  h->d_rk = h->d_dense = h->d_xs = h->d_xm = nullptr;
  h->d_z = nullptr;
  h->d_counter = nullptr;
  h->d_io = nullptr;
  h->xs_bytes = h->io_bytes = h->xm_bytes = 0;
  lu_free(h);
}

}  // namespace hm
