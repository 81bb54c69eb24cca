/*
 * CPU FP64 oracle in C for the Hmatrix.jl hot path at large n.
 *
 * TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline.  Only tests/,
 * __graft_entry__.smoke() and the CPU legs of bench.py load it; the product
 * (hmatrix.jl_b200) never does.
 *
 * Restates, following the reference line by line:
 *   orc_partition : the block partition of __c1 (src/cluster.jl:48-133) for
 *                   ConsMethod "aca2" with the identity adjacency, restricted
 *                   to the blocks that touch a row range [rlo, rhi)
 *   orc_aca2      : aca2, d-D form (src/hlu.jl:59-111), deterministic pivots
 *                   (the reference draws rand(findall(Ia)), hlu.jl:83)
 *   orc_matvec    : hmat_matvec! (src/harithm.jl:340-354) over the leaves:
 *                   dense r += C v, low-rank r += A (B' v)
 * Every function works on a leaf range [i0, i1) on the calling thread; the
 * Python loader runs ranges on several threads (ctypes drops the GIL).
 * Kernels use the arithmetic order of the Python oracle (no FMA contraction:
 * compiled with -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { K_CAUCHY = 1, K_INVQUAD = 2, K_GAUSS = 3 };

static inline double orc_kernel(int kind, int dim, double p, const double* g, int64_t ng, int64_t i,
                                int64_t j) {
  double s = 0.0;
  for (int q = 0; q < dim; ++q) {
    double d = g[i + q * ng] - g[j + q * ng];
    if (kind == K_CAUCHY && p != 1.0) d = d / p;
    double t = d * d;
    s = (q == 0) ? t : s + t;
  }
  if (kind == K_GAUSS) return exp(-(s / (2.0 * p * p)));
  if (kind == K_INVQUAD) return 1.0 / (p + s);
  return 1.0 / (1.0 + s);
}

double orc_kernel_value(int kind, int dim, double p, const double* g, int64_t ng, int64_t i, int64_t j) {
  return orc_kernel(kind, dim, p, g, ng, i, j);
}

/* __c1 for ConsMethod "aca2", Adj = I: out[5*i..] = (type 0 dense/1 rk, row0, col0, m, n) */
typedef struct {
  const int64_t *s, *e, *l, *r;
  int64_t minb, maxb, rlo, rhi, cap, cnt;
  int64_t* out;
} part_ctx;

static void part_rec(part_ctx* c, int64_t s, int64_t t) {
  const int64_t m = c->e[s] - c->s[s], n = c->e[t] - c->s[t];
  if (c->e[s] <= c->rlo || c->s[s] >= c->rhi) return; /* rows outside the sample */
  int type;
  if (m <= c->minb || n <= c->minb || c->l[s] < 0 || c->l[t] < 0) type = 0;
  else if (m > c->maxb || n > c->maxb) type = 2;
  else if (c->s[s] == c->s[t] && c->e[s] == c->e[t]) type = 2;
  else type = 1; /* disjoint clusters at the same depth: Neighbors == 0 */
  if (type == 2) {
    part_rec(c, c->l[s], c->l[t]);
    part_rec(c, c->l[s], c->r[t]);
    part_rec(c, c->r[s], c->l[t]);
    part_rec(c, c->r[s], c->r[t]);
    return;
  }
  if (c->cnt < c->cap) {
    int64_t* o = c->out + 5 * c->cnt;
    o[0] = type; o[1] = c->s[s]; o[2] = c->s[t]; o[3] = m; o[4] = n;
  }
  c->cnt++;
}

int64_t orc_partition(const int64_t* s, const int64_t* e, const int64_t* l, const int64_t* r, int64_t min_block,
                      int64_t max_block, int64_t rlo, int64_t rhi, int64_t cap, int64_t* out) {
  part_ctx c = {s, e, l, r, min_block, max_block, rlo, rhi, cap, 0, out};
  part_rec(&c, 0, 0);
  return c.cnt;
}

/* aca2, d-D (src/hlu.jl:59-111).  A: m x R, B: n x R column-major; returns rank. */
int orc_aca2(int kind, int dim, double p, const double* g, int64_t ng, int64_t row0, int64_t col0, int m, int n,
             int R, double eps_comp, double* A, double* B) {
  unsigned char* used = (unsigned char*)calloc((size_t)m, 1);
  int tau = 0, rank = R;
  double na0 = 1.0, nb0 = 1.0;
  for (int r = 0; r < R; ++r) {
    double best = -1.0, delta = 0.0, nB = 0.0;
    int sigma = 0;
    double* b = B + (int64_t)r * n;
    for (int j = 0; j < n; ++j) {
      double v = orc_kernel(kind, dim, p, g, ng, row0 + tau, col0 + j);
      double s = 0.0;
      for (int q = 0; q < r; ++q) s += B[j + (int64_t)q * n] * A[tau + (int64_t)q * m];
      v = v - s;
      b[j] = v;
      nB += v * v;
      if (fabs(v) > best) { best = fabs(v); sigma = j; delta = v; }
    }
    if (delta == 0.0) { rank = r; break; }
    used[tau] = 1;
    double* a = A + (int64_t)r * m;
    double nA = 0.0, best2 = -1.0;
    int idx2 = -1;
    for (int i = 0; i < m; ++i) {
      double v = orc_kernel(kind, dim, p, g, ng, row0 + i, col0 + sigma);
      double s = 0.0;
      for (int q = 0; q < r; ++q) s += A[i + (int64_t)q * m] * B[sigma + (int64_t)q * n];
      v = (v - s) / delta;
      a[i] = v;
      nA += v * v;
      if (!used[i] && fabs(v) > best2) { best2 = fabs(v); idx2 = i; }
    }
    double na = sqrt(nA), nb = sqrt(nB);
    if (r == 0) { na0 = na; nb0 = nb; }
    if (idx2 < 0) { rank = r + 1; break; }
    tau = idx2;
    if (na * nb / na0 / nb0 <= eps_comp) { rank = r + 1; break; }
  }
  free(used);
  return rank;
}

/* Build the factors of leaves [i0, i1) (5 ints per leaf as orc_partition
 * writes).  pool == NULL: ranks into rank[] only.  Otherwise pool[off[i]..]
 * gets A (m x k) then B (n x k) for low-rank leaves and C (m x n) for dense. */
void orc_build(int kind, int dim, double p, const double* g, int64_t ng, int64_t i0, int64_t i1, const int64_t* lv,
               int R, double eps_comp, int32_t* rank, const int64_t* off, double* pool) {
  double* sa = NULL;
  size_t cap = 0;
  for (int64_t i = i0; i < i1; ++i) {
    const int64_t* o = lv + 5 * i;
    const int m = (int)o[3], n = (int)o[4];
    if (o[0] == 0) {
      if (pool) {
        double* C = pool + off[i];
        for (int j = 0; j < n; ++j)
          for (int ii = 0; ii < m; ++ii) C[ii + (int64_t)j * m] = orc_kernel(kind, dim, p, g, ng, o[1] + ii, o[2] + j);
      }
      rank[i] = 0;
      continue;
    }
    size_t need = (size_t)R * (size_t)(m + n);
    if (need > cap) { free(sa); sa = (double*)malloc(sizeof(double) * need); cap = need; }
    int k = orc_aca2(kind, dim, p, g, ng, o[1], o[2], m, n, R, eps_comp, sa, sa + (size_t)R * m);
    rank[i] = k;
    if (pool) {
      memcpy(pool + off[i], sa, sizeof(double) * (size_t)m * k);
      memcpy(pool + off[i] + (int64_t)m * k, sa + (size_t)R * m, sizeof(double) * (size_t)n * k);
    }
  }
  free(sa);
}

/* hmat_matvec! over leaves [i0, i1): y[t] += contribution to row rlo + t for
 * the rows inside [rlo, rhi).  lv: 5 ints per leaf, rank[i], off[i] into pool. */
void orc_matvec(int64_t i0, int64_t i1, const int64_t* lv, const int32_t* rank, const int64_t* off,
                const double* pool, const double* x, double* y, int64_t rlo, int64_t rhi) {
  double z[256];
  for (int64_t i = i0; i < i1; ++i) {
    const int64_t* o = lv + 5 * i;
    const int64_t m = o[3], n = o[4], r0 = o[1], c0 = o[2];
    const double* d = pool + off[i];
    const int64_t lo = r0 < rlo ? rlo - r0 : 0;
    const int64_t hi = r0 + m > rhi ? rhi - r0 : m;
    if (o[0] == 0) {
      for (int64_t j = 0; j < n; ++j) {
        const double xv = x[c0 + j];
        const double* col = d + j * m;
        for (int64_t ii = lo; ii < hi; ++ii) y[r0 + ii - rlo] += col[ii] * xv;
      }
    } else {
      const int k = rank[i];
      const double* A = d;
      const double* B = d + m * k;
      for (int q = 0; q < k; ++q) {
        double s = 0.0;
        const double* b = B + (int64_t)q * n;
        for (int64_t j = 0; j < n; ++j) s += b[j] * x[c0 + j];
        z[q] = s;
      }
      for (int q = 0; q < k; ++q) {
        const double* a = A + (int64_t)q * m;
        const double zq = z[q];
        for (int64_t ii = lo; ii < hi; ++ii) y[r0 + ii - rlo] += a[ii] * zq;
      }
    }
  }
}
