/* ORACLE — test infrastructure only. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker; the product path never links or calls it.
 *
 * CPU restatement of the sparse symmetric-indefinite multifrontal LDL^T that hsolve obtains from
 * MUMPS 5.8.2 (SYM=2), following its documented behaviour, not its code:
 *   - symmetric iterative scaling of K (ICNTL(8)=7, hsolve src/factor/mumps_factorization.cpp:170-176),
 *     restated as Ruiz infinity-norm equilibration;
 *   - multifrontal elimination on the elimination tree of the given pivot order (PERM_IN), with
 *     fundamental supernodes;
 *   - threshold pivoting with 1x1 and 2x2 pivots restricted to the fully-summed block
 *     (MUMPS dfac_front_LDLT_type1.F behaviour, threshold u = CNTL(1) = 0.01), pivots that fail
 *     are delayed to the parent front (INFOG(13));
 *   - null-pivot detection (ICNTL(24)=1, CNTL(3)=1e-8 relative to the largest entry of the scaled
 *     matrix; hsolve include/hsolve/factor.hpp:79-114): such pivots count as zero, and the
 *     factorization is reported invalid (factorize() == false, factor.hpp:374-381);
 *   - inertia from D (neg = INFOG(12), zero = null pivots; src/factor/mumps_factorization.cpp:360-381);
 *   - forward / diagonal / backward solves with nrhs right-hand sides (JOB=3, :459-527).
 * Parity is anchored on exact spectra (Sylvester counts) and dense checks, not on MUMPS bits.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int64_t m;      /* front order */
  int64_t e;      /* eliminated pivots */
  int32_t *idx;   /* global (permuted) index of each front position, m entries */
  double *L;      /* m x e, column-major: unit lower part holds L, diag/2x2 hold D */
  int8_t *piv;    /* e entries: 1 = 1x1, 2 = first of a 2x2, 3 = second of a 2x2, 0 = null pivot */
} front_t;

typedef struct {
  int64_t n;
  int32_t *perm;   /* new -> old */
  int32_t *iperm;  /* old -> new */
  /* lower CSC of the permuted matrix: column j holds rows i >= j (diag first) */
  int64_t *lp;
  int32_t *li;
  int64_t *lsrc;   /* index into the caller's upper-CSR value array */
  int32_t *parent; /* elimination tree */
  int32_t ns;
  int32_t *sn_first;   /* ns + 1 */
  int32_t *sn_parent;
  int64_t *sn_rp;      /* structure rows per supernode */
  int32_t *sn_rows;
  /* numeric */
  double *scale;       /* per original index */
  front_t *fronts;
  int64_t neg, zero, pos, delayed, twobytwo, nullpiv;
  int valid;
  double flops;
  int64_t nnz_l;
} mf_t;

static void *xmalloc(size_t s) { void *p = malloc(s ? s : 1); if (!p) abort(); return p; }
static void *xcalloc(size_t n, size_t s) { void *p = calloc(n ? n : 1, s ? s : 1); if (!p) abort(); return p; }

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* Build the permuted lower CSC and the elimination tree for the order `perm` (new -> old). */
static void build_pattern(mf_t *f, int64_t n, const int64_t *rp, const int32_t *ci) {
  int64_t nnz = rp[n];
  int64_t *cnt = xcalloc(n + 1, sizeof(int64_t));
  for (int64_t r = 0; r < n; ++r)
    for (int64_t p = rp[r]; p < rp[r + 1]; ++p) {
      int32_t a = f->iperm[r], b = f->iperm[ci[p]];
      cnt[(a < b ? a : b) + 1]++;
    }
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  f->lp = xmalloc((n + 1) * sizeof(int64_t));
  memcpy(f->lp, cnt, (n + 1) * sizeof(int64_t));
  f->li = xmalloc(nnz * sizeof(int32_t));
  f->lsrc = xmalloc(nnz * sizeof(int64_t));
  for (int64_t r = 0; r < n; ++r)
    for (int64_t p = rp[r]; p < rp[r + 1]; ++p) {
      int32_t a = f->iperm[r], b = f->iperm[ci[p]];
      int32_t col = a < b ? a : b, row = a < b ? b : a;
      int64_t q = cnt[col]++;
      f->li[q] = row;
      f->lsrc[q] = p;
    }
  free(cnt);
  /* etree (Liu) needs, for each k, the columns j < k with K(k, j) != 0: walk the lower CSC */
  int32_t *anc = xmalloc(n * sizeof(int32_t));
  f->parent = xmalloc(n * sizeof(int32_t));
  /* row lists: transpose of the strictly lower part */
  int64_t *tp = xcalloc(n + 1, sizeof(int64_t));
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = f->lp[j]; p < f->lp[j + 1]; ++p)
      if (f->li[p] > j) tp[f->li[p] + 1]++;
  for (int64_t k = 0; k < n; ++k) tp[k + 1] += tp[k];
  int32_t *tj = xmalloc((tp[n] + 1) * sizeof(int32_t));
  int64_t *tc = xmalloc((n + 1) * sizeof(int64_t));
  memcpy(tc, tp, (n + 1) * sizeof(int64_t));
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = f->lp[j]; p < f->lp[j + 1]; ++p)
      if (f->li[p] > j) tj[tc[f->li[p]]++] = (int32_t)j;
  for (int64_t k = 0; k < n; ++k) {
    f->parent[k] = -1;
    anc[k] = -1;
    for (int64_t p = tp[k]; p < tp[k + 1]; ++p) {
      int32_t r = tj[p];
      while (anc[r] != -1 && anc[r] != k) { int32_t t = anc[r]; anc[r] = (int32_t)k; r = t; }
      if (anc[r] == -1) { anc[r] = (int32_t)k; f->parent[r] = (int32_t)k; }
    }
  }
  free(anc); free(tp); free(tj); free(tc);
}

static void free_pattern(mf_t *f) {
  free(f->lp); free(f->li); free(f->lsrc); free(f->parent);
  f->lp = NULL; f->li = NULL; f->lsrc = NULL; f->parent = NULL;
}

/* Analyse: order (new -> old, NULL = natural), postorder the etree, fundamental supernodes. */
void *mf_analyze(int64_t n, const int64_t *rp, const int32_t *ci, const int32_t *order) {
  mf_t *f = xcalloc(1, sizeof(mf_t));
  f->n = n;
  f->perm = xmalloc(n * sizeof(int32_t));
  f->iperm = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) f->perm[i] = order ? order[i] : (int32_t)i;
  for (int64_t i = 0; i < n; ++i) f->iperm[f->perm[i]] = (int32_t)i;
  build_pattern(f, n, rp, ci);
  /* postorder of the etree (children visited in increasing order) */
  int32_t *head = xmalloc(n * sizeof(int32_t)), *next = xmalloc(n * sizeof(int32_t));
  int32_t *stack = xmalloc(n * sizeof(int32_t)), *post = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) head[i] = -1;
  for (int64_t j = n - 1; j >= 0; --j)
    if (f->parent[j] >= 0) { next[j] = head[f->parent[j]]; head[f->parent[j]] = (int32_t)j; }
  int64_t k = 0;
  for (int64_t r = 0; r < n; ++r) {
    if (f->parent[r] != -1) continue;
    int64_t top = 0;
    stack[top++] = (int32_t)r;
    while (top) {
      int32_t v = stack[top - 1];
      int32_t c = head[v];
      if (c == -1) { top--; post[k++] = v; }
      else { head[v] = next[c]; stack[top++] = c; }
    }
  }
  int32_t *perm2 = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) perm2[i] = f->perm[post[i]];
  memcpy(f->perm, perm2, n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) f->iperm[f->perm[i]] = (int32_t)i;
  free(perm2); free(post); free(stack); free(head); free(next);
  free_pattern(f);
  build_pattern(f, n, rp, ci);
  /* column structures by merging children (sorted int arrays) */
  int64_t *cp = xmalloc((n + 1) * sizeof(int64_t));
  int32_t **cs = xmalloc(n * sizeof(int32_t *));
  int64_t *clen = xmalloc(n * sizeof(int64_t));
  int32_t *mark = xmalloc(n * sizeof(int32_t));
  int32_t *nchild = xcalloc(n, sizeof(int32_t));
  int32_t *buf = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) mark[i] = -1;
  int32_t *chead = xmalloc(n * sizeof(int32_t)), *cnext = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) chead[i] = -1;
  for (int64_t j = n - 1; j >= 0; --j)
    if (f->parent[j] >= 0) { cnext[j] = chead[f->parent[j]]; chead[f->parent[j]] = (int32_t)j; nchild[f->parent[j]]++; }
  for (int64_t j = 0; j < n; ++j) {
    int64_t len = 0;
    buf[len++] = (int32_t)j; mark[j] = (int32_t)j;
    for (int64_t p = f->lp[j]; p < f->lp[j + 1]; ++p) {
      int32_t i = f->li[p];
      if (mark[i] != j) { mark[i] = (int32_t)j; buf[len++] = i; }
    }
    for (int32_t c = chead[j]; c != -1; c = cnext[c]) {
      for (int64_t q = 1; q < clen[c]; ++q) {
        int32_t i = cs[c][q];
        if (mark[i] != j) { mark[i] = (int32_t)j; buf[len++] = i; }
      }
    }
    qsort(buf, len, sizeof(int32_t), cmp_i32);
    cs[j] = xmalloc(len * sizeof(int32_t));
    memcpy(cs[j], buf, len * sizeof(int32_t));
    clen[j] = len;
  }
  free(cp);
  /* fundamental supernodes */
  int32_t *first = xmalloc((n + 1) * sizeof(int32_t));
  int32_t ns = 0;
  for (int64_t j = 0; j < n; ++j) {
    int join = j > 0 && f->parent[j - 1] == j && clen[j - 1] == clen[j] + 1 && nchild[j] == 1;
    if (!join) first[ns++] = (int32_t)j;
  }
  first[ns] = (int32_t)n;
  f->ns = ns;
  f->sn_first = xmalloc((ns + 1) * sizeof(int32_t));
  memcpy(f->sn_first, first, (ns + 1) * sizeof(int32_t));
  int32_t *col2sn = xmalloc(n * sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s)
    for (int32_t j = first[s]; j < first[s + 1]; ++j) col2sn[j] = s;
  f->sn_parent = xmalloc(ns * sizeof(int32_t));
  f->sn_rp = xmalloc((ns + 1) * sizeof(int64_t));
  f->sn_rp[0] = 0;
  for (int32_t s = 0; s < ns; ++s) {
    int32_t last = first[s + 1] - 1;
    f->sn_parent[s] = f->parent[last] >= 0 ? col2sn[f->parent[last]] : -1;
    f->sn_rp[s + 1] = f->sn_rp[s] + clen[first[s]];
  }
  f->sn_rows = xmalloc(f->sn_rp[ns] * sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s) memcpy(f->sn_rows + f->sn_rp[s], cs[first[s]], clen[first[s]] * sizeof(int32_t));
  for (int64_t j = 0; j < n; ++j) free(cs[j]);
  free(cs); free(clen); free(mark); free(nchild); free(buf); free(chead); free(cnext); free(first); free(col2sn);
  f->fronts = xcalloc(ns, sizeof(front_t));
  return f;
}

static void free_numeric(mf_t *f) {
  if (!f->fronts) return;
  for (int32_t s = 0; s < f->ns; ++s) {
    free(f->fronts[s].idx); free(f->fronts[s].L); free(f->fronts[s].piv);
    memset(&f->fronts[s], 0, sizeof(front_t));
  }
  free(f->scale); f->scale = NULL;
}

void mf_free(void *h) {
  mf_t *f = h;
  if (!f) return;
  free_numeric(f);
  free(f->fronts);
  free_pattern(f);
  free(f->perm); free(f->iperm); free(f->sn_first); free(f->sn_parent); free(f->sn_rp); free(f->sn_rows);
  free(f);
}

/* symmetric swap of positions p < q of the lower-stored front F (order m, ld m) */
static void sym_swap(double *F, int64_t m, int32_t *idx, int64_t p, int64_t q) {
  if (p == q) return;
  if (p > q) { int64_t t = p; p = q; q = t; }
#define A_(i, j) F[(i) + (j) * m]
  for (int64_t c = 0; c < p; ++c) { double t = A_(p, c); A_(p, c) = A_(q, c); A_(q, c) = t; }
  { double t = A_(p, p); A_(p, p) = A_(q, q); A_(q, q) = t; }
  for (int64_t c = p + 1; c < q; ++c) { double t = A_(c, p); A_(c, p) = A_(q, c); A_(q, c) = t; }
  for (int64_t i = q + 1; i < m; ++i) { double t = A_(i, p); A_(i, p) = A_(i, q); A_(i, q) = t; }
  int32_t t = idx[p]; idx[p] = idx[q]; idx[q] = t;
#undef A_
}

/* max |F(i, c)| over rows/cols i != c and i not in `skip` (skip < 0: none), i >= j0 */
static double col_max(const double *F, int64_t m, int64_t j0, int64_t c, int64_t skip) {
  double g = 0.0;
  for (int64_t i = j0; i < c; ++i) if (i != skip) { double v = fabs(F[c + i * m]); if (v > g) g = v; }
  for (int64_t i = c + 1; i < m; ++i) if (i != skip) { double v = fabs(F[i + c * m]); if (v > g) g = v; }
  return g;
}

/* rank-1 / rank-2 update of the trailing matrix rows/cols >= j0 */
static void update1(double *F, int64_t m, int64_t j, int64_t j0) {
  const double d = F[j + j * m];
  const double *col = F + j * m;
  int64_t cnt = m - j0;
#pragma omp parallel for schedule(static) if (cnt > 384)
  for (int64_t c = j0; c < m; ++c) {
    const double f = col[c] / d;
    double *dst = F + c * m;
    for (int64_t i = c; i < m; ++i) dst[i] -= col[i] * f;
  }
}

static void update2(double *F, int64_t m, int64_t j, int64_t j0) {
  const double a = F[j + j * m], b = F[(j + 1) + j * m], c2 = F[(j + 1) + (j + 1) * m];
  const double det = a * c2 - b * b;
  const double ia = c2 / det, ib = -b / det, ic = a / det;
  const double *c0 = F + j * m, *c1 = F + (j + 1) * m;
  int64_t cnt = m - j0;
#pragma omp parallel for schedule(static) if (cnt > 384)
  for (int64_t c = j0; c < m; ++c) {
    /* w = D^{-1} [F(c,j); F(c,j+1)] */
    const double w0 = ia * c0[c] + ib * c1[c];
    const double w1 = ib * c0[c] + ic * c1[c];
    double *dst = F + c * m;
    for (int64_t i = c; i < m; ++i) dst[i] -= c0[i] * w0 + c1[i] * w1;
  }
}

typedef struct {
  double u, null_thr;
  int detect;
} piv_opts;

/* Partial LDL^T of front F (order m, fully summed nfs). Returns eliminated count; the front's
 * positions [e, nfs) are delayed. Counts go to f. root: no parent, pivots may not be delayed. */
static void eliminate1(mf_t *f, double *F, int64_t m, int64_t j, int8_t *piv) {
  piv[j] = 1;
  if (F[j + j * m] < 0) f->neg++; else f->pos++;
  update1(F, m, j, j + 1);
  for (int64_t i = j + 1; i < m; ++i) F[i + j * m] /= F[j + j * m];
}

static void eliminate2(mf_t *f, double *F, int64_t m, int64_t j, int8_t *piv) {
  piv[j] = 2; piv[j + 1] = 3; f->twobytwo++;
  const double a2 = F[j + j * m], b2 = F[(j + 1) + j * m], c2 = F[(j + 1) + (j + 1) * m];
  const double d2 = a2 * c2 - b2 * b2;
  if (d2 < 0) { f->neg++; f->pos++; } else if (a2 + c2 < 0) f->neg += 2; else f->pos += 2;
  update2(F, m, j, j + 2);
  const double ia2 = c2 / d2, ib2 = -b2 / d2, ic2 = a2 / d2;
  for (int64_t i = j + 2; i < m; ++i) {
    const double x0 = F[i + j * m], x1 = F[i + (j + 1) * m];
    F[i + j * m] = ia2 * x0 + ib2 * x1;
    F[i + (j + 1) * m] = ib2 * x0 + ic2 * x1;
  }
}

static void null_pivot(mf_t *f, double *F, int64_t m, int64_t j, int8_t *piv) {
  piv[j] = 0; f->zero++; f->nullpiv++; f->valid = 0;
  for (int64_t i = j + 1; i < m; ++i) F[i + j * m] = 0.0;
}

/* Partial LDL^T of front F (order m, fully summed nfs). Returns eliminated count; the front's
 * positions [e, nfs) are delayed. Counts go to f. root: no parent, pivots may not be delayed.
 * Candidate columns that fail are moved behind a shrinking limit and retried after any progress. */
static int64_t factor_front(mf_t *f, double *F, int64_t m, int64_t nfs, int32_t *idx, int8_t *piv,
                            const piv_opts *o, int root) {
  int64_t j = 0, lim = nfs;
  int progress = 0;
  while (j < nfs) {
    if (j >= lim) {
      if (progress) { lim = nfs; progress = 0; continue; }
      if (!root) break;
      /* root: nothing can be delayed; Bunch-Kaufman's choice on column j without threshold */
      const double alpha = 0.6403882032022076;
      const double dcc = fabs(F[j + j * m]);
      const double gc = col_max(F, m, j, j, -1);
      int64_t r = -1; double best = 0.0;
      for (int64_t i = j + 1; i < nfs; ++i) { double v = fabs(F[i + j * m]); if (v > best) { best = v; r = i; } }
      if (r < 0 || dcc >= alpha * gc) {
        if (F[j + j * m] == 0.0) null_pivot(f, F, m, j, piv); else eliminate1(f, F, m, j, piv);
        j++;
      } else {
        sym_swap(F, m, idx, j + 1, r);
        eliminate2(f, F, m, j, piv);
        j += 2;
      }
      lim = nfs;
      continue;
    }
    const int64_t c = j;
    const double dcc = fabs(F[c + c * m]);
    const double gc = col_max(F, m, j, c, -1);
    if (o->detect && (dcc > gc ? dcc : gc) <= o->null_thr) {
      null_pivot(f, F, m, j, piv);
      j++; progress = 1; continue;
    }
    if (dcc >= o->u * gc && dcc > 0.0) {
      eliminate1(f, F, m, j, piv);
      j++; progress = 1; continue;
    }
    /* candidate partner r among fully-summed rows */
    int64_t r = -1; double best = 0.0;
    for (int64_t i = j + 1; i < nfs; ++i) { double v = fabs(F[i + c * m]); if (v > best) { best = v; r = i; } }
    if (r >= 0) {
      const double a = F[c + c * m], b = F[r + c * m], cc = F[r + r * m];
      const double det = a * cc - b * b;
      const double gc2 = col_max(F, m, j, c, r), gr2 = col_max(F, m, j, r, c);
      if (det != 0.0) {
        const double ia = fabs(cc / det), ib = fabs(b / det), ic = fabs(a / det);
        if (ia * gc2 + ib * gr2 <= 1.0 / o->u && ib * gc2 + ic * gr2 <= 1.0 / o->u) {
          sym_swap(F, m, idx, j + 1, r);
          if (lim == j + 1) lim = j + 2;  /* the partner came from behind the limit */
          eliminate2(f, F, m, j, piv);
          j += 2; progress = 1; if (lim < j) lim = j; continue;
        }
      }
      const double drr = fabs(F[r + r * m]);
      const double gr = col_max(F, m, j, r, -1);
      if (drr >= o->u * gr && drr > 0.0) {
        sym_swap(F, m, idx, j, r);
        eliminate1(f, F, m, j, piv);
        j++; progress = 1; if (lim < j) lim = j; continue;
      }
    }
    /* column c fails: move it behind the limit */
    lim--;
    sym_swap(F, m, idx, j, lim);
  }
  return j;
}

/* Ruiz symmetric equilibration of the upper-CSR matrix: scale[i] for original indices */
static void ruiz(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, double *d) {
  double *r = xmalloc(n * sizeof(double));
  for (int64_t i = 0; i < n; ++i) d[i] = 1.0;
  for (int it = 0; it < 20; ++it) {
    for (int64_t i = 0; i < n; ++i) r[i] = 0.0;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
        const int32_t j = ci[p];
        const double a = fabs(v[p]) * d[i] * d[j];
        if (a > r[i]) r[i] = a;
        if (a > r[j]) r[j] = a;
      }
    double dev = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      if (r[i] > 0.0) { d[i] /= sqrt(r[i]); double e = fabs(1.0 - r[i]); if (e > dev) dev = e; }
    }
    if (dev < 1e-2) break;
  }
  free(r);
}

/* Numeric factorization of the symmetric matrix given by its upper CSR (same pattern as
 * analysed) with values v. Returns 1 if valid (no null pivot), 0 otherwise; inertia in out[0..2],
 * out[3] = delayed pivots, out[4] = 2x2 pivots, out[5] = null pivots. */
int mf_factor(void *h, const int64_t *rp, const int32_t *ci, const double *v, double u, double null_tol,
              int detect, int scaling, int64_t *out) {
  mf_t *f = h;
  const int64_t n = f->n;
  free_numeric(f);
  f->neg = f->zero = f->pos = f->delayed = f->twobytwo = f->nullpiv = 0;
  f->valid = 1;
  f->flops = 0.0;
  f->nnz_l = 0;
  f->scale = xmalloc(n * sizeof(double));
  if (scaling) ruiz(n, rp, ci, v, f->scale);
  else for (int64_t i = 0; i < n; ++i) f->scale[i] = 1.0;
  double amax = 0.0;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
      double a = fabs(v[p]) * f->scale[i] * f->scale[ci[p]];
      if (a > amax) amax = a;
    }
  piv_opts o = {u, null_tol * amax, detect};
  int32_t *pos = xmalloc(n * sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) pos[i] = -1;
  /* contribution blocks of finished fronts, waiting for their parent */
  double **cb = xcalloc(f->ns, sizeof(double *));
  int32_t **cbidx = xcalloc(f->ns, sizeof(int32_t *));
  int64_t *cbm = xcalloc(f->ns, sizeof(int64_t));
  int64_t *cbdel = xcalloc(f->ns, sizeof(int64_t));
  int32_t *chead = xmalloc(f->ns * sizeof(int32_t)), *cnext = xmalloc(f->ns * sizeof(int32_t));
  for (int32_t s = 0; s < f->ns; ++s) chead[s] = -1;
  for (int32_t s = f->ns - 1; s >= 0; --s)
    if (f->sn_parent[s] >= 0) { cnext[s] = chead[f->sn_parent[s]]; chead[f->sn_parent[s]] = s; }
  for (int32_t s = 0; s < f->ns; ++s) {
    const int64_t k = f->sn_first[s + 1] - f->sn_first[s];
    const int64_t nr = f->sn_rp[s + 1] - f->sn_rp[s];
    const int32_t *rows = f->sn_rows + f->sn_rp[s];
    int64_t nd = 0;
    for (int32_t c = chead[s]; c != -1; c = cnext[c]) nd += cbdel[c];
    const int64_t m = nr + nd, nfs = k + nd;
    int32_t *idx = xmalloc(m * sizeof(int32_t));
    int64_t t = 0;
    for (int64_t q = 0; q < k; ++q) idx[t++] = rows[q];
    for (int32_t c = chead[s]; c != -1; c = cnext[c])
      for (int64_t q = 0; q < cbdel[c]; ++q) idx[t++] = cbidx[c][q];
    for (int64_t q = k; q < nr; ++q) idx[t++] = rows[q];
    for (int64_t q = 0; q < m; ++q) pos[idx[q]] = (int32_t)q;
    double *F = xcalloc(m * m, sizeof(double));
    for (int64_t j = f->sn_first[s]; j < f->sn_first[s + 1]; ++j)
      for (int64_t p = f->lp[j]; p < f->lp[j + 1]; ++p) {
        const int32_t i = f->li[p];
        const int64_t src = f->lsrc[p];
        const double val = v[src] * f->scale[f->perm[i]] * f->scale[f->perm[j]];
        int64_t a = pos[i], b = pos[j];
        if (a < b) { int64_t tt = a; a = b; b = tt; }
        F[a + b * m] += val;
      }
    for (int32_t c = chead[s]; c != -1; c = cnext[c]) {
      const int64_t mc = cbm[c];
      for (int64_t bb = 0; bb < mc; ++bb) {
        const int64_t pb = pos[cbidx[c][bb]];
        for (int64_t aa = bb; aa < mc; ++aa) {
          int64_t pa = pos[cbidx[c][aa]], pc = pb;
          if (pa < pc) { int64_t tt = pa; pa = pc; pc = tt; }
          F[pa + pc * m] += cb[c][aa + bb * mc];
        }
      }
      free(cb[c]); free(cbidx[c]); cb[c] = NULL; cbidx[c] = NULL;
    }
    for (int64_t q = 0; q < m; ++q) pos[idx[q]] = -1;
    int8_t *piv = xcalloc(nfs > 0 ? nfs : 1, 1);
    const int root = f->sn_parent[s] < 0;
    const int64_t e = factor_front(f, F, m, nfs, idx, piv, &o, root);
    for (int64_t jj = 0; jj < e; ++jj) {
      const double r = (double)(m - jj - 1);
      f->flops += r + r * (r + 1.0);
    }
    f->nnz_l += e * m - e * (e - 1) / 2;
    /* keep L (m x e) and the contribution block (positions e..m-1) */
    front_t *fr = &f->fronts[s];
    fr->m = m; fr->e = e; fr->idx = idx; fr->piv = piv;
    fr->L = xmalloc((e > 0 ? e : 1) * m * sizeof(double));
    memcpy(fr->L, F, e * m * sizeof(double));
    const int64_t mc = m - e;
    if (mc > 0 && !root) {
      cb[s] = xmalloc(mc * mc * sizeof(double));
      for (int64_t bb = 0; bb < mc; ++bb)
        for (int64_t aa = bb; aa < mc; ++aa) cb[s][aa + bb * mc] = F[(e + aa) + (e + bb) * m];
      cbidx[s] = xmalloc(mc * sizeof(int32_t));
      memcpy(cbidx[s], idx + e, mc * sizeof(int32_t));
      cbm[s] = mc;
      cbdel[s] = nfs - e;
      f->delayed += nfs - e;
    }
    free(F);
  }
  free(pos); free(cb); free(cbidx); free(cbm); free(cbdel); free(chead); free(cnext);
  out[0] = f->neg; out[1] = f->zero; out[2] = f->pos;
  out[3] = f->delayed; out[4] = f->twobytwo; out[5] = f->nullpiv;
  return f->valid;
}

/* Solve K X = B in place (B n x nrhs, column-major, leading dimension ldb, original ordering). */
int mf_solve(void *h, double *b, int64_t nrhs, int64_t ldb) {
  mf_t *f = h;
  const int64_t n = f->n;
  double *y = xmalloc(n * sizeof(double));
  for (int64_t r = 0; r < nrhs; ++r) {
    double *x = b + r * ldb;
    for (int64_t i = 0; i < n; ++i) y[i] = x[f->perm[i]] * f->scale[f->perm[i]];
    for (int32_t s = 0; s < f->ns; ++s) {
      const front_t *fr = &f->fronts[s];
      for (int64_t j = 0; j < fr->e; ++j) {
        if (fr->piv[j] == 0 || fr->piv[j] == 3) continue;
        if (fr->piv[j] == 1) {
          const double yj = y[fr->idx[j]];
          for (int64_t i = j + 1; i < fr->m; ++i) y[fr->idx[i]] -= fr->L[i + j * fr->m] * yj;
        } else {
          const double y0 = y[fr->idx[j]], y1 = y[fr->idx[j + 1]];
          for (int64_t i = j + 2; i < fr->m; ++i)
            y[fr->idx[i]] -= fr->L[i + j * fr->m] * y0 + fr->L[i + (j + 1) * fr->m] * y1;
        }
      }
    }
    for (int32_t s = 0; s < f->ns; ++s) {
      const front_t *fr = &f->fronts[s];
      for (int64_t j = 0; j < fr->e; ++j) {
        const int64_t m = fr->m;
        if (fr->piv[j] == 0) { y[fr->idx[j]] = 0.0; continue; }
        if (fr->piv[j] == 1) { y[fr->idx[j]] /= fr->L[j + j * m]; continue; }
        if (fr->piv[j] == 2) {
          const double a = fr->L[j + j * m], bb = fr->L[(j + 1) + j * m], c = fr->L[(j + 1) + (j + 1) * m];
          const double det = a * c - bb * bb;
          const double y0 = y[fr->idx[j]], y1 = y[fr->idx[j + 1]];
          y[fr->idx[j]] = (c * y0 - bb * y1) / det;
          y[fr->idx[j + 1]] = (-bb * y0 + a * y1) / det;
        }
      }
    }
    for (int32_t s = f->ns - 1; s >= 0; --s) {
      const front_t *fr = &f->fronts[s];
      for (int64_t j = fr->e - 1; j >= 0; --j) {
        if (fr->piv[j] == 0) continue;
        if (fr->piv[j] == 3) continue;
        const int64_t m = fr->m;
        if (fr->piv[j] == 1) {
          double acc = 0.0;
          for (int64_t i = j + 1; i < m; ++i) acc += fr->L[i + j * m] * y[fr->idx[i]];
          y[fr->idx[j]] -= acc;
        } else {
          double a0 = 0.0, a1 = 0.0;
          for (int64_t i = j + 2; i < m; ++i) {
            a0 += fr->L[i + j * m] * y[fr->idx[i]];
            a1 += fr->L[i + (j + 1) * m] * y[fr->idx[i]];
          }
          y[fr->idx[j]] -= a0;
          y[fr->idx[j + 1]] -= a1;
        }
      }
    }
    for (int64_t i = 0; i < n; ++i) x[f->perm[i]] = y[i] * f->scale[f->perm[i]];
  }
  free(y);
  return 0;
}

double mf_flops(void *h) { return ((mf_t *)h)->flops; }
int64_t mf_nnz_l(void *h) { return ((mf_t *)h)->nnz_l; }
int32_t mf_supernodes(void *h) { return ((mf_t *)h)->ns; }
void mf_order(void *h, int32_t *perm_out) { mf_t *f = h; memcpy(perm_out, f->perm, f->n * sizeof(int32_t)); }
int mf_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
