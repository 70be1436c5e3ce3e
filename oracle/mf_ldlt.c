/* ORACLE — test infrastructure only. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, as the checker; the product path never links or calls it.
 *
 * CPU restatement of the sparse symmetric-indefinite multifrontal LDL^T that hsolve obtains from
 * MUMPS 5.8.2 (SYM=2), following its documented behaviour, not its code:
 *   - symmetric iterative scaling of K (ICNTL(8)=7, hsolve src/factor/mumps_factorization.cpp:170-176),
 *     restated as Ruiz infinity-norm equilibration;
 *   - multifrontal elimination on the elimination tree of the given pivot order (PERM_IN), with
 *     fundamental supernodes (optionally amalgamated, as MUMPS amalgamates its tree); fronts of
 *     one tree height in parallel, the Schur updates of a front applied in blocks through BLAS;
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

static void relax_supernodes(mf_t *f);

/* Analyse: order (new -> old, NULL = natural), postorder the etree, fundamental supernodes;
 * relax != 0 then amalgamates them (relax_supernodes). */
void *mf_analyze_relaxed(int64_t n, const int64_t *rp, const int32_t *ci, const int32_t *order, int relax);

void *mf_analyze(int64_t n, const int64_t *rp, const int32_t *ci, const int32_t *order) {
  return mf_analyze_relaxed(n, rp, ci, order, 0);
}

void *mf_analyze_relaxed(int64_t n, const int64_t *rp, const int32_t *ci, const int32_t *order, int relax) {
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
  if (relax) relax_supernodes(f);
  f->fronts = xcalloc(f->ns, sizeof(front_t));
  return f;
}

/* Relaxed amalgamation: a supernode is merged into its parent when it is the parent's last child
 * (their columns are contiguous in the postorder) and the merged front stores few explicit zeros,
 * by the rule CHOLMOD uses (merge up to 4 columns always, up to 16 while zeros stay below 80 % of
 * the merged panel, up to 48 below 10 %, any size below 5 %). The merged front's rows are the
 * child's columns followed by the parent's rows (in the elimination tree the child's off-diagonal
 * structure lies inside the parent's). */
static void relax_supernodes(mf_t *f) {
  const int32_t ns = f->ns;
  int32_t *first = xmalloc(ns * sizeof(int32_t)), *last = xmalloc(ns * sizeof(int32_t));
  int32_t *rep = xmalloc(ns * sizeof(int32_t));
  int64_t *nrows = xmalloc(ns * sizeof(int64_t));
  double *zeros = xcalloc(ns, sizeof(double));
  for (int32_t s = 0; s < ns; ++s) {
    first[s] = f->sn_first[s];
    last[s] = f->sn_first[s + 1] - 1;
    rep[s] = s;
    nrows[s] = f->sn_rp[s + 1] - f->sn_rp[s];
  }
  for (int32_t s = 0; s < ns; ++s) {
    const int32_t p = f->sn_parent[s];
    if (p < 0 || last[s] + 1 != first[p]) continue;
    const int64_t ks = last[s] - first[s] + 1, kp = last[p] - first[p] + 1;
    const int64_t ds = nrows[p] - (nrows[s] - ks);  /* zeros added to every column of s */
    const int64_t km = ks + kp, mm = ks + nrows[p];
    const double entries = (double)km * (double)mm - 0.5 * (double)km * (double)(km - 1);
    const double z = zeros[s] + zeros[p] + (double)ks * (double)ds;
    const double frac = z / entries;
    if (km <= 4 || (km <= 16 && frac < 0.8) || (km <= 48 && frac < 0.1) || frac < 0.05) {
      first[p] = first[s];
      nrows[p] = mm;
      zeros[p] = z;
      rep[s] = p;
    }
  }
  /* representatives of the merged supernodes, and the new numbering (increasing first column) */
  int32_t *find = xmalloc(ns * sizeof(int32_t)), *newid = xmalloc(ns * sizeof(int32_t));
  for (int32_t s = ns - 1; s >= 0; --s) find[s] = rep[s] == s ? s : find[rep[s]];
  int32_t nn = 0;
  for (int32_t s = 0; s < ns; ++s) newid[s] = rep[s] == s ? nn++ : -1;
  int32_t *nfirst = xmalloc((nn + 1) * sizeof(int32_t)), *nparent = xmalloc((nn > 0 ? nn : 1) * sizeof(int32_t));
  int64_t *nrp = xmalloc((nn + 1) * sizeof(int64_t));
  nrp[0] = 0;
  for (int32_t s = 0; s < ns; ++s) {
    if (rep[s] != s) continue;
    const int32_t q = newid[s];
    nfirst[q] = first[s];
    nparent[q] = f->sn_parent[s] >= 0 ? newid[find[f->sn_parent[s]]] : -1;
    nrp[q + 1] = nrp[q] + nrows[s];
  }
  nfirst[nn] = (int32_t)f->n;
  int32_t *nrows_arr = xmalloc((nrp[nn] > 0 ? nrp[nn] : 1) * sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s) {
    if (rep[s] != s) continue;
    int32_t *out = nrows_arr + nrp[newid[s]];
    int64_t t = 0;
    for (int32_t c = first[s]; c < f->sn_first[s]; ++c) out[t++] = c;  /* absorbed columns */
    for (int64_t p = f->sn_rp[s]; p < f->sn_rp[s + 1]; ++p) out[t++] = f->sn_rows[p];
  }
  free(f->sn_first); free(f->sn_parent); free(f->sn_rp); free(f->sn_rows);
  f->ns = nn;
  f->sn_first = nfirst;
  f->sn_parent = nparent;
  f->sn_rp = nrp;
  f->sn_rows = nrows_arr;
  free(first); free(last); free(rep); free(nrows); free(zeros); free(find); free(newid);
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

/* ------------------------------------------------------------------------------ dense BLAS */

/* Fortran dgemm (C = alpha op(A) op(B) + beta C). The Python front end passes the dgemm of the
 * BLAS that numpy / scipy already load (scipy.linalg.cython_blas); without it a plain loop runs. */
typedef void (*dgemm_fn)(const char *, const char *, const int *, const int *, const int *, const double *,
                         const double *, const int *, const double *, const int *, const double *, double *,
                         const int *);
static dgemm_fn g_dgemm = NULL;
void mf_set_dgemm(void *fn) { g_dgemm = (dgemm_fn)fn; }

/* C (mr x nc, ld ldc) -= A (mr x k, ld lda) * B(nc x k, ld ldb)^T */
static void gemm_nt_sub(int64_t mr, int64_t nc, int64_t k, const double *A, int64_t lda, const double *B, int64_t ldb,
                        double *C, int64_t ldc) {
  if (mr <= 0 || nc <= 0 || k <= 0) return;
  if (g_dgemm) {
    const int M = (int)mr, N = (int)nc, K = (int)k, LA = (int)lda, LB = (int)ldb, LC = (int)ldc;
    const double one = 1.0, mone = -1.0;
    g_dgemm("N", "T", &M, &N, &K, &mone, A, &LA, B, &LB, &one, C, &LC);
    return;
  }
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t p = 0; p < k; ++p) {
      const double w = B[c + p * ldb];
      if (w == 0.0) continue;
      const double *a = A + p * lda;
      double *cc = C + c * ldc;
      for (int64_t i = 0; i < mr; ++i) cc[i] -= a[i] * w;
    }
}

/* -------------------------------------------------------------------- front factorization */

typedef struct {
  int64_t neg, zero, pos, twobytwo, nullpiv;
  int valid;
} counts_t;

typedef struct {
  double u, null_thr;
  int detect;
} piv_opts;

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

/* The front is factorized pivot by pivot with the decisions of the right-looking algorithm
 * (threshold 1x1 / 2x2 tests on up-to-date columns, failed candidates moved behind a shrinking limit
 * and retried after progress), but the Schur updates of the eliminated pivots are applied lazily:
 * the pivots [fb, j) are pending, a column is brought up to date only when it is examined, and the
 * trailing matrix receives all pending pivots at once (one matrix product) when kLazyMax pivots are
 * pending, before any symmetric swap, and at the end of the front. The pivot decisions therefore
 * read the same values as with immediate updates (up to the order of the floating-point sums). */
enum { kLazyMax = 64, kFlushCols = 128 };

typedef struct {
  double *F;
  int64_t m;
  int8_t *piv;
  int64_t fb;      /* first pending pivot */
  int64_t j;       /* next position */
  int cur_upd;     /* the current column (position j) holds the updates of [fb, j) */
  double *W;       /* m x kLazyMax: W = L D of the pending pivots */
  int inner;       /* parallelism inside the front */
} lazy_t;

/* W(c, p) for pending pivot p: 1x1 d L(c, p); 2x2 [a b; b e]: a L(c,p) + b L(c,p+1) for the first,
 * b L(c,p-1) + e L(c,p) for the second; null pivots have L = 0 */
static double w_entry(const lazy_t *z, int64_t c, int64_t p) {
  const double *F = z->F;
  const int64_t m = z->m;
  switch (z->piv[p]) {
    case 1: return F[p + p * m] * F[c + p * m];
    case 2: return F[p + p * m] * F[c + p * m] + F[(p + 1) + p * m] * F[c + (p + 1) * m];
    case 3: return F[p + (p - 1) * m] * F[c + (p - 1) * m] + F[p + p * m] * F[c + p * m];
    default: return 0.0;
  }
}

/* dst[i] = F[i, c] - sum_{p in [fb, j)} L(i, p) W(c, p) for rows i in [r0, m) (dst may be column c) */
static void updated_column(const lazy_t *z, int64_t c, int64_t r0, double *dst) {
  const int64_t m = z->m, np = z->j - z->fb;
  const double *F = z->F;
  double w[kLazyMax];
  for (int64_t q = 0; q < np; ++q) w[q] = w_entry(z, c, z->fb + q);
  if (dst != F + c * m)
    for (int64_t i = r0; i < m; ++i) dst[i] = F[i + c * m];
  const int64_t rows = m - r0;
#pragma omp parallel for schedule(static) if (z->inner && rows > 4096)
  for (int64_t i0 = r0; i0 < m; i0 += 1024) {
    const int64_t i1 = i0 + 1024 < m ? i0 + 1024 : m;
    for (int64_t q = 0; q < np; ++q) {
      const double wq = w[q];
      if (wq == 0.0) continue;
      const double *l = F + (z->fb + q) * m;
      for (int64_t i = i0; i < i1; ++i) dst[i] -= l[i] * wq;
    }
  }
}

/* entries (r, i) of row r for i in [j, r), brought up to date, into dst[i] */
static void updated_row(const lazy_t *z, int64_t r, double *dst) {
  const int64_t m = z->m, np = z->j - z->fb;
  const double *F = z->F;
  for (int64_t i = z->j; i < r; ++i) {
    double v = F[r + i * m];
    for (int64_t q = 0; q < np; ++q) v -= F[r + (z->fb + q) * m] * w_entry(z, i, z->fb + q);
    dst[i] = v;
  }
}

/* apply the pending pivots to every trailing column [j, m) not yet holding them; the current column
 * (position j) is skipped when it was brought up to date already */
static void flush(lazy_t *z) {
  const int64_t m = z->m, np = z->j - z->fb, j = z->j;
  if (np > 0 && j < m) {
    double *F = z->F, *W = z->W;
    for (int64_t q = 0; q < np; ++q) {
      const int64_t p = z->fb + q;
      for (int64_t c = j; c < m; ++c) W[c + q * m] = w_entry(z, c, p);
    }
    const int64_t c_start = z->cur_upd ? j + 1 : j;
    const int64_t nblk = (m - c_start + kFlushCols - 1) / kFlushCols;
#pragma omp parallel for schedule(dynamic) if (z->inner && nblk > 1)
    for (int64_t b = 0; b < nblk; ++b) {
      const int64_t c0 = c_start + b * kFlushCols;
      const int64_t c1 = c0 + kFlushCols < m ? c0 + kFlushCols : m;
      gemm_nt_sub(m - c0, c1 - c0, np, F + c0 + z->fb * m, m, W + c0, m, F + c0 + c0 * m, m);
    }
  }
  z->fb = z->j;
  z->cur_upd = 0;
}

/* the column at position j, up to date (in place) */
static void make_current(lazy_t *z) {
  if (z->cur_upd) return;
  updated_column(z, z->j, z->j, z->F + z->j * z->m);
  z->cur_upd = 1;
}

/* max |F(i, j)| over rows i > j of the up-to-date current column */
static double cur_col_max(const lazy_t *z) {
  const int64_t m = z->m, c = z->j;
  const double *col = z->F + c * m;
  double g = 0.0;
  for (int64_t i = c + 1; i < m; ++i) { double v = fabs(col[i]); if (v > g) g = v; }
  return g;
}

static void take1(lazy_t *z, counts_t *ct) {
  const int64_t j = z->j, m = z->m;
  double *F = z->F;
  z->piv[j] = 1;
  const double d = F[j + j * m];
  if (d < 0) ct->neg++; else ct->pos++;
  for (int64_t i = j + 1; i < m; ++i) F[i + j * m] /= d;
  z->j = j + 1;
  z->cur_upd = 0;
}

static void take2(lazy_t *z, counts_t *ct) {
  const int64_t j = z->j, m = z->m;
  double *F = z->F;
  z->piv[j] = 2; z->piv[j + 1] = 3; ct->twobytwo++;
  const double a2 = F[j + j * m], b2 = F[(j + 1) + j * m], c2 = F[(j + 1) + (j + 1) * m];
  const double d2 = a2 * c2 - b2 * b2;
  if (d2 < 0) { ct->neg++; ct->pos++; } else if (a2 + c2 < 0) ct->neg += 2; else ct->pos += 2;
  const double ia2 = c2 / d2, ib2 = -b2 / d2, ic2 = a2 / d2;
  for (int64_t i = j + 2; i < m; ++i) {
    const double x0 = F[i + j * m], x1 = F[i + (j + 1) * m];
    F[i + j * m] = ia2 * x0 + ib2 * x1;
    F[i + (j + 1) * m] = ib2 * x0 + ic2 * x1;
  }
  z->j = j + 2;
  z->cur_upd = 0;
}

static void take_null(lazy_t *z, counts_t *ct) {
  const int64_t j = z->j, m = z->m;
  z->piv[j] = 0; ct->zero++; ct->nullpiv++; ct->valid = 0;
  for (int64_t i = j + 1; i < m; ++i) z->F[i + j * m] = 0.0;
  z->j = j + 1;
  z->cur_upd = 0;
}

/* Partial LDL^T of front F (order m, fully summed nfs). Returns the eliminated count; the front's
 * positions [e, nfs) are delayed. root: no parent, pivots may not be delayed. tmp: 2m doubles,
 * W: m x kLazyMax doubles. */
static int64_t factor_front(counts_t *ct, double *F, int64_t m, int64_t nfs, int32_t *idx, int8_t *piv,
                            const piv_opts *o, int root, double *tmp, double *W, int inner) {
  lazy_t z = {F, m, piv, 0, 0, 0, W, inner};
  double *colr = tmp, *rowr = tmp + m;
  int64_t lim = nfs;
  int progress = 0;
  while (z.j < nfs) {
    if (z.j - z.fb + 2 > kLazyMax) flush(&z);
    const int64_t j = z.j;
    if (j >= lim) {
      if (progress) { lim = nfs; progress = 0; continue; }
      if (!root) break;
      /* root: nothing can be delayed; Bunch-Kaufman's choice on column j without threshold */
      flush(&z);
      make_current(&z);
      const double alpha = 0.6403882032022076;
      const double dcc = fabs(F[j + j * m]);
      const double gc = cur_col_max(&z);
      int64_t r = -1; double best = 0.0;
      for (int64_t i = j + 1; i < nfs; ++i) { double v = fabs(F[i + j * m]); if (v > best) { best = v; r = i; } }
      if (r < 0 || dcc >= alpha * gc) {
        if (F[j + j * m] == 0.0) take_null(&z, ct); else take1(&z, ct);
      } else {
        sym_swap(F, m, idx, j + 1, r);  /* everything is up to date after the flush above */
        take2(&z, ct);
      }
      lim = nfs;
      continue;
    }
    make_current(&z);
    const double dcc = fabs(F[j + j * m]);
    const double gc = cur_col_max(&z);
    if (o->detect && (dcc > gc ? dcc : gc) <= o->null_thr) { take_null(&z, ct); progress = 1; continue; }
    if (dcc >= o->u * gc && dcc > 0.0) { take1(&z, ct); progress = 1; continue; }
    /* candidate partner r among fully-summed rows (column j is up to date) */
    int64_t r = -1; double best = 0.0;
    for (int64_t i = j + 1; i < nfs; ++i) { double v = fabs(F[i + j * m]); if (v > best) { best = v; r = i; } }
    int decided = 0;
    if (r >= 0) {
      /* column r (rows >= r) and row r (entries (r, i), i in [j, r)) brought up to date aside */
      updated_column(&z, r, r, colr);
      updated_row(&z, r, rowr);
      double gc2 = 0.0, gr2 = 0.0, gr = 0.0;
      for (int64_t i = j + 1; i < m; ++i) if (i != r) { double v = fabs(F[i + j * m]); if (v > gc2) gc2 = v; }
      for (int64_t i = j; i < r; ++i) { double v = fabs(rowr[i]); if (v > gr) gr = v; if (i != j && v > gr2) gr2 = v; }
      for (int64_t i = r + 1; i < m; ++i) { double v = fabs(colr[i]); if (v > gr) gr = v; if (v > gr2) gr2 = v; }
      const double a = F[j + j * m], b = F[r + j * m], cc = colr[r];
      const double det = a * cc - b * b;
      if (det != 0.0) {
        const double ia = fabs(cc / det), ib = fabs(b / det), ic = fabs(a / det);
        if (ia * gc2 + ib * gr2 <= 1.0 / o->u && ib * gc2 + ic * gr2 <= 1.0 / o->u) {
          flush(&z);
          sym_swap(F, m, idx, j + 1, r);
          if (lim == j + 1) lim = j + 2;  /* the partner came from behind the limit */
          take2(&z, ct);
          progress = 1; if (lim < z.j) lim = z.j;
          decided = 1;
        }
      }
      if (!decided) {
        const double drr = fabs(cc);
        if (drr >= o->u * gr && drr > 0.0) {
          flush(&z);
          sym_swap(F, m, idx, j, r);
          z.cur_upd = 1;  /* position j now holds column r, up to date after the flush */
          take1(&z, ct);
          progress = 1; if (lim < z.j) lim = z.j;
          decided = 1;
        }
      }
    }
    if (decided) continue;
    /* column j fails: move it behind the limit */
    flush(&z);
    lim--;
    sym_swap(F, m, idx, j, lim);
  }
  flush(&z);
  return z.j;
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

/* supernodes grouped by height in the assembly tree (leaves 0): lptr[l]..lptr[l+1] index lsn */
static void sn_levels(const mf_t *f, int32_t *nlev, int32_t **lptr, int32_t **lsn) {
  const int32_t ns = f->ns;
  int32_t *level = xcalloc(ns > 0 ? ns : 1, sizeof(int32_t));
  int32_t L = 0;
  for (int32_t s = 0; s < ns; ++s) {  /* children precede parents (postorder) */
    const int32_t p = f->sn_parent[s];
    if (p >= 0 && level[p] < level[s] + 1) level[p] = level[s] + 1;
    if (level[s] + 1 > L) L = level[s] + 1;
  }
  int32_t *ptr = xcalloc(L + 1, sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s) ptr[level[s] + 1]++;
  for (int32_t l = 0; l < L; ++l) ptr[l + 1] += ptr[l];
  int32_t *fill = xmalloc((L + 1) * sizeof(int32_t));
  memcpy(fill, ptr, (L + 1) * sizeof(int32_t));
  int32_t *out = xmalloc((ns > 0 ? ns : 1) * sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s) out[fill[level[s]]++] = s;
  free(fill);
  free(level);
  *nlev = L; *lptr = ptr; *lsn = out;
}

static int max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static int thread_id(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

/* Numeric factorization of the symmetric matrix given by its upper CSR (same pattern as
 * analysed) with values v. Returns 1 if valid (no null pivot), 0 otherwise; inertia in out[0..2],
 * delayed pivots, 2x2 pivots and null pivots in out[3..5]. Fronts of one height in the tree are
 * factorized in parallel; a level with few fronts runs them one after another, each with parallel
 * updates. */
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
  const int nt = max_threads();
  int32_t **pos = xmalloc(nt * sizeof(int32_t *));
  for (int t = 0; t < nt; ++t) {
    pos[t] = xmalloc(n * sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) pos[t][i] = -1;
  }
  /* contribution blocks of finished fronts, waiting for their parent */
  double **cb = xcalloc(f->ns, sizeof(double *));
  int32_t **cbidx = xcalloc(f->ns, sizeof(int32_t *));
  int64_t *cbm = xcalloc(f->ns, sizeof(int64_t));
  int64_t *cbdel = xcalloc(f->ns, sizeof(int64_t));
  int32_t *chead = xmalloc(f->ns * sizeof(int32_t)), *cnext = xmalloc(f->ns * sizeof(int32_t));
  for (int32_t s = 0; s < f->ns; ++s) chead[s] = -1;
  for (int32_t s = f->ns - 1; s >= 0; --s)
    if (f->sn_parent[s] >= 0) { cnext[s] = chead[f->sn_parent[s]]; chead[f->sn_parent[s]] = s; }
  int32_t nlev = 0, *lptr = NULL, *lsn = NULL;
  sn_levels(f, &nlev, &lptr, &lsn);
  for (int32_t l = 0; l < nlev; ++l) {
    const int32_t cnt = lptr[l + 1] - lptr[l];
    const int outer = cnt >= 2 * nt;
#pragma omp parallel for schedule(dynamic, 1) if (outer)
    for (int32_t q = lptr[l]; q < lptr[l + 1]; ++q) {
      const int32_t s = lsn[q];
      int32_t *ps = pos[outer ? thread_id() : 0];
      const int64_t k = f->sn_first[s + 1] - f->sn_first[s];
      const int64_t nr = f->sn_rp[s + 1] - f->sn_rp[s];
      const int32_t *rows = f->sn_rows + f->sn_rp[s];
      int64_t nd = 0;
      for (int32_t c = chead[s]; c != -1; c = cnext[c]) nd += cbdel[c];
      const int64_t m = nr + nd, nfs = k + nd;
      int32_t *idx = xmalloc(m * sizeof(int32_t));
      int64_t t = 0;
      for (int64_t qq = 0; qq < k; ++qq) idx[t++] = rows[qq];
      for (int32_t c = chead[s]; c != -1; c = cnext[c])
        for (int64_t qq = 0; qq < cbdel[c]; ++qq) idx[t++] = cbidx[c][qq];
      for (int64_t qq = k; qq < nr; ++qq) idx[t++] = rows[qq];
      for (int64_t qq = 0; qq < m; ++qq) ps[idx[qq]] = (int32_t)qq;
      double *F = xcalloc(m * m, sizeof(double));
      for (int64_t j = f->sn_first[s]; j < f->sn_first[s + 1]; ++j)
        for (int64_t p = f->lp[j]; p < f->lp[j + 1]; ++p) {
          const int32_t i = f->li[p];
          const int64_t src = f->lsrc[p];
          const double val = v[src] * f->scale[f->perm[i]] * f->scale[f->perm[j]];
          int64_t a = ps[i], b = ps[j];
          if (a < b) { int64_t tt = a; a = b; b = tt; }
          F[a + b * m] += val;
        }
      for (int32_t c = chead[s]; c != -1; c = cnext[c]) {
        const int64_t mc = cbm[c];
        for (int64_t bb = 0; bb < mc; ++bb) {
          const int64_t pb = ps[cbidx[c][bb]];
          for (int64_t aa = bb; aa < mc; ++aa) {
            int64_t pa = ps[cbidx[c][aa]], pc = pb;
            if (pa < pc) { int64_t tt = pa; pa = pc; pc = tt; }
            F[pa + pc * m] += cb[c][aa + bb * mc];
          }
        }
        free(cb[c]); free(cbidx[c]); cb[c] = NULL; cbidx[c] = NULL;
      }
      for (int64_t qq = 0; qq < m; ++qq) ps[idx[qq]] = -1;
      int8_t *piv = xcalloc(nfs > 0 ? nfs : 1, 1);
      const int root = f->sn_parent[s] < 0;
      counts_t ct = {0, 0, 0, 0, 0, 1};
      double *tmp = xmalloc((2 * m + (int64_t)kLazyMax * m) * sizeof(double));
      const int64_t e = factor_front(&ct, F, m, nfs, idx, piv, &o, root, tmp, tmp + 2 * m, !outer);
      free(tmp);
      double fl = 0.0;
      for (int64_t jj = 0; jj < e; ++jj) {
        const double r = (double)(m - jj - 1);
        fl += r + r * (r + 1.0);
      }
      /* keep L (m x e) and the contribution block (positions e..m-1) */
      front_t *fr = &f->fronts[s];
      fr->m = m; fr->e = e; fr->idx = idx; fr->piv = piv;
      fr->L = xmalloc((e > 0 ? e : 1) * m * sizeof(double));
      memcpy(fr->L, F, e * m * sizeof(double));
      const int64_t mc = m - e;
      int64_t dl = 0;
      if (mc > 0 && !root) {
        cb[s] = xmalloc(mc * mc * sizeof(double));
        for (int64_t bb = 0; bb < mc; ++bb)
          for (int64_t aa = bb; aa < mc; ++aa) cb[s][aa + bb * mc] = F[(e + aa) + (e + bb) * m];
        cbidx[s] = xmalloc(mc * sizeof(int32_t));
        memcpy(cbidx[s], idx + e, mc * sizeof(int32_t));
        cbm[s] = mc;
        cbdel[s] = nfs - e;
        dl = nfs - e;
      }
      free(F);
#pragma omp critical(mf_counts)
      {
        f->neg += ct.neg; f->zero += ct.zero; f->pos += ct.pos; f->twobytwo += ct.twobytwo;
        f->nullpiv += ct.nullpiv; if (!ct.valid) f->valid = 0;
        f->flops += fl;
        f->nnz_l += e * m - e * (e - 1) / 2;
        f->delayed += dl;
      }
    }
  }
  for (int t = 0; t < nt; ++t) free(pos[t]);
  free(pos); free(cb); free(cbidx); free(cbm); free(cbdel); free(chead); free(cnext);
  free(lptr); free(lsn);
  out[0] = f->neg; out[1] = f->zero; out[2] = f->pos;
  out[3] = f->delayed; out[4] = f->twobytwo; out[5] = f->nullpiv;
  return f->valid;
}

/* ---------------------------------------------------------------------------------- solve */

/* Solve K X = B in place (B n x nrhs, column-major, leading dimension ldb, original ordering).
 * Forward: fronts by height, in parallel; a front gathers its pivot entries and its children's
 * contribution vectors, eliminates its pivots and leaves -L21 z (plus the children's entries for its
 * non-pivot rows) as its own contribution vector. Diagonal: D y = z. Backward: fronts from the top,
 * in parallel by height; a front reads its ancestors' final entries and writes its own pivots. A
 * front's work vector is row-major (t[i * nrhs + r]), so every L entry is read once per sweep. */
int mf_solve(void *h, double *b, int64_t nrhs, int64_t ldb) {
  mf_t *f = h;
  const int64_t n = f->n;
  const int32_t ns = f->ns;
  const int nt = max_threads();
  int32_t nlev = 0, *lptr = NULL, *lsn = NULL;
  sn_levels(f, &nlev, &lptr, &lsn);
  int32_t *chead = xmalloc((ns > 0 ? ns : 1) * sizeof(int32_t)), *cnext = xmalloc((ns > 0 ? ns : 1) * sizeof(int32_t));
  for (int32_t s = 0; s < ns; ++s) chead[s] = -1;
  for (int32_t s = ns - 1; s >= 0; --s)
    if (f->sn_parent[s] >= 0) { cnext[s] = chead[f->sn_parent[s]]; chead[f->sn_parent[s]] = s; }
  int32_t **pos = xmalloc(nt * sizeof(int32_t *));
  for (int t = 0; t < nt; ++t) {
    pos[t] = xmalloc(n * sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) pos[t][i] = -1;
  }
  double **cv = xcalloc(ns > 0 ? ns : 1, sizeof(double *));  /* contribution vectors, (m - e) x nrhs */
  double *y = xmalloc((n > 0 ? n : 1) * nrhs * sizeof(double));
  for (int64_t r = 0; r < nrhs; ++r)
    for (int64_t i = 0; i < n; ++i) y[i + r * n] = b[f->perm[i] + r * ldb] * f->scale[f->perm[i]];
  /* forward */
  for (int32_t l = 0; l < nlev; ++l) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t q = lptr[l]; q < lptr[l + 1]; ++q) {
      const int32_t s = lsn[q];
      const front_t *fr = &f->fronts[s];
      const int64_t m = fr->m, e = fr->e;
      int32_t *ps = pos[thread_id()];
      double *t = xmalloc((m > 0 ? m : 1) * nrhs * sizeof(double));
      for (int64_t i = 0; i < m; ++i) ps[fr->idx[i]] = (int32_t)i;
      for (int64_t i = 0; i < m; ++i)
        for (int64_t r = 0; r < nrhs; ++r) t[i * nrhs + r] = i < e ? y[fr->idx[i] + r * n] : 0.0;
      for (int32_t c = chead[s]; c != -1; c = cnext[c]) {
        const front_t *fc = &f->fronts[c];
        const int64_t mc = fc->m - fc->e;
        for (int64_t a = 0; a < mc; ++a) {
          double *ta = t + (int64_t)ps[fc->idx[fc->e + a]] * nrhs;
          const double *ca = cv[c] + a * nrhs;
          for (int64_t r = 0; r < nrhs; ++r) ta[r] += ca[r];
        }
        free(cv[c]);
        cv[c] = NULL;
      }
      for (int64_t i = 0; i < m; ++i) ps[fr->idx[i]] = -1;
      for (int64_t j = 0; j < e; ++j) {
        if (fr->piv[j] == 0 || fr->piv[j] == 3) continue;
        const double *l0 = fr->L + j * m;
        if (fr->piv[j] == 1) {
          const double *yj = t + j * nrhs;
          for (int64_t i = j + 1; i < m; ++i) {
            const double li = l0[i];
            double *ti = t + i * nrhs;
            for (int64_t r = 0; r < nrhs; ++r) ti[r] -= li * yj[r];
          }
        } else {
          const double *l1 = l0 + m;
          const double *y0 = t + j * nrhs, *y1 = t + (j + 1) * nrhs;
          for (int64_t i = j + 2; i < m; ++i) {
            const double a0 = l0[i], a1 = l1[i];
            double *ti = t + i * nrhs;
            for (int64_t r = 0; r < nrhs; ++r) ti[r] -= a0 * y0[r] + a1 * y1[r];
          }
        }
      }
      for (int64_t i = 0; i < e; ++i)
        for (int64_t r = 0; r < nrhs; ++r) y[fr->idx[i] + r * n] = t[i * nrhs + r];
      const int64_t mc = m - e;
      if (mc > 0 && f->sn_parent[s] >= 0) {
        cv[s] = xmalloc(mc * nrhs * sizeof(double));
        memcpy(cv[s], t + e * nrhs, mc * nrhs * sizeof(double));
      }
      free(t);
    }
  }
  /* diagonal */
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t s = 0; s < ns; ++s) {
    const front_t *fr = &f->fronts[s];
    const int64_t m = fr->m;
    for (int64_t j = 0; j < fr->e; ++j)
      for (int64_t r = 0; r < nrhs; ++r) {
        double *yr = y + r * n;
        if (fr->piv[j] == 0) { yr[fr->idx[j]] = 0.0; continue; }
        if (fr->piv[j] == 1) { yr[fr->idx[j]] /= fr->L[j + j * m]; continue; }
        if (fr->piv[j] == 2) {
          const double a = fr->L[j + j * m], bb = fr->L[(j + 1) + j * m], c = fr->L[(j + 1) + (j + 1) * m];
          const double det = a * c - bb * bb;
          const double y0 = yr[fr->idx[j]], y1 = yr[fr->idx[j + 1]];
          yr[fr->idx[j]] = (c * y0 - bb * y1) / det;
          yr[fr->idx[j + 1]] = (-bb * y0 + a * y1) / det;
        }
      }
  }
  /* backward */
  for (int32_t l = nlev - 1; l >= 0; --l) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t q = lptr[l]; q < lptr[l + 1]; ++q) {
      const front_t *fr = &f->fronts[lsn[q]];
      const int64_t m = fr->m, e = fr->e;
      double *t = xmalloc((m > 0 ? m : 1) * nrhs * sizeof(double));
      for (int64_t i = 0; i < m; ++i)
        for (int64_t r = 0; r < nrhs; ++r) t[i * nrhs + r] = y[fr->idx[i] + r * n];
      double acc0[16], acc1[16];
      for (int64_t j = e - 1; j >= 0; --j) {
        if (fr->piv[j] == 0 || fr->piv[j] == 3) continue;
        const double *l0 = fr->L + j * m;
        for (int64_t r0 = 0; r0 < nrhs; r0 += 16) {
          const int64_t rr = nrhs - r0 < 16 ? nrhs - r0 : 16;
          for (int64_t r = 0; r < rr; ++r) { acc0[r] = 0.0; acc1[r] = 0.0; }
          if (fr->piv[j] == 1) {
            for (int64_t i = j + 1; i < m; ++i) {
              const double li = l0[i];
              const double *ti = t + i * nrhs + r0;
              for (int64_t r = 0; r < rr; ++r) acc0[r] += li * ti[r];
            }
            for (int64_t r = 0; r < rr; ++r) t[j * nrhs + r0 + r] -= acc0[r];
          } else {
            const double *l1 = l0 + m;
            for (int64_t i = j + 2; i < m; ++i) {
              const double a0 = l0[i], a1 = l1[i];
              const double *ti = t + i * nrhs + r0;
              for (int64_t r = 0; r < rr; ++r) { acc0[r] += a0 * ti[r]; acc1[r] += a1 * ti[r]; }
            }
            for (int64_t r = 0; r < rr; ++r) {
              t[j * nrhs + r0 + r] -= acc0[r];
              t[(j + 1) * nrhs + r0 + r] -= acc1[r];
            }
          }
        }
      }
      for (int64_t i = 0; i < e; ++i)
        for (int64_t r = 0; r < nrhs; ++r) y[fr->idx[i] + r * n] = t[i * nrhs + r];
      free(t);
    }
  }
  for (int64_t r = 0; r < nrhs; ++r)
    for (int64_t i = 0; i < n; ++i) b[f->perm[i] + r * ldb] = y[i + r * n] * f->scale[f->perm[i]];
  for (int t = 0; t < nt; ++t) free(pos[t]);
  free(pos); free(cv); free(y); free(lptr); free(lsn); free(chead); free(cnext);
  return 0;
}

double mf_flops(void *h) { return ((mf_t *)h)->flops; }
int64_t mf_nnz_l(void *h) { return ((mf_t *)h)->nnz_l; }
int32_t mf_supernodes(void *h) { return ((mf_t *)h)->ns; }
void mf_order(void *h, int32_t *perm_out) { mf_t *f = h; memcpy(perm_out, f->perm, f->n * sizeof(int32_t)); }
int mf_threads(void) { return max_threads(); }
