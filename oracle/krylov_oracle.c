/* CPU oracle for the solver_cpp Krylov hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Single-threaded restatement of the reference's host path. Each routine cites
 * the reference file:line it follows and performs the same floating point
 * operations in the same order as the reference built with -O2 (no FMA
 * contraction) and run with -t 1. Only tests/, the smoke check and the CPU
 * baseline leg of the benchmark may load it; the product never does.
 */
#include "krylov_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* blas.cpp primitives                                                       */
/* ------------------------------------------------------------------------ */

/* blas::MtxVec_mult (blas.cpp:43-65): row-sequential sum from 0.0. */
static void csr_mv(long n, const int *ptr, const int *col, const double *val,
                   const double *x, double *y) {
  for (long i = 0; i < n; i++) {
    double t = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) t += val[j] * x[col[j]];
    y[i] = t;
  }
}

void oracle_spmv(const or_mat *A, const double *x, double *y) {
  csr_mv(A->n, A->ptr, A->col, A->val, x, y);
}

/* blas::MtxVec_mult(Tval,Tcol,Tptr,...) (blas.cpp:112-129). */
void oracle_spmv_t(const or_mat *A, const double *x, double *y) {
  csr_mv(A->n, A->tptr, A->tcol, A->tval, x, y);
}

/* Number of partial sums of dot/norm_2 for the solve in progress (see
 * or_params.sum_chunks). The oracle is single-threaded test code. */
static int g_sum_chunks = 1;

/* Pairwise (recursive halving) sum of x[i]*y[i], runs of 8 summed in
 * order: the accuracy class of a parallel tree reduction. */
static double pair_dot(long n, const double *x, const double *y) {
  if (n <= 8) {
    double t = 0.0;
    for (long i = 0; i < n; i++) t += x[i] * y[i];
    return t;
  }
  const long h = n / 2;
  return pair_dot(h, x, y) + pair_dot(n - h, x + h, y + h);
}

/* blas::dot (blas.cpp:149-162). With g_sum_chunks = T > 1 the index range is
 * split as OpenMP schedule(static) splits it over T threads (the first n % T
 * threads take one extra element), each part summed from 0.0 in order and
 * the parts added in thread order. g_sum_chunks = -1: pairwise summation. */
double oracle_dot(long n, const double *x, const double *y) {
  if (g_sum_chunks == -1 || g_sum_chunks == -2) return pair_dot(n, x, y);
  if (g_sum_chunks <= 1) {
    double t = 0.0;
    for (long i = 0; i < n; i++) t += x[i] * y[i];
    return t;
  }
  const long T = g_sum_chunks, q = n / T, rem = n % T;
  double total = 0.0;
  long s = 0;
  for (long c = 0; c < T; c++) {
    const long len = q + (c < rem ? 1 : 0);
    double t = 0.0;
    for (long i = s; i < s + len; i++) t += x[i] * y[i];
    total += t;
    s += len;
  }
  return total;
}

/* A dot product the reference always sums sequentially: the ones inside
 * Gcr_sp_1's parallel loop (blas.cpp:529-535) run as nested, one-thread
 * regions. */
static double seq_dot(long n, const double *x, const double *y) {
  if (g_sum_chunks == -2) return pair_dot(n, x, y);
  double t = 0.0;
  for (long i = 0; i < n; i++) t += x[i] * y[i];
  return t;
}

/* blas::norm_2 (blas.cpp:31-41). */
double oracle_norm2(long n, const double *x) {
  return sqrt(oracle_dot(n, x, x));
}

/* Scalar_axy (blas.cpp:226-233): out = (a*x) + y. */
static void axy(long n, double a, const double *x, const double *y,
                double *out) {
  for (long i = 0; i < n; i++) out[i] = (a * x[i]) + y[i];
}

/* Vec_sub (blas.cpp:132-136). */
static void vsub(long n, const double *x, const double *y, double *out) {
  for (long i = 0; i < n; i++) out[i] = x[i] - y[i];
}

/* Vec_add (blas.cpp:138-142). */
static void vadd(long n, const double *x, const double *y, double *out) {
  for (long i = 0; i < n; i++) out[i] = x[i] + y[i];
}

/* Scalar_x_div_a (blas.cpp:257-264). */
static void xdiva(long n, const double *x, double a, double *out) {
  for (long i = 0; i < n; i++) out[i] = x[i] / a;
}

/* Scalar_ax (blas.cpp:217-224): out = a*x (overwrites). */
static void ax(long n, double a, const double *x, double *out) {
  for (long i = 0; i < n; i++) out[i] = a * x[i];
}

/* CSR -> CSC by a stable counting sort; same layout as cuSPARSE csr2csc
 * (cudaFunction.cu:933-982): rows ascend inside each column. */
void oracle_csr_transpose(long n, long nnz, const int *ptr, const int *col,
                          const double *val, int *tptr, int *trow,
                          double *tval) {
  long *cnt = (long *)calloc((size_t)n + 1, sizeof(long));
  for (long j = 0; j < nnz; j++) cnt[col[j] + 1]++;
  for (long c = 0; c < n; c++) cnt[c + 1] += cnt[c];
  for (long c = 0; c <= n; c++) tptr[c] = (int)cnt[c];
  for (long r = 0; r < n; r++)
    for (int j = ptr[r]; j < ptr[r + 1]; j++) {
      long d = cnt[col[j]]++;
      trow[d] = (int)r;
      tval[d] = val[j];
    }
  free(cnt);
}

/* blas::Kskip_cg_bicg_base (blas.cpp:353-399): Ar[i] = A^{i+1} r for
 * i <= 2k, Ap[i] = A^{i+1} p for i <= 2k+1; vectors stored contiguously. */
void oracle_matpow(const or_mat *A, const double *r, const double *p, int k,
                   double *Ar, double *Ap) {
  long n = A->n;
  csr_mv(n, A->ptr, A->col, A->val, r, Ar);
  csr_mv(n, A->ptr, A->col, A->val, p, Ap);
  for (int ii = 1; ii < 2 * k + 2; ii++) {
    if (ii < 2 * k + 1)
      csr_mv(n, A->ptr, A->col, A->val, Ar + (long)(ii - 1) * n,
             Ar + (long)ii * n);
    csr_mv(n, A->ptr, A->col, A->val, Ap + (long)(ii - 1) * n,
           Ap + (long)ii * n);
  }
}

/* blas::Kskip_cg_innerProduce (blas.cpp:401-435). */
void oracle_gram_cg(long n, int k, const double *Ar, const double *Ap,
                    const double *r, const double *p, double *delta,
                    double *eta, double *zeta) {
  if (g_sum_chunks == -2) {  /* every Gram value summed pairwise */
    for (int i = 0; i < 2 * k + 2; i++) {
      if (i < 2 * k) delta[i] = pair_dot(n, r, Ar + (long)i * n);
      if (i < 2 * k + 1) eta[i] = pair_dot(n, r, Ap + (long)i * n);
      zeta[i] = pair_dot(n, p, Ap + (long)i * n);
    }
    return;
  }
  for (int i = 0; i < 2 * k + 2; i++) {
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (long j = 0; j < n; j++) {
      if (i < 2 * k) t1 += r[j] * Ar[(long)i * n + j];
      if (i < 2 * k + 1) t2 += r[j] * Ap[(long)i * n + j];
      t3 += p[j] * Ap[(long)i * n + j];
    }
    if (i < 2 * k) delta[i] = t1;
    if (i < 2 * k + 1) eta[i] = t2;
    zeta[i] = t3;
  }
}

/* blas::Kskip_bicg_innerProduce (blas.cpp:437-475). */
void oracle_gram_bicg(long n, int k, const double *Ar, const double *Ap,
                      const double *rs, const double *ps, double *theta,
                      double *eta, double *rho, double *phi) {
  if (g_sum_chunks == -2) {  /* every Gram value summed pairwise */
    for (int i = 0; i < 2 * k + 2; i++) {
      if (i < 2 * k) theta[i] = pair_dot(n, rs, Ar + (long)i * n);
      if (i < 2 * k + 1) {
        eta[i] = pair_dot(n, rs, Ap + (long)i * n);
        rho[i] = pair_dot(n, ps, Ar + (long)i * n);
      }
      phi[i] = pair_dot(n, ps, Ap + (long)i * n);
    }
    return;
  }
  for (int i = 0; i < 2 * k + 2; i++) {
    double t1 = 0.0, t2 = 0.0, t3 = 0.0, t4 = 0.0;
    for (long j = 0; j < n; j++) {
      if (i < 2 * k) t1 += rs[j] * Ar[(long)i * n + j];
      if (i < 2 * k + 1) {
        t2 += rs[j] * Ap[(long)i * n + j];
        t3 += ps[j] * Ar[(long)i * n + j];
      }
      t4 += ps[j] * Ap[(long)i * n + j];
    }
    if (i < 2 * k) theta[i] = t1;
    if (i < 2 * k + 1) {
      eta[i] = t2;
      rho[i] = t3;
    }
    phi[i] = t4;
  }
}

/* blas::Check_error (blas.cpp:266-301). */
double oracle_check_error(const or_mat *A, const double *b, const double *x,
                          const double *x0) {
  long n = A->n;
  double *e1 = (double *)malloc(sizeof(double) * (size_t)n);
  double *e0 = (double *)malloc(sizeof(double) * (size_t)n);
  for (long i = 0; i < n; i++) {
    double t1 = 0.0, t2 = 0.0;
    for (int j = A->ptr[i]; j < A->ptr[i + 1]; j++) {
      t1 += A->val[j] * x[A->col[j]];
      t2 += A->val[j] * x0[A->col[j]];
    }
    e1[i] = b[i] - t1;
    e0[i] = b[i] - t2;
  }
  double r = log10(oracle_norm2(n, e1) / oracle_norm2(n, e0));
  free(e1);
  free(e0);
  return r;
}

void oracle_pattern_grad(const or_mat *A, const double *lambda,
                         const double *x, double *grad_val) {
  for (long i = 0; i < A->n; i++)
    for (int j = A->ptr[i]; j < A->ptr[i + 1]; j++)
      grad_val[j] = -lambda[i] * x[A->col[j]];
}

/* blas::Hye (blas.cpp:303-314), H stored row-major with row stride ld. */
static void hye(const double *h, long ld, double *y, const double *e,
                long size) {
  for (long i = 0; i < size; i++) y[i] = 0.0;
  for (long i = size - 1; i >= 0; i--) {
    double t = 0.0;
    for (long j = i + 1; j < size; j++) t += y[j] * h[i * ld + j];
    y[i] = (e[i] - t) / h[i * ld + i];
  }
}

/* ------------------------------------------------------------------------ */
/* Solver context                                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  long *it;
  double *err;
  long cap, len;
} hist_t;

typedef struct {
  const or_mat *A;
  const or_params *p;
  long spmv;
  int is_vp;
} ctx_t;

static void H(hist_t *h, long it, double err) {
  if (!h) return;
  if (h->len < h->cap) {
    h->it[h->len] = it;
    h->err[h->len] = err;
  }
  h->len++;
}

static void MV(ctx_t *c, const double *x, double *y) {
  c->spmv++;
  csr_mv(c->A->n, c->A->ptr, c->A->col, c->A->val, x, y);
}

static void MVT(ctx_t *c, const double *x, double *y) {
  c->spmv++;
  csr_mv(c->A->n, c->A->tptr, c->A->tcol, c->A->tval, x, y);
}

static double *vnew(long n) {
  return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
}

/* Parameters a solver instance uses: inner ones only for an inner solve of a
 * VP method (e.g. cg.cpp:68-74). */
typedef struct {
  long maxloop, restart;
  double eps;
  int kskip, fix;
} sp_t;

static sp_t params_for(const ctx_t *c, int inner) {
  sp_t s;
  if (c->is_vp && inner) {
    s.maxloop = c->p->inner_maxloop;
    s.eps = c->p->inner_eps;
    s.restart = c->p->inner_restart;
    s.kskip = c->p->inner_kskip;
    s.fix = c->p->inner_fix;
  } else {
    s.maxloop = c->p->outer_maxloop;
    s.eps = c->p->outer_eps;
    s.restart = c->p->outer_restart;
    s.kskip = c->p->outer_kskip;
    s.fix = c->p->outer_fix;
  }
  return s;
}

typedef struct {
  int status;
  long loop;
} res_t;

/* ------------------------------------------------------------------------ */
/* Plain Krylov methods                                                      */
/* ------------------------------------------------------------------------ */

/* cg::solve (cg.cpp:148-240). */
static res_t solve_cg(ctx_t *c, const double *b, double *x, int inner,
                      hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  double *r = vnew(n), *p = vnew(n), *mv = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  MV(c, x, mv);
  vsub(n, b, mv, r);
  memcpy(p, r, sizeof(double) * (size_t)n);
  double rr = oracle_dot(n, r, r);
  long loop;
  for (loop = 1; loop <= s.maxloop; loop++) {
    double err = oracle_norm2(n, r) / bnorm;
    if (!inner) H(h, loop, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    MV(c, p, mv);
    double d = oracle_dot(n, p, mv);
    double alpha = rr / d;
    axy(n, alpha, p, x, x);
    axy(n, -alpha, mv, r, r);
    double rr2 = oracle_dot(n, r, r);
    double beta = rr2 / rr;
    rr = rr2;
    axy(n, beta, p, r, p);
  }
  res.loop = loop;
  free(r);
  free(p);
  free(mv);
  return res;
}

/* cr::solve (cr.cpp:152-263). */
static res_t solve_cr(ctx_t *c, const double *b, double *x, int inner,
                      hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  double *r = vnew(n), *p = vnew(n), *q = vnew(n), *sv = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  MV(c, x, q);
  vsub(n, b, q, r);
  memcpy(p, r, sizeof(double) * (size_t)n);
  MV(c, p, q);
  memcpy(sv, q, sizeof(double) * (size_t)n);
  double rs = oracle_dot(n, r, sv);
  long loop;
  for (loop = 1; loop <= s.maxloop; loop++) {
    double err = oracle_norm2(n, r) / bnorm;
    if (!inner) H(h, loop, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    double d = oracle_dot(n, q, q);
    double alpha = rs / d;
    axy(n, alpha, p, x, x);
    axy(n, -alpha, q, r, r);
    MV(c, r, sv);
    double rs2 = oracle_dot(n, r, sv);
    double beta = rs2 / rs;
    rs = rs2;
    axy(n, beta, p, r, p);
    axy(n, beta, q, sv, q);
  }
  res.loop = loop;
  free(r);
  free(p);
  free(q);
  free(sv);
  return res;
}

/* bicg::solve (bicg.cpp:162-277). */
static res_t solve_bicg(ctx_t *c, const double *b, double *x, int inner,
                        hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  double *r = vnew(n), *rs = vnew(n), *p = vnew(n), *ps = vnew(n),
         *mv = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  MV(c, x, mv);
  vsub(n, b, mv, r);
  memcpy(rs, r, sizeof(double) * (size_t)n);
  memcpy(p, r, sizeof(double) * (size_t)n);
  memcpy(ps, rs, sizeof(double) * (size_t)n);
  double rr = oracle_dot(n, rs, r);
  long loop;
  for (loop = 1; loop <= s.maxloop; loop++) {
    double err = oracle_norm2(n, r) / bnorm;
    if (!inner) H(h, loop, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    MV(c, p, mv);
    double d = oracle_dot(n, ps, mv);
    double alpha = rr / d;
    axy(n, alpha, p, x, x);
    axy(n, -alpha, mv, r, r);
    MVT(c, ps, mv);
    axy(n, -alpha, mv, rs, rs);
    double rr2 = oracle_dot(n, rs, r);
    double beta = rr2 / rr;
    rr = rr2;
    axy(n, beta, p, r, p);
    axy(n, beta, ps, rs, ps);
  }
  res.loop = loop;
  free(r);
  free(rs);
  free(p);
  free(ps);
  free(mv);
  return res;
}

/* gcr::solve (gcr.cpp:178-317); orthogonalisation is blas::Gcr_sp_1
 * (blas.cpp:526-543). P and Q hold `restart` vectors. */
static res_t solve_gcr(ctx_t *c, const double *b, double *x, int inner,
                       hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  long m = s.restart;
  double *r = vnew(n), *Av = vnew(n);
  double *P = vnew(n * m), *Q = vnew(n * m);
  double *qq = vnew(m), *beta = vnew(m);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  long loop = 1;
  int out = 0;
  while (loop < s.maxloop) {
    MV(c, x, Av);
    vsub(n, b, Av, r);
    memcpy(P, r, sizeof(double) * (size_t)n);
    MV(c, P, Q);
    for (long k = 0; k < m; k++) {
      double err = oracle_norm2(n, r) / bnorm;
      if (!inner) H(h, loop, err);
      if (err <= s.eps) {
        res.status = 0;
        out = 1;
        break;
      } else if (loop >= s.maxloop) {
        res.status = 2;
        out = 1;
        break;
      }
      loop++;
      qq[k] = oracle_dot(n, Q + k * n, Q + k * n);
      double alpha = oracle_dot(n, r, Q + k * n) / qq[k];
      axy(n, alpha, P + k * n, x, x);
      if (k == m - 1) break;
      axy(n, -alpha, Q + k * n, r, r);
      MV(c, r, Av);
      double *pk1 = P + (k + 1) * n, *qk1 = Q + (k + 1) * n;
      memset(pk1, 0, sizeof(double) * (size_t)n);
      memset(qk1, 0, sizeof(double) * (size_t)n);
      for (long i = 0; i <= k; i++)
        beta[i] = -(seq_dot(n, Av, Q + i * n)) / qq[i];
      for (long i = 0; i <= k; i++) {
        axy(n, beta[i], P + i * n, pk1, pk1);
        axy(n, beta[i], Q + i * n, qk1, qk1);
      }
      vadd(n, r, pk1, pk1);
      vadd(n, Av, qk1, qk1);
    }
    if (out) break;
  }
  res.loop = loop;
  free(r);
  free(Av);
  free(P);
  free(Q);
  free(qq);
  free(beta);
  return res;
}

/* Shared GMRES / VPGMRES cycle: gmres::solve (gmres.cpp:232-422) and
 * vpgmres::solve (vpgmres.cpp:746-944). With flexible != 0 each Arnoldi
 * step first runs the inner solver on v_k and keeps its result in Z.
 * H is (restart+1) x restart, row-major. */
static res_t run_inner(ctx_t *c, const double *b, double *x);

static res_t solve_gmres_core(ctx_t *c, const double *b, double *x, int inner,
                              hist_t *h, int flexible) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  long m = s.restart;
  long ld = m; /* row stride of H */
  double *Av = vnew(n), *r = vnew(n), *v = vnew(n), *w = vnew(n);
  double *V = vnew(n * (m + 1)), *Z = flexible ? vnew(n * (m + 1)) : NULL;
  double *Hm = vnew((m + 1) * ld), *e = vnew(m + 1), *y = vnew(m + 1);
  double *cs = vnew(m + 1), *sn = vnew(m + 1);
  double *x0 = vnew(n), *tmpv = vnew(n), *z = flexible ? vnew(n) : NULL;
  double *tv = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  long count = 0;
  int over = 0;
  const double *B = flexible ? Z : V; /* basis the correction lives in */
  while (count < s.maxloop) {
    MV(c, x, Av);
    vsub(n, b, Av, r);
    double t = oracle_norm2(n, r);
    xdiva(n, r, t, v);
    memcpy(V, v, sizeof(double) * (size_t)n);
    for (long i = 0; i < m; i++) e[i] = 0.0;
    e[0] = t;
    for (long k = 0; k < m - 1; k++) {
      double err = fabs(e[k]) / bnorm;
      if (!inner) H(h, count + 1, err);
      int stop = 0;
      if (count + 1 >= s.maxloop) {
        over = 1;
        stop = 1;
      } else if (err <= s.eps) {
        res.status = 0;
        stop = 1;
      }
      if (stop) {
        hye(Hm, ld, y, e, k);
        memset(tmpv, 0, sizeof(double) * (size_t)n);
        for (long i = 0; i < k; i++) {
          if (c->p->fix_gmres_assembly)
            axy(n, y[i], B + i * n, tmpv, tmpv);
          else
            ax(n, y[i], B + i * n, tmpv);
        }
        vadd(n, x0, tmpv, x);
        break;
      }
      if (flexible) {
        memcpy(tv, v, sizeof(double) * (size_t)n);
        memset(z, 0, sizeof(double) * (size_t)n);
        run_inner(c, tv, z);
        MV(c, z, tv);
        memcpy(w, tv, sizeof(double) * (size_t)n);
        memcpy(Z + k * n, z, sizeof(double) * (size_t)n);
        for (long i = 0; i <= k; i++)
          Hm[i * ld + k] = oracle_dot(n, w, V + i * n);
      } else {
        memcpy(tv, V + k * n, sizeof(double) * (size_t)n);
        MV(c, tv, w);
        for (long i = 0; i <= k; i++)
          Hm[i * ld + k] = oracle_dot(n, w, V + i * n);
      }
      /* Gmres_sp_1 (blas.cpp:477-488) */
      for (long j = 0; j < n; j++)
        for (long i = 0; i <= k; i++) w[j] -= Hm[i * ld + k] * V[i * n + j];
      t = oracle_norm2(n, w);
      Hm[(k + 1) * ld + k] = t;
      xdiva(n, w, t, v);
      memcpy(V + (k + 1) * n, v, sizeof(double) * (size_t)n);
      for (long i = 0; i <= k - 1; i++) {
        double t1 = Hm[i * ld + k], t2 = Hm[(i + 1) * ld + k];
        Hm[i * ld + k] = cs[i] * t1 - sn[i] * t2;
        Hm[(i + 1) * ld + k] = sn[i] * t1 + cs[i] * t2;
      }
      double a = sqrt(Hm[k * ld + k] * Hm[k * ld + k] +
                      Hm[(k + 1) * ld + k] * Hm[(k + 1) * ld + k]);
      cs[k] = Hm[k * ld + k] / a;
      sn[k] = -Hm[(k + 1) * ld + k] / a;
      e[k + 1] = sn[k] * e[k];
      e[k] = cs[k] * e[k];
      Hm[k * ld + k] = cs[k] * Hm[k * ld + k] - sn[k] * Hm[(k + 1) * ld + k];
      Hm[(k + 1) * ld + k] = 0.0;
      count++;
    }
    if (res.status == 0 || over) break;
    /* end of cycle (gmres.cpp:409-421): y[restart-1] is never set by Hye; the
     * reference's buffer holds zero there, so the sum runs to restart-1. */
    hye(Hm, ld, y, e, m - 1);
    y[m - 1] = 0.0;
    memset(tmpv, 0, sizeof(double) * (size_t)n);
    for (long i = 0; i < m; i++)
      for (long j = 0; j < n; j++) tmpv[j] += y[i] * B[i * n + j];
    vadd(n, x0, tmpv, x);
    memcpy(x0, x, sizeof(double) * (size_t)n);
  }
  res.loop = count + 1;
  free(Av);
  free(r);
  free(v);
  free(w);
  free(V);
  free(Z);
  free(Hm);
  free(e);
  free(y);
  free(cs);
  free(sn);
  free(x0);
  free(tmpv);
  free(z);
  free(tv);
  return res;
}

/* Gram-coefficient updates of one k-skip CG step.
 * Reference form (kskipcg.cpp:284-289) and corrected form:
 *   delta'_j = delta_j - 2 a eta_{j+1} + a^2 zeta_{j+2}
 *   eta'_j   = delta'_j + b (eta_j - a zeta_{j+1})
 *   zeta'_j  = eta'_j + b (eta_j - a zeta_{j+1}) + b^2 zeta_j          */
static void kskipcg_update(int fixed, int cnt, double alpha, double beta,
                           double *delta, double *eta, double *zeta) {
  for (int j = 0; j < cnt; j++) {
    if (!fixed) {
      delta[j] = delta[j] - 2 * alpha * eta[j + 1] +
                 alpha * alpha * eta[j + 2];
      double eta_old = eta[j];
      eta[j] = delta[j] + beta * zeta[j + 1] - alpha * beta * zeta[j + 1];
      zeta[j] = eta[j + 1] + beta * eta_old + beta * beta * zeta[j] -
                alpha * beta * zeta[j + 1];
    } else {
      double d = delta[j] - 2 * alpha * eta[j + 1] +
                 alpha * alpha * zeta[j + 2];
      double rp = eta[j] - alpha * zeta[j + 1]; /* (r', A^{j+1} p) */
      double e = d + beta * rp;
      double z = e + beta * rp + beta * beta * zeta[j];
      delta[j] = d;
      eta[j] = e;
      zeta[j] = z;
    }
  }
}

/* kskipcg::solve (kskipcg.cpp:187-310). */
static res_t solve_kskipcg(ctx_t *c, const double *b, double *x, int inner,
                           hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  int k = s.kskip;
  double *r = vnew(n), *p = vnew(n), *Av = vnew(n);
  double *Ar = vnew(n * (2 * k + 1)), *Ap = vnew(n * (2 * k + 2));
  double *delta = vnew(2 * k + 2), *eta = vnew(2 * k + 3),
         *zeta = vnew(2 * k + 4);
  memset(x, 0, sizeof(double) * (size_t)n);
  MV(c, x, Av);
  vsub(n, b, Av, r);
  memcpy(p, r, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  long nloop;
  for (nloop = 0; nloop < s.maxloop; nloop += k + 1) {
    double err = oracle_norm2(n, r) / bnorm;
    if (!inner) H(h, nloop + 1, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    oracle_matpow(c->A, r, p, k, Ar, Ap);
    c->spmv += 4 * k + 3;
    double gamma = oracle_dot(n, r, r);
    oracle_gram_cg(n, k, Ar, Ap, r, p, delta, eta, zeta);
    for (long il = nloop; il <= nloop + k; il++) {
      double alpha = gamma / zeta[0];
      double beta = alpha * zeta[1] / zeta[0] - 1.0;
      if (s.fix == 1) {
        gamma = beta * gamma;
      } else if (s.fix == 2) {
        double t0 = gamma - alpha * eta[0];
        double t1 = eta[0] - alpha * zeta[1];
        gamma = t0 - alpha * t1;
      }
      kskipcg_update(c->p->fix_kskipcg, (int)(2 * k - 2 * (il - nloop)), alpha,
                     beta, delta, eta, zeta);
      MV(c, p, Av);
      axy(n, alpha, p, x, x);
      axy(n, -alpha, Av, r, r);
      axy(n, beta, p, r, p);
    }
  }
  res.loop = nloop - k + 1;
  free(r);
  free(p);
  free(Av);
  free(Ar);
  free(Ap);
  free(delta);
  free(eta);
  free(zeta);
  return res;
}

/* kskipBicg::solve (kskipbicg.cpp:207-352). */
static res_t solve_kskipbicg(ctx_t *c, const double *b, double *x, int inner,
                             hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, inner);
  res_t res = {2, 0};
  int k = s.kskip;
  double *r = vnew(n), *p = vnew(n), *rs = vnew(n), *ps = vnew(n),
         *Av = vnew(n);
  double *Ar = vnew(n * (2 * k + 1)), *Ap = vnew(n * (2 * k + 2));
  double *theta = vnew(2 * k + 2), *eta = vnew(2 * k + 3),
         *rho = vnew(2 * k + 3), *phi = vnew(2 * k + 4);
  memset(x, 0, sizeof(double) * (size_t)n);
  MV(c, x, Av);
  vsub(n, b, Av, r);
  memcpy(p, r, sizeof(double) * (size_t)n);
  memcpy(rs, r, sizeof(double) * (size_t)n);
  memcpy(ps, rs, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  long nloop;
  for (nloop = 0; nloop < s.maxloop; nloop += k + 1) {
    double err = oracle_norm2(n, r) / bnorm;
    if (!inner) H(h, nloop + 1, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    oracle_matpow(c->A, r, p, k, Ar, Ap);
    c->spmv += 4 * k + 3;
    double gamma = oracle_dot(n, rs, r);
    oracle_gram_bicg(n, k, Ar, Ap, rs, ps, theta, eta, rho, phi);
    for (long il = nloop; il <= nloop + k; il++) {
      double alpha = gamma / phi[0];
      double beta = 1.0 - (eta[0] + rho[0] - alpha * phi[1]) / phi[0];
      gamma = gamma * beta;
      for (int j = 0; j < 2 * k - 2 * (il - nloop); j++) {
        theta[j] = theta[j] - alpha * eta[j + 1] - alpha * rho[j + 1] +
                   alpha * alpha * phi[j + 2];
        double t = theta[j] - alpha * beta * phi[j + 1];
        eta[j] = t + beta * eta[j];
        rho[j] = t + beta * rho[j];
        phi[j] = eta[j] + rho[j] - theta[j] + beta * beta * phi[j];
      }
      MV(c, p, Av);
      axy(n, alpha, p, x, x);
      axy(n, -alpha, Av, r, r);
      MVT(c, ps, Av);
      axy(n, -alpha, Av, rs, rs);
      axy(n, beta, p, r, p);
      axy(n, beta, ps, rs, ps);
    }
  }
  res.loop = nloop + 1;
  free(r);
  free(p);
  free(rs);
  free(ps);
  free(Av);
  free(Ar);
  free(Ap);
  free(theta);
  free(eta);
  free(rho);
  free(phi);
  return res;
}

/* ------------------------------------------------------------------------ */
/* Variable-preconditioned (flexible) outer methods                          */
/* ------------------------------------------------------------------------ */

static res_t solve_gmres(ctx_t *c, const double *b, double *x, int inner,
                         hist_t *h) {
  return solve_gmres_core(c, b, x, inner, h, 0);
}

/* innerMethods::innerSelect (innerMethods.cpp:71-118). */
static res_t run_inner(ctx_t *c, const double *b, double *x) {
  switch (c->p->inner) {
    case OR_CG: return solve_cg(c, b, x, 1, NULL);
    case OR_CR: return solve_cr(c, b, x, 1, NULL);
    case OR_GCR: return solve_gcr(c, b, x, 1, NULL);
    case OR_BICG: return solve_bicg(c, b, x, 1, NULL);
    case OR_GMRES: return solve_gmres(c, b, x, 1, NULL);
    case OR_KSKIPCG: return solve_kskipcg(c, b, x, 1, NULL);
    case OR_KSKIPBICG: return solve_kskipbicg(c, b, x, 1, NULL);
    default: {
      res_t r = {99, 0};
      return r;
    }
  }
}

/* vpcg::solve (vpcg.cpp:659-750). */
static res_t solve_vpcg(ctx_t *c, const double *b, double *x, hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, 0);
  res_t res = {2, 0};
  double *r = vnew(n), *p = vnew(n), *z = vnew(n), *mv = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  MV(c, x, mv);
  vsub(n, b, mv, r);
  run_inner(c, r, z);
  memcpy(p, z, sizeof(double) * (size_t)n);
  double rr = oracle_dot(n, r, z);
  long loop;
  for (loop = 1; loop <= s.maxloop; loop++) {
    double err = oracle_norm2(n, r) / bnorm;
    H(h, loop, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    MV(c, p, mv);
    double d = oracle_dot(n, p, mv);
    double alpha = rr / d;
    axy(n, alpha, p, x, x);
    axy(n, -alpha, mv, r, r);
    memset(z, 0, sizeof(double) * (size_t)n);
    run_inner(c, r, z);
    double rr2 = oracle_dot(n, r, z);
    double beta = rr2 / rr;
    rr = rr2;
    axy(n, beta, p, z, p);
  }
  res.loop = loop;
  free(r);
  free(p);
  free(z);
  free(mv);
  return res;
}

/* vpcr::solve (vpcr.cpp:670-775). */
static res_t solve_vpcr(ctx_t *c, const double *b, double *x, hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, 0);
  res_t res = {2, 0};
  double *r = vnew(n), *p = vnew(n), *z = vnew(n), *Av = vnew(n),
         *Ap = vnew(n);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  MV(c, x, Av);
  vsub(n, b, Av, r);
  run_inner(c, r, z);
  memcpy(p, z, sizeof(double) * (size_t)n);
  MV(c, z, Av);
  memcpy(Ap, Av, sizeof(double) * (size_t)n);
  double zaz = oracle_dot(n, z, Av);
  long loop;
  for (loop = 1; loop <= s.maxloop; loop++) {
    double err = oracle_norm2(n, r) / bnorm;
    H(h, loop, err);
    if (err <= s.eps) {
      res.status = 0;
      break;
    }
    double t = oracle_dot(n, Ap, Ap);
    double alpha = zaz / t;
    axy(n, alpha, p, x, x);
    axy(n, -alpha, Ap, r, r);
    memset(z, 0, sizeof(double) * (size_t)n);
    run_inner(c, r, z);
    MV(c, z, Av);
    double zaz2 = oracle_dot(n, z, Av);
    double beta = zaz2 / zaz;
    zaz = zaz2;
    axy(n, beta, p, z, p);
    axy(n, beta, Ap, Av, Ap);
  }
  res.loop = loop;
  free(r);
  free(p);
  free(z);
  free(Av);
  free(Ap);
  return res;
}

/* vpgcr::solve (vpgcr.cpp:693-846). */
static res_t solve_vpgcr(ctx_t *c, const double *b, double *x, hist_t *h) {
  long n = c->A->n;
  sp_t s = params_for(c, 0);
  res_t res = {2, 0};
  long m = s.restart;
  double *r = vnew(n), *Av = vnew(n), *z = vnew(n);
  double *P = vnew(n * m), *Q = vnew(n * m);
  double *qq = vnew(m), *beta = vnew(m);
  memset(x, 0, sizeof(double) * (size_t)n);
  double bnorm = oracle_norm2(n, b);
  long loop = 1;
  int out = 0;
  while (loop < s.maxloop) {
    MV(c, x, Av);
    vsub(n, b, Av, r);
    memset(P, 0, sizeof(double) * (size_t)n);
    run_inner(c, r, Av);
    memcpy(P, Av, sizeof(double) * (size_t)n);
    MV(c, P, Q);
    for (long k = 0; k < m; k++) {
      double err = oracle_norm2(n, r) / bnorm;
      H(h, loop, err);
      if (err <= s.eps) {
        res.status = 0;
        out = 1;
        break;
      } else if (loop >= s.maxloop) {
        res.status = 2;
        out = 1;
        break;
      }
      loop++;
      qq[k] = oracle_dot(n, Q + k * n, Q + k * n);
      double alpha = oracle_dot(n, r, Q + k * n) / qq[k];
      axy(n, alpha, P + k * n, x, x);
      if (k == m - 1) break;
      axy(n, -alpha, Q + k * n, r, r);
      memset(z, 0, sizeof(double) * (size_t)n);
      run_inner(c, r, z);
      MV(c, z, Av);
      double *pk1 = P + (k + 1) * n, *qk1 = Q + (k + 1) * n;
      memset(pk1, 0, sizeof(double) * (size_t)n);
      memset(qk1, 0, sizeof(double) * (size_t)n);
      for (long i = 0; i <= k; i++)
        beta[i] = -(seq_dot(n, Av, Q + i * n)) / qq[i];
      for (long i = 0; i <= k; i++) {
        axy(n, beta[i], P + i * n, pk1, pk1);
        axy(n, beta[i], Q + i * n, qk1, qk1);
      }
      vadd(n, z, pk1, pk1);
      vadd(n, Av, qk1, qk1);
    }
    if (out) break;
  }
  res.loop = loop;
  free(r);
  free(Av);
  free(z);
  free(P);
  free(Q);
  free(qq);
  free(beta);
  return res;
}

/* ------------------------------------------------------------------------ */
/* Entry points                                                              */
/* ------------------------------------------------------------------------ */

void oracle_default_params(or_params *p) {
  memset(p, 0, sizeof(*p));
  p->outer = OR_NONE;
  p->inner = OR_NONE;
  p->outer_maxloop = 10000;
  p->inner_maxloop = 50;
  p->outer_eps = 1e-8;
  p->inner_eps = 1e-1;
  p->outer_restart = 1000;
  p->inner_restart = 1000;
  p->outer_kskip = 2;
  p->inner_kskip = 2;
  p->outer_fix = 2;
  p->inner_fix = 2;
  p->fix_kskipcg = 0;
  p->fix_gmres_assembly = 0;
  p->sum_chunks = 1;
}

/* outerMethods::outerSelect (outerMethods.cpp:20-82). */
int oracle_solve(const or_mat *A, const or_params *p, const double *b,
                 double *x, long *hist_iter, double *hist_err, long hist_cap,
                 or_report *rep) {
  ctx_t c = {A, p, 0, p->inner != OR_NONE};
  g_sum_chunks = p->sum_chunks > 1 || p->sum_chunks == -1 || p->sum_chunks == -2 ? p->sum_chunks : 1;
  hist_t h = {hist_iter, hist_err, hist_iter && hist_err ? hist_cap : 0, 0};
  res_t res = {99, 0};
  long n = A->n;
  switch (p->outer) {
    case OR_CG: res = solve_cg(&c, b, x, 0, &h); break;
    case OR_CR: res = solve_cr(&c, b, x, 0, &h); break;
    case OR_GCR: res = solve_gcr(&c, b, x, 0, &h); break;
    case OR_BICG: res = solve_bicg(&c, b, x, 0, &h); break;
    case OR_GMRES: res = solve_gmres(&c, b, x, 0, &h); break;
    case OR_KSKIPCG: res = solve_kskipcg(&c, b, x, 0, &h); break;
    case OR_KSKIPBICG: res = solve_kskipbicg(&c, b, x, 0, &h); break;
    case OR_VPCG: res = solve_vpcg(&c, b, x, &h); break;
    case OR_VPCR: res = solve_vpcr(&c, b, x, &h); break;
    case OR_VPGCR: res = solve_vpgcr(&c, b, x, &h); break;
    case OR_VPGMRES: res = solve_gmres_core(&c, b, x, 0, &h, 1); break;
    default: break; /* KSKIPCR, VPBICG, NONE: "Not implemented" */
  }
  if (rep) {
    rep->status = res.status;
    rep->loop = res.loop;
    rep->hist_len = h.len;
    rep->spmv = c.spmv;
    rep->true_res_log10 = 0.0;
    if (res.status != 99) {
      double *x0 = vnew(n);
      rep->true_res_log10 = oracle_check_error(A, b, x, x0);
      free(x0);
    }
  }
  g_sum_chunks = 1;
  return res.status;
}
