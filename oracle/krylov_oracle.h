/* CPU oracle for the solver_cpp Krylov hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A single-threaded C restatement of the reference's CPU path (blas.cpp and the
 * solver loops cg.cpp, cr.cpp, bicg.cpp, gcr.cpp, gmres.cpp, kskipcg.cpp,
 * kskipbicg.cpp, vpcg.cpp, vpcr.cpp, vpgcr.cpp, vpgmres.cpp). Every floating
 * point operation is done in the same order as the reference run with one
 * OpenMP thread (-t 1), so its residual histories match that run bit for bit.
 *
 * Only tests/, the smoke check and the benchmark's CPU-baseline leg may load
 * this library, and only as the checker. The product path never calls it.
 *
 * Two reference defects can be switched to corrected forms:
 *   fix_kskipcg        k-skip CG Gram recurrences (kskipcg.cpp:284-287)
 *   fix_gmres_assembly GMRES/VPGMRES solution assembly on convergence or at
 *                      maxloop inside a restart cycle (gmres.cpp:286-324,
 *                      vpgmres.cpp:793-831: Scalar_ax overwrites instead of
 *                      accumulating)
 */
#ifndef KRYLOV_ORACLE_H
#define KRYLOV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Values follow the reference's SOLVERS_NAME (solver_collection.hpp:7-24). */
enum {
  OR_NONE = 0, OR_CG = 1, OR_BICG = 2, OR_CR = 3, OR_GCR = 4, OR_GMRES = 5,
  OR_KSKIPCG = 6, OR_KSKIPCR = 7, OR_KSKIPBICG = 8, OR_VPCG = 9,
  OR_VPBICG = 10, OR_VPCR = 11, OR_VPGCR = 12, OR_VPGMRES = 13
};

typedef struct {
  long n;
  const int *ptr, *col;   /* CSR, 0-based, square n x n */
  const double *val;
  const int *tptr, *tcol; /* CSR of A^T (may be NULL unless BiCG family) */
  const double *tval;
} or_mat;

typedef struct {
  int outer, inner;       /* SOLVERS_NAME codes; inner = OR_NONE for plain runs */
  long outer_maxloop;     /* -L */
  double outer_eps;       /* -E */
  long outer_restart;     /* -R */
  int outer_kskip;        /* -K */
  int outer_fix;          /* -F */
  long inner_maxloop;     /* -l */
  double inner_eps;       /* -e */
  long inner_restart;     /* -r */
  int inner_kskip;        /* -k */
  int inner_fix;          /* -f */
  int fix_kskipcg;        /* 1: corrected recurrences */
  int fix_gmres_assembly; /* 1: accumulate the correction */
  int sum_chunks;         /* >1: dot products and norms summed as that many
                             contiguous partial sums added in order, the way
                             an OpenMP static reduction with that many
                             threads does; 0/1: one sequential sum (-t 1);
                             -1: pairwise (recursive halving) sums;
                             -2: pairwise, and so are the dots the
                             reference always sums sequentially (the
                             k-skip Gram values, GCR's beta dots) */
} or_params;

typedef struct {
  int status;          /* 0 converged, 2 not converged, 99 not implemented */
  long loop;           /* the value the reference prints as "loop =" */
  long hist_len;       /* history entries produced (may exceed capacity) */
  double true_res_log10; /* blas::Check_error(x, x_0) */
  long spmv;           /* SpMV count (A and A^T), outer and inner */
} or_report;

/* Reference defaults (solver_collection.cpp:26-49). */
void oracle_default_params(or_params *p);

/* Full solve. x is overwritten (the reference zeroes it first). History
 * entries are (iteration label, relative residual) as written to
 * ./output/<NAME>_his.txt. Returns report->status. */
int oracle_solve(const or_mat *A, const or_params *p, const double *b,
                 double *x, long *hist_iter, double *hist_err, long hist_cap,
                 or_report *report);

/* Primitives (blas.cpp) for unit tests. */
void oracle_spmv(const or_mat *A, const double *x, double *y);
void oracle_spmv_t(const or_mat *A, const double *x, double *y);
double oracle_dot(long n, const double *x, const double *y);
double oracle_norm2(long n, const double *x);
void oracle_csr_transpose(long n, long nnz, const int *ptr, const int *col,
                          const double *val, int *tptr, int *trow,
                          double *tval);
void oracle_matpow(const or_mat *A, const double *r, const double *p, int k,
                   double *Ar, double *Ap);
void oracle_gram_cg(long n, int k, const double *Ar, const double *Ap,
                    const double *r, const double *p, double *delta,
                    double *eta, double *zeta);
void oracle_gram_bicg(long n, int k, const double *Ar, const double *Ap,
                      const double *rs, const double *ps, double *theta,
                      double *eta, double *rho, double *phi);
double oracle_check_error(const or_mat *A, const double *b, const double *x,
                          const double *x0);
/* Gradient of L(x(A,b)) through the adjoint A^T lambda = g:
 * grad_b = lambda, grad_val[j] = -lambda[row(j)] * x[col[j]]. */
void oracle_pattern_grad(const or_mat *A, const double *lambda,
                         const double *x, double *grad_val);

#ifdef __cplusplus
}
#endif
#endif
