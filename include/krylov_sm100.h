/*
 * krylov_sm100.h -- C ABI of the B200 (sm_100a) Krylov hot path of solver_cpp.
 *
 * This library replaces the reference's host math class `blas`
 * (blas.hpp:8-78) and its device offload class `cuda` (cudaFunction.hpp:7-129)
 * with device-resident kernels, and runs the reference's Krylov methods
 * (cg.cpp, cr.cpp, bicg.cpp, gcr.cpp, gmres.cpp, kskipcg.cpp, kskipbicg.cpp,
 * vpcg.cpp, vpcr.cpp, vpgcr.cpp, vpgmres.cpp) with every vector kept in HBM.
 * Only scalars (convergence flags, the residual history) come back to the host.
 *
 * Conventions
 *  - Every entry point returns a ks_status and never exits or traps. On failure
 *    ks_last_error() describes the cause.
 *  - Matrices are square CSR with 0-based int32 indices, as the reference's
 *    collection holds them (solver_collection.hpp:100-117).
 *  - Work is issued on the context's stream. Calls that return host scalars
 *    synchronise that stream; all others are asynchronous.
 *  - One context may be used by one host thread at a time.
 */
#ifndef KRYLOV_SM100_H
#define KRYLOV_SM100_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KS_ABI_VERSION 4

typedef enum {
  KS_OK = 0,              /* converged / success (reference solve() == 0)      */
  KS_NOT_CONVERGED = 2,   /* maxloop reached (reference solve() == 2)           */
  KS_BREAKDOWN = 3,       /* a Krylov denominator was exactly zero              */
  KS_NAN_DETECTED = 4,    /* a recurrence produced a non-finite scalar          */
  KS_BAD_INPUT = 5,       /* invalid argument, shape or handle                  */
  KS_CUDA_ERROR = 6,      /* a CUDA runtime call failed                         */
  KS_TIMEOUT = 7,         /* a bounded device wait gave up                      */
  KS_OUT_OF_MEMORY = 8,   /* device (CRS text I/O: host) allocation failed      */
  KS_NO_DEVICE = 9,       /* no usable CUDA device                              */
  KS_IO_ERROR = 10,       /* CRS text files missing or malformed                */
  KS_UNIMPLEMENTED = 99   /* reference's "Not implemented" (KSKIPCR, VPBICG)    */
} ks_status;

/* Method names; values equal the reference's SOLVERS_NAME
 * (solver_collection.hpp:7-24). */
typedef enum {
  KS_NONE = 0, KS_CG = 1, KS_BICG = 2, KS_CR = 3, KS_GCR = 4, KS_GMRES = 5,
  KS_KSKIPCG = 6, KS_KSKIPCR = 7, KS_KSKIPBICG = 8, KS_VPCG = 9,
  KS_VPBICG = 10, KS_VPCR = 11, KS_VPGCR = 12, KS_VPGMRES = 13
} ks_solver;

/* Element type of a vector, or of the matrix values an operation reads. */
typedef enum { KS_FP64 = 0, KS_FP32 = 1, KS_BF16 = 2 } ks_precision;

typedef struct ks_ctx ks_ctx;
typedef struct ks_mat ks_mat;
typedef struct ks_vec ks_vec;

/* ---------------------------------------------------------------- context */

/* Replaces the reference's per-solver `new cuda(times*, N, ...)` buffer owner
 * (cudaFunction.cu:270-372) and cuda::Reset/GetDeviceNum
 * (cudaFunction.cu:571-578,1905-1909): a context owns the stream, the
 * reduction scratch and a workspace pool reused across solves. */
ks_status ks_ctx_create(int device, ks_ctx **out);
ks_status ks_ctx_destroy(ks_ctx *ctx);
/* Use an existing cudaStream_t (passed as void*); NULL restores the
 * context's own stream. */
ks_status ks_ctx_set_stream(ks_ctx *ctx, void *stream);
/* Waits for the context's queued work; KS_TIMEOUT if a bounded device wait of
 * a queued kernel ran out since the last call that reported one (asynchronous
 * calls such as ks_spmv report it here, at the next call returning host
 * scalars, or at the next ks_solve). */
ks_status ks_ctx_synchronize(ks_ctx *ctx);
/* Number of CUDA devices (cuda::GetDeviceNum, cudaFunction.cu:1905). */
int ks_device_count(void);
const char *ks_status_string(ks_status s);
/* Kernels this context has launched so far (diagnostics; the reference's
 * `times` class counts time, not launches: times.hpp:15-88). */
int64_t ks_ctx_launches(const ks_ctx *ctx);
const char *ks_last_error(const ks_ctx *ctx);
int ks_abi_version(void);
/* Limit of every bounded device wait of this context's kernels (the SpMV's
 * shared-memory staging barriers), in nanoseconds; ns <= 0 restores the
 * default of 2 s. A wait that runs out ends its kernel early with the
 * context's timeout flag set, and the call returns KS_TIMEOUT; the kernel
 * still drains its own copies in flight (bounded by the default limit), so
 * the context stays usable. Lowering it is a way to exercise that path. No
 * counterpart in the reference, whose waits are unbounded (cudaDeviceSynchronize
 * in checkCudaErrors). */
ks_status ks_ctx_set_wait_limit(ks_ctx *ctx, int64_t ns);

/* ----------------------------------------------------------------- matrix */

#define KS_MAT_TRANSPOSE 1u /* also build A^T (the reference's CTval/CTcol/CTptr) */
#define KS_MAT_FP32 2u      /* keep an FP32 copy of the values                    */
#define KS_MAT_BF16 4u      /* keep a BF16 copy of the values                     */
/* By default the SpMV reads column indices as 16-bit offsets from the row
 * (col - row) whenever every offset of the matrix fits in int16, halving the
 * index bytes of banded and stencil matrices; results are identical. This
 * flag keeps the int32 columns instead. */
#define KS_MAT_INDEX32 8u
/* By default a matrix whose rows hold their columns at no more than 8
 * distinct offsets from the row (stencils, banded matrices), each row in
 * increasing column order, with the diagonals at least 3/4 full, also keeps
 * a diagonal copy (values diagonal-major, one presence mask byte per row),
 * which the SpMV reads instead of the CSR arrays: no column indices at all,
 * coalesced reads of x. Results are identical. This flag keeps CSR only. */
#define KS_MAT_NO_DIAG 16u

/* Upload a host CSR matrix (collection::CudaCopy_Part1,
 * solver_collection.cpp:932-942) and build the row-block schedule of the
 * adaptive SpMV. With KS_MAT_TRANSPOSE the transpose is built on the device;
 * it replaces cuda::CSR2CSC (cudaFunction.cu:896-982), whose cuSPARSE call no
 * longer exists in CUDA 12. */
ks_status ks_csr_upload(ks_ctx *ctx, int64_t n, int64_t nnz,
                        const int32_t *ptr, const int32_t *col,
                        const double *val, unsigned flags, ks_mat **out);
/* Same from device arrays (copied; the caller keeps ownership). */
ks_status ks_csr_upload_device(ks_ctx *ctx, int64_t n, int64_t nnz,
                               const int32_t *d_ptr, const int32_t *d_col,
                               const double *d_val, unsigned flags,
                               ks_mat **out);
ks_status ks_mat_destroy(ks_mat *mat);
/* n, nnz, and the number of SpMV row blocks. */
ks_status ks_mat_info(const ks_mat *mat, int64_t *n, int64_t *nnz,
                      int64_t *row_blocks);
/* Bytes per column index the SpMV reads for A (2 or 4) and for A^T (0 when
 * there is no transpose). No counterpart in the reference. */
ks_status ks_mat_index_bytes(const ks_mat *mat, int *a_bytes, int *t_bytes);
/* Diagonals of the diagonal copy of A and of A^T (0: the SpMV reads CSR). No
 * counterpart in the reference. */
ks_status ks_mat_diagonals(const ks_mat *mat, int *a_diagonals, int *t_diagonals);
/* 1 where the diagonal copy of A (of A^T) keeps only its main and upper
 * diagonals because the matrix equals its transpose bit for bit: the SpMV
 * then reads each lower diagonal as its upper mirror, shifted (4 instead of 7
 * value streams for a 7-point stencil). No counterpart in the reference. */
ks_status ks_mat_dia_symmetric(const ks_mat *mat, int *a_sym, int *t_sym);
/* Copy the device-built transpose back (CSR of A^T: tptr[n+1], trow[nnz],
 * tval[nnz]), i.e. the CSC arrays the reference's CSR2CSC returns. */
ks_status ks_mat_transpose_download(const ks_mat *mat, int32_t *tptr,
                                    int32_t *trow, double *tval);

/* ----------------------------------------------------------------- vector */

/* Device vectors (the reference keeps them on the host and copies them on
 * every SpMV: cuda::H2D/D2H, cudaFunction.cu:421-471). */
ks_status ks_vec_create(ks_ctx *ctx, int64_t n, ks_precision type,
                        ks_vec **out);
/* Non-owning view of caller device memory (e.g. a torch tensor). */
ks_status ks_vec_wrap(ks_ctx *ctx, int64_t n, ks_precision type,
                      void *device_ptr, ks_vec **out);
ks_status ks_vec_destroy(ks_vec *v);
ks_status ks_vec_upload(ks_vec *v, const void *host);      /* synchronous */
ks_status ks_vec_download(const ks_vec *v, void *host);    /* synchronous */
/* Part of a vector: elements [offset, offset+count). */
ks_status ks_vec_upload_range(ks_vec *v, int64_t offset, int64_t count,
                              const void *host);
ks_status ks_vec_download_range(const ks_vec *v, int64_t offset,
                                int64_t count, void *host);
ks_status ks_vec_fill(ks_vec *v, double value);
void *ks_vec_device_ptr(ks_vec *v);
int64_t ks_vec_length(const ks_vec *v);

/* ------------------------------------------------------------ primitives */

/* y = A x (trans = 0) or y = A^T x (trans = 1). Replaces cuda::MtxVec_mult
 * (cudaFunction.cu:613-638) and blas::MtxVec_mult (blas.cpp:43-129). The
 * matrix values read follow the vectors: FP64 vectors read the FP64 values,
 * FP32 vectors the FP32 copy. For FP64 rows of up to 2048 nonzeros the sum
 * runs in the reference's order and matches it bit for bit. */
ks_status ks_spmv(const ks_mat *mat, int trans, const ks_vec *x, ks_vec *y);
/* As ks_spmv, choosing the matrix value copy explicitly (KS_BF16 values with
 * FP32 vectors is the BF16-stored variant). */
ks_status ks_spmv_values(const ks_mat *mat, int trans, ks_precision values,
                         const ks_vec *x, ks_vec *y);
/* blas::dot / blas::norm_2 (blas.cpp:149-209, 31-41); deterministic. */
ks_status ks_dot(const ks_vec *x, const ks_vec *y, double *result);
ks_status ks_nrm2(const ks_vec *x, double *result);
/* y = a*x + y (blas::Scalar_axy, blas.cpp:226-233). */
ks_status ks_axpy(double a, const ks_vec *x, ks_vec *y);
/* Fused y = a*x + y and result = (y, w) in one pass. */
ks_status ks_axpy_dot(double a, const ks_vec *x, ks_vec *y, const ks_vec *w,
                      double *result);
/* h[i] = (V_i, w) for i < k, V_i = V[i*ld .. i*ld+n). GMRES's H column
 * (gmres.cpp:354-371) and GCR's beta dots (blas.cpp:532-535) as one
 * tall-skinny pass. h may be host memory (the call returns with the k
 * results in it) or device memory of the context's GPU (the results are
 * written there in stream order and the call returns without waiting). */
ks_status ks_block_dot(const ks_vec *V, int64_t ld, int k, const ks_vec *w,
                       double *h);
/* Allocation-free form of ks_block_dot, for callers that cannot allocate
 * device memory when they need the product: code running inside a CUDA stream
 * capture (cudaMalloc is not allowed there), applications whose device memory
 * is all owned by their own pool allocator, and loops that must not reach the
 * driver allocator (cudaMalloc/cudaFree can synchronise the device). It needs
 * no context. V (k vectors of length n, stride ld), w (n) and h (k results)
 * are device pointers of the current device; the work is queued on `stream`
 * (a cudaStream_t; NULL is the legacy default stream) and the call returns
 * without waiting. Its only scratch is one fixed 151,808-byte device array that
 * every GPU loading the library holds until the process exits; the first call
 * on a device looks up that array's address, so make it before any stream
 * capture starts. Every call uses the same array and clears its counters on
 * entry: calls that can overlap on the GPU (other streams, other host threads
 * on the same device) race and must be serialised by the caller. k must be at
 * most KS_NOALLOC_MAX_K; larger k returns KS_BAD_INPUT (with a message on
 * stderr). This entry point has no counterpart in the reference. */
#define KS_NOALLOC_MAX_K 64
ks_status ks_block_dot_noalloc(const double *V, int64_t ld, int k, const double *w, int64_t n, double *h,
                               void *stream);
/* w[j] -= h[i] * V_i[j] for i = 0..k-1 in order (blas::Gmres_sp_1,
 * blas.cpp:477-488). h in host memory is copied in and the call waits for
 * the update; h in device memory of the context's GPU is read in stream
 * order and the call returns without waiting. */
ks_status ks_block_axpy(const ks_vec *V, int64_t ld, int k, const double *h,
                        ks_vec *w);
/* Matrix powers Ar[i] = A^{i+1} r (i <= 2k), Ap[i] = A^{i+1} p (i <= 2k+1),
 * stored contiguously with stride n (blas::Kskip_cg_bicg_base,
 * blas.cpp:353-399; cuda::Kskip_cg_bicg_base, cudaFunction.cu:984-1026). */
ks_status ks_matpow(const ks_mat *mat, const ks_vec *r, const ks_vec *p,
                    int k, ks_vec *Ar, ks_vec *Ap);
/* k-skip CG Gram values delta[2k], eta[2k+1], zeta[2k+2]
 * (blas::Kskip_cg_innerProduce, blas.cpp:401-435). */
ks_status ks_gram_cg(const ks_vec *Ar, const ks_vec *Ap, const ks_vec *r,
                     const ks_vec *p, int k, double *delta, double *eta,
                     double *zeta);
/* k-skip BiCG Gram values theta[2k], eta[2k+1], rho[2k+1], phi[2k+2]
 * against the shadow vectors (blas::Kskip_bicg_innerProduce,
 * blas.cpp:437-475). */
ks_status ks_gram_bicg(const ks_vec *Ar, const ks_vec *Ap, const ks_vec *rs,
                       const ks_vec *ps, int k, double *theta, double *eta,
                       double *rho, double *phi);

/* ------------------------------------------------------------------ solve */

/* Mirrors the reference's flags (solver_collection.cpp:278-307):
 * -L -E -R -K -F (outer) and -l -e -r -k -f (inner). */
typedef struct {
  int64_t outer_maxloop;   /* -L, default 10000 */
  double outer_eps;        /* -E, default 1e-8  */
  int64_t outer_restart;   /* -R, default 1000  */
  int32_t outer_kskip;     /* -K, default 2     */
  int32_t outer_fix;       /* -F, default 2     */
  int64_t inner_maxloop;   /* -l, default 50    */
  double inner_eps;        /* -e, default 1e-1  */
  int64_t inner_restart;   /* -r, default 1000  */
  int32_t inner_kskip;     /* -k, default 2     */
  int32_t inner_fix;       /* -f, default 2     */
  int32_t inner_precision; /* ks_precision of a VP method's inner solve      */
  int32_t reference_defects; /* 1: reproduce the reference's k-skip CG
                                recurrences and GMRES assembly; 0: corrected */
  int32_t transpose;       /* 1: solve A^T x = b (adjoint solves)            */
  int32_t poll_interval;   /* iterations in flight between host polls; 0=auto */
  int32_t x_update;        /* CG, CR, BiCG, and VPCG with the on-chip
                              FP32/BF16 inner CG: 0 auto, 1 x += alpha p
                              every iteration, 2 deferred through a ring of
                              32 directions (same x bit for bit)           */
  int32_t cluster_solve;   /* CG, CR, BiCG on at most 32768 rows (one GPU): 0
                              auto, the whole solve in one launch of one
                              thread-block cluster where the device can hold
                              it; 1 never (one kernel per step, as for larger
                              systems)                                      */
  int32_t inner_fast;      /* VP methods whose inner CG runs in FP32 / with
                              BF16 values on a one-GPU matrix with a diagonal
                              copy: 0 auto, the whole inner solve as one
                              cooperative kernel with its vectors on chip
                              where the system fits (up to ~28,900 rows per
                              SM); 1 one kernel per step. Both apply the same
                              operations to every element; the order in which
                              the dot products add their terms differs.    */
  int32_t true_residual;   /* VP methods: when the recurrence residual
                              passes -E, recompute |b - A x| / |b| in FP64
                              and stop only if it passes too, else go on
                              (the residual history carries on). 0 auto: on
                              for an FP32 / BF16 inner solve, off for FP64
                              (the reference stops on the recurrence
                              residual, vpcg.cpp:704-713); 1 on; 2 off.     */
  int32_t profile;         /* 1: device time per kernel class in the report
                              (ks_report.t_*); adds two events per launch  */
  int32_t reserved0;
  const double *x_ref;     /* NULL, or a device FP64 solution of the same
                              system (e.g. from the plain FP64 method):
                              ks_report.x_rel_diff = |x - x_ref| / |x_ref|  */
} ks_params;

typedef struct {
  int32_t status;          /* ks_status of the method                        */
  int64_t loop;            /* the value the reference prints as "loop ="     */
  int64_t hist_len;        /* residual-history entries produced              */
  double final_rel_res;    /* last history value                             */
  double true_res_log10;   /* log10(|b-Ax|/|b-Ax0|), blas::Check_error       */
  double true_rel_res;     /* |b-Ax|_2/|b|_2 in FP64                         */
  int64_t spmv_count;      /* SpMVs issued (A and A^T, outer and inner)      */
  int64_t inner_iterations;/* inner-solver iterations (VP methods)          */
  double solve_seconds;    /* device time of the solve loop (CUDA events)    */
  double x_rel_diff;       /* |x - x_ref| / |x_ref| (params.x_ref), else -1  */
  int64_t true_residual_checks; /* FP64 true-residual checks of a VP method  */
  /* Device seconds per kernel class with params.profile = 1 (else 0), the
   * classes of the reference's times report (times.cpp:60-76): SpMVs with
   * their fused epilogues; reductions (dots, norms, Gram and block dots);
   * other kernels (vector updates, basis combinations, scalar steps);
   * memsets; host<->device copies of the solve (ks_solve_host). */
  double t_mv, t_dot, t_other, t_memset, t_h2d, t_d2h;
  /* With params.profile = 1: kernels launched per class (SpMVs, reductions,
   * other, memsets), and the share of the SpMV class that read FP32 / BF16
   * values (a VP method's inner solves): its time and launches. */
  int64_t n_mv, n_dot, n_other, n_memset;
  double t_mv_low;
  int64_t n_mv_low;
} ks_report;

void ks_params_default(ks_params *p);

/* Run one Krylov method on device vectors (outerMethods::outerSelect,
 * outerMethods.cpp:20-82; innerMethods::innerSelect, innerMethods.cpp:71-118).
 * x is overwritten (the reference zeroes it: cg.cpp:79). If hist_err is not
 * NULL the residual history (iteration label, relative residual) -- the
 * contents of ./output/<NAME>_his.txt -- is copied out, up to hist_cap rows.
 * Returns the method's status (KS_OK, KS_NOT_CONVERGED, ...). */
ks_status ks_solve(ks_ctx *ctx, const ks_mat *mat, ks_solver outer,
                   ks_solver inner, const ks_params *params, const ks_vec *b,
                   ks_vec *x, int64_t *hist_iter, double *hist_err,
                   int64_t hist_cap, ks_report *report);
/* Same with host arrays: b is uploaded, x downloaded (end to end). */
ks_status ks_solve_host(ks_ctx *ctx, const ks_mat *mat, ks_solver outer,
                        ks_solver inner, const ks_params *params,
                        const double *b, double *x, int64_t *hist_iter,
                        double *hist_err, int64_t hist_cap,
                        ks_report *report);
/* log10(|b - A x| / |b - A x0|) with x0 = 0 (blas::Check_error,
 * blas.cpp:266-301), plus |b - A x|/|b| in *rel (may be NULL). */
ks_status ks_check_error(const ks_mat *mat, const ks_vec *b, const ks_vec *x,
                         double *log10_ratio, double *rel);

/* ---------------------------------------------------------------- adjoint */

/* Gradient of a loss L(x) with x = A^{-1} b, given g = dL/dx:
 * solve A^T lambda = g with `solver` (on the transpose), then
 * grad_b = lambda and grad_val[j] = -lambda[row(j)] * x[col(j)] over the CSR
 * pattern. grad_b and grad_val may be NULL. The reference has no counterpart. */
ks_status ks_adjoint_grad(ks_ctx *ctx, const ks_mat *mat, ks_solver solver,
                          ks_solver inner, const ks_params *params,
                          const ks_vec *x, const ks_vec *g, ks_vec *grad_b,
                          ks_vec *grad_val, ks_report *report);
/* The fused pattern gather alone: grad_val[j] = -lambda[row(j)] * x[col(j)]. */
ks_status ks_pattern_grad(const ks_mat *mat, const ks_vec *lambda,
                          const ks_vec *x, ks_vec *grad_val);

/* ---------------------------------------------------------------- CRS I/O */

/* The reference's text format (collection::checkCRSMatrix / readMatrix,
 * solver_collection.cpp:655-828): dir/ColVal.txt, dir/Ptr.txt, dir/bx.txt. */
ks_status ks_crs_read_header(const char *dir, int64_t *n, int64_t *nnz);
ks_status ks_crs_read(const char *dir, int64_t n, int64_t nnz, int32_t *ptr,
                      int32_t *col, double *val, double *b, double *x);
ks_status ks_crs_write(const char *dir, int64_t n, int64_t nnz,
                       const int32_t *ptr, const int32_t *col,
                       const double *val, const double *b, const double *x);

/* -------------------------------------------------------------- multi-GPU */

/* Row partition for a solve split over `nranks` GPUs (host only): contiguous
 * blocks row_start[0] = 0 <= ... <= row_start[nranks] = n with every inner
 * boundary a multiple of `align` rows (for a grid matrix: one plane). With
 * align = 1 and two ranks the first block has ceil(n/2) rows, the reference's
 * two-GPU split (solver_collection.cpp:1022-1031). */
ks_status ks_partition_rows(int64_t n, int nranks, int64_t align, int64_t *row_start);
/* The contiguous column window [lo, hi) that rows r0..r1-1 read, lo <= r0,
 * hi >= r1 (host only). ptr holds r1 - r0 + 1 offsets (any base) and col the
 * global column indices of those rows. A rank keeps x over its window. */
ks_status ks_halo_window(int64_t r0, int64_t r1, const int32_t *ptr, const int32_t *col,
                         int64_t *lo, int64_t *hi);
/* The exchange before every SpMV of rank `rank` (host only), from every
 * rank's rows (row_start) and window: for each peer q its own rows
 * [send_lo[q], send_hi[q]) go to q and x[recv_lo[q], recv_hi[q]) comes from
 * q; empty ranges have lo == hi. Replaces the reference's host gather of x
 * around each split SpMV (cudaFunction.cu:1942-2226). */
ks_status ks_halo_plan(int nranks, int rank, const int64_t *row_start, const int64_t *win_lo,
                       const int64_t *win_hi, int64_t *send_lo, int64_t *send_hi,
                       int64_t *recv_lo, int64_t *recv_hi);

/* A row-split solve: every rank (one GPU each, one process or host thread
 * each) holds a contiguous block of rows and runs the same calls. */
typedef struct ks_comm ks_comm;
/* NCCL transport, libnccl.so.2 loaded at run time: rank 0 makes the 128-byte
 * id, the caller hands it to the other ranks (e.g. over torch.distributed),
 * and every rank joins with the context of its own GPU. KS_UNIMPLEMENTED when
 * NCCL cannot be loaded. */
ks_status ks_comm_unique_id(void *id128);
ks_status ks_comm_create_nccl(ks_ctx *ctx, int nranks, int rank,
                              const void *id128, ks_comm **out);
/* Ranks emulated inside one process (e.g. several contexts on one GPU): the
 * same split solve, the halo copied device to device from the peer's vector
 * and the dots summed by a kernel in rank order, with CUDA events ordering the
 * streams. Every rank's calls must come from its own host thread; a rank that
 * does not arrive within 120 s ends the others' calls with KS_TIMEOUT. */
ks_status ks_comm_create_local(ks_ctx *const *ctxs, int nranks, ks_comm **comms);
ks_status ks_comm_destroy(ks_comm *comm);
ks_status ks_comm_info(const ks_comm *comm, int *nranks, int *rank);
/* This rank's rows r0..r1-1 of an n_global x n_global matrix (global column
 * indices; ptr holds r1 - r0 + 1 offsets of any base) and, with
 * KS_MAT_TRANSPOSE, the same rows of A^T (tptr/tcol/tval). Every rank calls
 * it with its own block, blocks contiguous in rank order (ks_partition_rows
 * gives one). ks_solve / ks_solve_host / ks_spmv / ks_adjoint_grad /
 * ks_pattern_grad on the result take vectors of the local length r1 - r0
 * (grad_val: the local nonzeros) and run the split method: before each SpMV the
 * halo of the input vector comes from the peers (ks_halo_plan), and every
 * reduction is summed over the ranks before its scalar step, so every rank
 * takes the same decisions. Replaces the reference's two-GPU split
 * (cudaFunction.cu:1942-2226), which gathers all of x through the host. */
ks_status ks_dist_upload(ks_ctx *ctx, ks_comm *comm, int64_t n_global,
                         int64_t r0, int64_t r1, const int32_t *ptr,
                         const int32_t *col, const double *val,
                         const int32_t *tptr, const int32_t *tcol,
                         const double *tval, unsigned flags, ks_mat **out);
/* Global size, own rows and the vector window [ext_lo, ext_hi) of a split
 * matrix (a single-GPU matrix reports 0..n for all). */
ks_status ks_mat_dist_info(const ks_mat *mat, int64_t *n_global, int64_t *r0,
                           int64_t *r1, int64_t *ext_lo, int64_t *ext_hi);

/* Matrix Market coordinate files: the input source the reference declares
 * (-P / -D / -M, solver_collection.cpp:278-286,505-601) but never reads.
 * Fields real / double / integer / pattern (pattern entries are 1.0);
 * symmetry general / symmetric / skew-symmetric (mirrored to both
 * triangles); square matrices only. The CSR rows are ordered by column and
 * entries repeated at one position are summed in file order. The header call
 * parses the file and returns n and the CSR nnz; ks_mm_read fills
 * caller-allocated ptr[n+1], col[nnz], val[nnz]. Complex fields and the dense
 * array format give KS_BAD_INPUT, a missing file KS_IO_ERROR. */
ks_status ks_mm_read_header(const char *file, int64_t *n, int64_t *nnz);
ks_status ks_mm_read(const char *file, int64_t n, int64_t nnz, int32_t *ptr,
                     int32_t *col, double *val);

#ifdef __cplusplus
}
#endif
#endif /* KRYLOV_SM100_H */
