// Primitive operations of the C ABI: SpMV, dots, AXPY, tall-skinny block
// operations, k-skip matrix powers and Gram values, adjoint pattern gather.
#include <cmath>

#include "ks_dist.cuh"
#include "ks_ops.cuh"

namespace ks {

__global__ void pattern_grad_kernel(CsrK<double> A, const double *__restrict__ lam,
                                    const double *__restrict__ x, double *__restrict__ g) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < A.n; r += gridDim.x * blockDim.x) {
    const double l = -lam[r];
    for (int j = A.ptr[r]; j < A.ptr[r + 1]; j++) g[j] = mul_rn(l, __ldg(x + A.col[j]));
  }
}

static const CsrDev *pick(const ks_mat *m, int trans) { return trans ? &m->T : &m->A; }

// y = A x with the matrix values in `vals` precision and vector types from x/y.
ks_status spmv_any(ks_ctx *ctx, const CsrDev &A, ks_precision vals, ks_precision vt,
                   const void *x, void *y, Stop stop) {
  if (vt == KS_FP64) {
    if (vals != KS_FP64) return set_error(ctx, KS_BAD_INPUT, "FP64 vectors need FP64 values");
    launch_spmv<double, double>(ctx, A, (const double *)x, StoreEpi<double, double>{(double *)y}, stop);
  } else if (vt == KS_FP32) {
    if (vals == KS_FP32) {
      if (!A.val32) return set_error(ctx, KS_BAD_INPUT, "matrix has no FP32 values (KS_MAT_FP32)");
      launch_spmv<float, float>(ctx, A, (const float *)x, StoreEpi<float, float>{(float *)y}, stop);
    } else if (vals == KS_BF16) {
      if (!A.val16) return set_error(ctx, KS_BAD_INPUT, "matrix has no BF16 values (KS_MAT_BF16)");
      launch_spmv<__nv_bfloat16, float>(ctx, A, (const float *)x, StoreEpi<float, float>{(float *)y},
                                        stop);
    } else {
      return set_error(ctx, KS_BAD_INPUT, "FP32 vectors need FP32 or BF16 values");
    }
  } else {
    return set_error(ctx, KS_BAD_INPUT, "vectors must be FP64 or FP32");
  }
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

static ks_status fetch(ks_ctx *ctx, int count, double *host) {
  KS_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_result, sizeof(double) * count,
                               cudaMemcpyDeviceToHost, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < count; i++) host[i] = ctx->h_pinned[i];
  return check_device_error(ctx);
}

static bool same_ctx(const ks_vec *a, const ks_vec *b) { return a && b && a->ctx == b->ctx; }

// True when p is device memory of the context's GPU (cudaMalloc, a torch
// tensor): the tall-skinny block calls then keep their k values there,
// ordered on the context's stream, with no copy and no synchronisation.
static bool on_ctx_device(const ks_ctx *ctx, const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // plain host memory on older drivers
    return false;
  }
  return a.type == cudaMemoryTypeDevice && a.device == ctx->device;
}

}  // namespace ks

using namespace ks;

extern "C" {

ks_status ks_spmv_values(const ks_mat *mat, int trans, ks_precision values, const ks_vec *x,
                         ks_vec *y) {
  if (!mat || !x || !y || x->ctx != mat->ctx || y->ctx != mat->ctx) return KS_BAD_INPUT;
  ks_ctx *ctx = mat->ctx;
  if (trans && !mat->has_T) return set_error(ctx, KS_BAD_INPUT, "transpose not built (KS_MAT_TRANSPOSE)");
  const CsrDev &A = *pick(mat, trans);
  if (x->n < A.n || y->n < A.n || x->type != y->type)
    return set_error(ctx, KS_BAD_INPUT, "spmv: vector length or type mismatch");
  if (mat->dist) {  // split rows: x into a window-sized buffer, halo from the peers
    const DistInfo &d = *mat->dist;
    const size_t es = elem_size(x->type);
    void *buf = nullptr;
    KS_TRY(pool_get(ctx, es * (size_t)d.ld() + 64, &buf));
    char *xl = (char *)buf + d.off() * (long long)es;
    const cudaError_t e = cudaMemcpyAsync(xl, x->d, es * (size_t)A.n, cudaMemcpyDeviceToDevice, ctx->stream);
    ks_status s = e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "spmv copy");
    if (s == KS_OK) s = d.comm->exchange(trans ? d.planT : d.planA, xl, es);
    if (s == KS_OK) s = spmv_any(ctx, A, values, x->type, xl, y->d, Stop{nullptr, nullptr});
    pool_release(ctx, buf);  // later users of the pool are queued behind this SpMV
    return s;
  }
  return spmv_any(ctx, A, values, x->type, x->d, y->d, Stop{nullptr, nullptr});
}

ks_status ks_spmv(const ks_mat *mat, int trans, const ks_vec *x, ks_vec *y) {
  if (!x) return KS_BAD_INPUT;
  return ks_spmv_values(mat, trans, x->type == KS_FP64 ? KS_FP64 : KS_FP32, x, y);
}

ks_status ks_dot(const ks_vec *x, const ks_vec *y, double *result) {
  if (!same_ctx(x, y) || !result || x->type != y->type || x->n != y->n) return KS_BAD_INPUT;
  ks_ctx *ctx = x->ctx;
  if (x->type == KS_FP64)
    launch_vec(ctx, x->n, DotOp<double>{(const double *)x->d, (const double *)y->d, ctx->d_result},
               Stop{nullptr, nullptr});
  else if (x->type == KS_FP32)
    launch_vec(ctx, x->n, DotOp<float>{(const float *)x->d, (const float *)y->d, ctx->d_result},
               Stop{nullptr, nullptr});
  else
    return set_error(ctx, KS_BAD_INPUT, "dot supports FP64 and FP32 vectors");
  KS_CUDA(ctx, cudaGetLastError());
  return fetch(ctx, 1, result);
}

ks_status ks_nrm2(const ks_vec *x, double *result) {
  KS_TRY(ks_dot(x, x, result));
  *result = std::sqrt(*result);
  return KS_OK;
}

ks_status ks_axpy(double a, const ks_vec *x, ks_vec *y) {
  if (!same_ctx(x, y) || x->type != y->type || x->n != y->n) return KS_BAD_INPUT;
  ks_ctx *ctx = x->ctx;
  if (x->type == KS_FP64)
    launch_vec(ctx, x->n, AxpyOp<double>{(const double *)x->d, (double *)y->d, a, nullptr, 1.0},
               Stop{nullptr, nullptr});
  else if (x->type == KS_FP32)
    launch_vec(ctx, x->n, AxpyOp<float>{(const float *)x->d, (float *)y->d, a, nullptr, 1.0},
               Stop{nullptr, nullptr});
  else
    return set_error(ctx, KS_BAD_INPUT, "axpy supports FP64 and FP32 vectors");
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

ks_status ks_axpy_dot(double a, const ks_vec *x, ks_vec *y, const ks_vec *w, double *result) {
  if (!same_ctx(x, y) || x->type != y->type || x->n != y->n || !result) return KS_BAD_INPUT;
  if (w && (!same_ctx(x, w) || w->type != x->type || w->n != x->n)) return KS_BAD_INPUT;
  ks_ctx *ctx = x->ctx;
  if (x->type == KS_FP64)
    launch_vec(ctx, x->n,
               AxpyDotOp<double>{(const double *)x->d, (double *)y->d,
                                 w ? (const double *)w->d : nullptr, a, ctx->d_result},
               Stop{nullptr, nullptr});
  else if (x->type == KS_FP32)
    launch_vec(ctx, x->n,
               AxpyDotOp<float>{(const float *)x->d, (float *)y->d, w ? (const float *)w->d : nullptr,
                                a, ctx->d_result},
               Stop{nullptr, nullptr});
  else
    return set_error(ctx, KS_BAD_INPUT, "axpy_dot supports FP64 and FP32 vectors");
  KS_CUDA(ctx, cudaGetLastError());
  return fetch(ctx, 1, result);
}

ks_status ks_block_dot(const ks_vec *V, int64_t ld, int k, const ks_vec *w, double *h) {
  if (!same_ctx(V, w) || !h || k < 0 || V->type != KS_FP64 || w->type != KS_FP64) return KS_BAD_INPUT;
  ks_ctx *ctx = V->ctx;
  const long long n = w->n;
  if (k == 0) return KS_OK;
  if (ld < n || (long long)(k - 1) * ld + n > V->n || (size_t)k > ctx->d_result_len)
    return set_error(ctx, KS_BAD_INPUT, "block_dot: basis does not fit");
  const bool dev = on_ctx_device(ctx, h);
  KS_TRY(launch_block_dot<1, double>(ctx, (const double *)V->d, ld, k, (const double *)w->d, nullptr, n,
                                     PutArray{dev ? h : ctx->d_result, 0, 1}, Stop{nullptr, nullptr}));
  KS_CUDA(ctx, cudaGetLastError());
  return dev ? KS_OK : fetch(ctx, k, h);
}

ks_status ks_block_axpy(const ks_vec *V, int64_t ld, int k, const double *h, ks_vec *w) {
  if (!same_ctx(V, w) || (!h && k > 0) || k < 0 || V->type != KS_FP64 || w->type != KS_FP64)
    return KS_BAD_INPUT;
  ks_ctx *ctx = V->ctx;
  const long long n = w->n;
  if (k == 0) return KS_OK;
  if (ld < n || (long long)(k - 1) * ld + n > V->n || (size_t)k > ctx->d_result_len)
    return set_error(ctx, KS_BAD_INPUT, "block_axpy: basis does not fit");
  const bool dev = on_ctx_device(ctx, h);
  if (!dev)
    KS_CUDA(ctx, cudaMemcpyAsync(ctx->d_result, h, sizeof(double) * k, cudaMemcpyHostToDevice, ctx->stream));
  launch_basis(ctx, n, k,
               BlockAxpyOp<double>{(const double *)V->d, ld, k, dev ? h : ctx->d_result, 1, (double *)w->d,
                                   nullptr},
               Stop{nullptr, nullptr});
  KS_CUDA(ctx, cudaGetLastError());
  if (!dev) KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the host array may be reused on return
  return KS_OK;
}

}  // extern "C"

namespace ks {

struct Store2Epi {
  using acc_t = double;
  double *y0, *y1;
  static constexpr int ND = 0;
  __device__ void row(int r, double a, double b, double (&)[1]) const {
    y0[r] = a;
    if (y1) y1[r] = b;
  }
  __device__ void finish(const double (&)[1]) const {}
};

// Ar[i] = A^{i+1} r (i <= 2k), Ap[i] = A^{i+1} p (i <= 2k+1); the r and p
// chains share each pass over A.
ks_status matpow(ks_ctx *ctx, const CsrDev &A, const double *r, const double *p, int k, double *Ar,
                 double *Ap, Stop stop) {
  const long long n = A.n;
  launch_spmv2<double, double>(ctx, A, r, p, Store2Epi{Ar, Ap}, stop);
  for (int i = 1; i < 2 * k + 1; i++)
    launch_spmv2<double, double>(ctx, A, Ar + (i - 1) * n, Ap + (i - 1) * n,
                                 Store2Epi{Ar + i * n, Ap + i * n}, stop);
  launch_spmv<double, double>(ctx, A, Ap + (long long)(2 * k) * n,
                              StoreEpi<double, double>{Ap + (long long)(2 * k + 1) * n}, stop);
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

// delta[i] = (r, Ar_i) i<2k; eta[i] = (r, Ap_i) i<2k+1; zeta[i] = (p, Ap_i) i<2k+2.
// eta must have room for 2k+2 entries (the last one is a by-product).
ks_status gram_cg(ks_ctx *ctx, long long n, int k, const double *Ar, const double *Ap,
                  const double *r, const double *p, double *delta, double *eta, double *zeta,
                  Stop stop) {
  if (k > 0)
    KS_TRY(launch_block_dot<1, double>(ctx, Ar, n, 2 * k, r, nullptr, n, PutArray{delta, 0, 1}, stop));
  KS_TRY(launch_block_dot<2, double>(ctx, Ap, n, 2 * k + 2, r, p, n,
                                     PutArray{eta, (long long)(zeta - eta), 1}, stop));
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

// theta[i] = (rs, Ar_i) i<2k; rho[i] = (ps, Ar_i) i<2k+1;
// eta[i] = (rs, Ap_i) i<2k+1; phi[i] = (ps, Ap_i) i<2k+2.
ks_status gram_bicg(ks_ctx *ctx, long long n, int k, const double *Ar, const double *Ap,
                    const double *rs, const double *ps, double *theta, double *eta, double *rho,
                    double *phi, Stop stop) {
  KS_TRY(launch_block_dot<2, double>(ctx, Ar, n, 2 * k + 1, rs, ps, n,
                                     PutArray{theta, (long long)(rho - theta), 1}, stop));
  KS_TRY(launch_block_dot<2, double>(ctx, Ap, n, 2 * k + 2, rs, ps, n,
                                     PutArray{eta, (long long)(phi - eta), 1}, stop));
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

}  // namespace ks

extern "C" {

ks_status ks_matpow(const ks_mat *mat, const ks_vec *r, const ks_vec *p, int k, ks_vec *Ar, ks_vec *Ap) {
  if (!mat || !r || !p || !Ar || !Ap || k < 0) return KS_BAD_INPUT;
  if (mat->dist) return set_error(mat->ctx, KS_UNIMPLEMENTED, "not available for split-row matrices");
  ks_ctx *ctx = mat->ctx;
  const long long n = mat->A.n;
  if (r->type != KS_FP64 || p->type != KS_FP64 || Ar->type != KS_FP64 || Ap->type != KS_FP64 ||
      r->n != n || p->n != n || Ar->n < (2 * k + 1) * n || Ap->n < (2 * k + 2) * n)
    return set_error(ctx, KS_BAD_INPUT, "matpow: FP64 vectors of n, (2k+1)n and (2k+2)n required");
  return matpow(ctx, mat->A, (const double *)r->d, (const double *)p->d, k, (double *)Ar->d,
                (double *)Ap->d, Stop{nullptr, nullptr});
}

ks_status ks_gram_cg(const ks_vec *Ar, const ks_vec *Ap, const ks_vec *r, const ks_vec *p, int k,
                     double *delta, double *eta, double *zeta) {
  if (!Ar || !Ap || !r || !p || k < 0 || !eta || !zeta || (k > 0 && !delta)) return KS_BAD_INPUT;
  ks_ctx *ctx = r->ctx;
  const long long n = r->n;
  if (Ar->n < (2 * k + 1) * n || Ap->n < (2 * k + 2) * n || p->n != n ||
      (size_t)(6 * k + 4) > ctx->d_result_len || 8 * k + 8 > 4096)
    return set_error(ctx, KS_BAD_INPUT, "gram_cg: sizes");
  double *d = ctx->d_result, *e = d + 2 * k, *z = e + 2 * k + 2;
  KS_TRY(gram_cg(ctx, n, k, (const double *)Ar->d, (const double *)Ap->d, (const double *)r->d,
                 (const double *)p->d, d, e, z, Stop{nullptr, nullptr}));
  double tmp[4096];
  KS_TRY(fetch(ctx, 6 * k + 4, tmp));
  for (int i = 0; i < 2 * k; i++) delta[i] = tmp[i];
  for (int i = 0; i < 2 * k + 1; i++) eta[i] = tmp[2 * k + i];
  for (int i = 0; i < 2 * k + 2; i++) zeta[i] = tmp[4 * k + 2 + i];
  return KS_OK;
}

ks_status ks_gram_bicg(const ks_vec *Ar, const ks_vec *Ap, const ks_vec *rs, const ks_vec *ps, int k,
                       double *theta, double *eta, double *rho, double *phi) {
  if (!Ar || !Ap || !rs || !ps || k < 0 || !eta || !rho || !phi || (k > 0 && !theta)) return KS_BAD_INPUT;
  ks_ctx *ctx = rs->ctx;
  const long long n = rs->n;
  if (Ar->n < (2 * k + 1) * n || Ap->n < (2 * k + 2) * n || ps->n != n ||
      (size_t)(8 * k + 8) > ctx->d_result_len || 8 * k + 8 > 4096)
    return set_error(ctx, KS_BAD_INPUT, "gram_bicg: sizes");
  // layout: theta[2k+1] (one spare), rho[2k+1], eta[2k+2] (one spare), phi[2k+2]
  double *t = ctx->d_result, *ro = t + 2 * k + 1, *e = ro + 2 * k + 1, *f = e + 2 * k + 2;
  KS_TRY(gram_bicg(ctx, n, k, (const double *)Ar->d, (const double *)Ap->d, (const double *)rs->d,
                   (const double *)ps->d, t, e, ro, f, Stop{nullptr, nullptr}));
  double tmp[4096];
  KS_TRY(fetch(ctx, 8 * k + 6, tmp));
  for (int i = 0; i < 2 * k; i++) theta[i] = tmp[i];
  for (int i = 0; i < 2 * k + 1; i++) rho[i] = tmp[2 * k + 1 + i];
  for (int i = 0; i < 2 * k + 1; i++) eta[i] = tmp[4 * k + 2 + i];
  for (int i = 0; i < 2 * k + 2; i++) phi[i] = tmp[6 * k + 4 + i];
  return KS_OK;
}

ks_status ks_pattern_grad(const ks_mat *mat, const ks_vec *lambda, const ks_vec *x, ks_vec *grad_val) {
  if (!mat || !lambda || !x || !grad_val) return KS_BAD_INPUT;
  ks_ctx *ctx = mat->ctx;
  if (lambda->type != KS_FP64 || x->type != KS_FP64 || grad_val->type != KS_FP64 ||
      lambda->n != mat->A.n || x->n != mat->A.n || grad_val->n < mat->A.nnz)
    return set_error(ctx, KS_BAD_INPUT, "pattern_grad: FP64 vectors of n, n, nnz required");
  const double *xs = (const double *)x->d;
  void *buf = nullptr;
  if (mat->dist) {  // split rows: the columns reach into the halo, so x goes into a window first
    const DistInfo &d = *mat->dist;
    KS_TRY(pool_get(ctx, sizeof(double) * (size_t)d.ld() + 64, &buf));
    double *xl = (double *)buf + d.off();
    const cudaError_t e =
        cudaMemcpyAsync(xl, x->d, sizeof(double) * (size_t)mat->A.n, cudaMemcpyDeviceToDevice, ctx->stream);
    ks_status s = e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "pattern_grad copy");
    if (s == KS_OK) s = d.comm->exchange(d.planA, xl, sizeof(double));
    if (s != KS_OK) {
      pool_release(ctx, buf);
      return s;
    }
    xs = xl;
  }
  pattern_grad_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(view<double>(mat->A), (const double *)lambda->d,
                                                                  xs, (double *)grad_val->d);
  const cudaError_t e = cudaGetLastError();
  if (buf) pool_release(ctx, buf);  // later users of the pool are queued behind the gather
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pattern_grad");
  return KS_OK;
}

ks_status ks_check_error(const ks_mat *mat, const ks_vec *b, const ks_vec *x, double *log10_ratio,
                         double *rel) {
  if (!mat || !b || !x || b->type != KS_FP64 || x->type != KS_FP64) return KS_BAD_INPUT;
  if (mat->dist) return set_error(mat->ctx, KS_UNIMPLEMENTED, "not available for split-row matrices");  // ks_solve reports it
  ks_ctx *ctx = mat->ctx;
  launch_spmv<double, double>(ctx, mat->A, (const double *)x->d,
                              ResidEpi<double>{(const double *)b->d, nullptr, ctx->d_result},
                              Stop{nullptr, nullptr});
  KS_CUDA(ctx, cudaGetLastError());
  double s[2];
  KS_TRY(fetch(ctx, 2, s));
  const double ratio = std::sqrt(s[0]) / std::sqrt(s[1]);
  if (log10_ratio) *log10_ratio = std::log10(ratio);
  if (rel) *rel = ratio;
  return KS_OK;
}

}  // extern "C"
