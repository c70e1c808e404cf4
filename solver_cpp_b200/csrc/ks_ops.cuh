// Element-wise operations (functors for vec_kernel / spmv_kernel) and the
// tall-skinny block kernels used by GMRES, GCR and the k-skip methods.
#pragma once

#include "ks_kernels.cuh"

namespace ks {

// ------------------------------------------------------------------ basic ops
template <class T>
struct FillOp {
  T *y;
  T v;
  static constexpr int ND = 0;
  __device__ void elem(long long i, double (&)[1]) const { y[i] = v; }
  __device__ void finish(const double (&)[1]) const {}
};

template <class S, class D>
struct ConvertOp {  // b = (D) a
  const S *a;
  D *b;
  static constexpr int ND = 0;
  struct Regs {
    S a;
  };
  __device__ Regs load(long long i) const { return {a[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const { b[i] = (D)g.a; }
  __device__ void finish(const double (&)[1]) const {}
};

// out = (x, y) into a device double.
template <class T>
struct DotOp {
  const T *x;
  const T *y;
  double *out;
  static constexpr int ND = 1;
  struct Regs {
    T x, y;
  };
  __device__ Regs load(long long i) const { return {x[i], y[i]}; }
  __device__ void store(long long, const Regs &g, double (&acc)[1]) const {
    acc[0] = add_rn(acc[0], mul_rn(widen(g.x), widen(g.y)));
  }
  __device__ void finish(const double (&s)[1]) const { *out = s[0]; }
};

// y = (a*x) + y  (blas::Scalar_axy), a from the host or from a device slot.
template <class T>
struct AxpyOp {
  const T *x;
  T *y;
  double a;
  const double *a_dev;  // if set, a = sign * (*a_dev)
  double sign;
  static constexpr int ND = 0;
  __device__ void elem(long long i, double (&)[1]) const {
    const T av = (T)(a_dev ? sign * (*a_dev) : a);
    y[i] = add_rn(mul_rn(av, x[i]), y[i]);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// y = (a*x) + y, then out = (y, w).
template <class T>
struct AxpyDotOp {
  const T *x;
  T *y;
  const T *w;
  double a;
  double *out;
  static constexpr int ND = 1;
  __device__ void elem(long long i, double (&acc)[1]) const {
    const T v = add_rn(mul_rn((T)a, x[i]), y[i]);
    y[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(v), widen(w ? w[i] : v)));
  }
  __device__ void finish(const double (&s)[1]) const { *out = s[0]; }
};

// y = A x (plain SpMV store).
template <class YT, class AT>
struct StoreEpi {
  using acc_t = AT;
  YT *y;
  static constexpr int ND = 0;
  __device__ void row(int r, AT v, double (&)[1]) const { y[r] = (YT)v; }
  // 4 consecutive rows from r (a multiple of 4; y aligned: dia_quad_ok)
  __device__ void row4(int r, const AT (&v)[4]) const {
    if constexpr (sizeof(YT) == 4) {
      *reinterpret_cast<float4 *>(y + r) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
    } else {
      reinterpret_cast<double2 *>(y + r)[0] = make_double2((double)v[0], (double)v[1]);
      reinterpret_cast<double2 *>(y + r)[1] = make_double2((double)v[2], (double)v[3]);
    }
  }
  __device__ void finish(const double (&)[1]) const {}
};

// r = b - A x; out[0] = (r, r); out[1] = (b, b).
template <class T>
struct ResidEpi {
  using acc_t = T;
  const T *b;
  T *r;  // may be null (norms only)
  double *out;
  static constexpr int ND = 2;
  __device__ void row(int i, T v, double (&acc)[2]) const {
    const T bi = b[i];
    const T ri = sub_rn(bi, v);
    if (r) r[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
    acc[1] = add_rn(acc[1], mul_rn(widen(bi), widen(bi)));
  }
  __device__ void finish(const double (&s)[2]) const {
    out[0] = s[0];
    out[1] = s[1];
  }
};

// grad[j] = -lambda[row] * x[col[j]] over the CSR pattern (adjoint gather).
__global__ void pattern_grad_kernel(CsrK<double> A, const double *__restrict__ lam,
                                    const double *__restrict__ x, double *__restrict__ g);

// ------------------------------------------------------------ block (tall-skinny)
// h[w][i] = (W_w, V_i) for i < k and NW left vectors W (1 or 2): one pass over
// the k basis vectors V_i = V + i*ld, kBlockDotGroup of them per group. The
// group is the fast grid index (blockIdx.x) and the slice of the vectors the
// slow one (blockIdx.y): the CTAs of every group that read the same slice of
// W run together, so W comes from DRAM about once rather than once per group.
// Each group is reduced deterministically with its own counter;
// Epi::put(w, i, value) receives every result (thread 0 of the group's last CTA).
template <int NW, class VT, class Epi>
__global__ void __launch_bounds__(kThreads, NW == 1 ? 4 : 2)
    block_dot_kernel(const VT *__restrict__ V, long long ld, int k,
                     const VT *__restrict__ W0, const VT *__restrict__ W1, long long n,
                     Epi epi, Stop stop, double *partials, unsigned *counters) {
  pdl_wait();
  if (stop()) return;
  constexpr int G8 = kBlockDotGroup;
  const int g = blockIdx.x;
  const int slice = blockIdx.y, nslices = gridDim.y;
  const int i0 = g * G8;
  const int cnt = min(G8, k - i0);
  double acc[NW * G8];
#pragma unroll
  for (int q = 0; q < NW * G8; q++) acc[q] = 0.0;
  const long long stride = (long long)nslices * kThreads;
  for (long long j = (long long)slice * kThreads + threadIdx.x; j < n; j += stride) {
    const double w0 = widen(W0[j]);
    const double w1 = NW > 1 ? widen(W1[j]) : 0.0;
#pragma unroll
    for (int q = 0; q < G8; q++) {
      if (q < cnt) {
        const double v = widen(V[(long long)(i0 + q) * ld + j]);
        acc[q] = add_rn(acc[q], mul_rn(w0, v));
        if (NW > 1) acc[G8 + q] = add_rn(acc[G8 + q], mul_rn(w1, v));
      }
    }
  }
  pdl_trigger();
  double *part = partials + (size_t)g * NW * G8 * nslices;
  if (grid_sum_n<NW * G8>(acc, part, counters + g, nslices, slice) && threadIdx.x == 0) {
    for (int q = 0; q < cnt; q++) {
      epi.put(0, i0 + q, acc[q]);
      if (NW > 1) epi.put(1, i0 + q, acc[G8 + q]);
    }
  }
}

struct PutArray {  // out[w * stride_w + i * stride_i] = value
  double *out;
  long long stride_w, stride_i;
  __device__ void put(int w, int i, double v) const { out[w * stride_w + i * stride_i] = v; }
};

// Split solves: the block dot leaves its results in the stage (w * k + i)
// and, once they are summed over the ranks, a scalar step hands each to the
// real epilogue.
template <class Epi>
struct StagePuts {
  double *stage;
  int k;
  __device__ void put(int w, int i, double v) const { stage[(long long)w * k + i] = v; }
};

template <class Epi>
struct PutSummed {
  Epi epi;
  const double *stage;
  int nw, k;
  __device__ void run() const {
    for (int w = 0; w < nw; w++)
      for (int i = 0; i < k; i++) epi.put(w, i, stage[(long long)w * k + i]);
  }
};

template <int NW, class VT, class Epi>
inline ks_status launch_block_dot(ks_ctx *ctx, const VT *V, long long ld, int k, const VT *W0,
                                  const VT *W1, long long n, const Epi &epi, Stop stop) {
  if (k <= 0) return KS_OK;
  const int groups = (k + kBlockDotGroup - 1) / kBlockDotGroup;
  if (groups > kMaxGroups)
    return set_error(ctx, KS_BAD_INPUT, "block dot: more than 1024 basis vectors in one pass");
  int gx = red_grid(ctx);
  const long long need = (n + kThreads - 1) / kThreads;
  if (need < gx) gx = (int)std::max<long long>(need, 1);
  dim3 grid(groups, gx);
  if (ctx->red_comm) {  // split solve: results summed over the ranks, then put
    if (NW * k > kStageLen) return set_error(ctx, KS_BAD_INPUT, "block dot: too many results for a split solve");
    ctx->next_class = kDot;
    launch_k(ctx, block_dot_kernel<NW, VT, StagePuts<Epi>>, grid, dim3(kThreads), 0, V, ld, k, W0, W1, n,
             StagePuts<Epi>{ctx->d_stage, k}, stop, ctx->partials, ctx->counters + 16);
    note_dist(ctx, ctx->red_comm->allreduce(ctx->d_stage, NW * k));
    launch_scalar(ctx, PutSummed<Epi>{epi, ctx->d_stage, NW, k}, stop);
    return KS_OK;
  }
  ctx->next_class = kDot;
  launch_k(ctx, block_dot_kernel<NW, VT, Epi>, grid, dim3(kThreads), 0, V, ld, k, W0, W1, n, epi, stop,
           ctx->partials, ctx->counters + 16);
  return KS_OK;
}

// w[j] -= h[i] * V_i[j] for i = 0..k-1 in order (blas::Gmres_sp_1,
// blas.cpp:477-488), h read from device memory; optionally out = (w, w), or
// its square root (the new basis vector's norm, GMRES). Runs in basis_kernel.
template <class VT>
struct BlockAxpyOp {
  using vt = VT;
  static constexpr int NB = 1, ND = 1;
  const VT *V;
  long long ld;
  int k;
  const double *h;
  long long hstride;
  VT *w;
  double *out;  // (w,w) after the update if not null
  int take_sqrt = 0;
  struct St {
    VT t;
  };
  __device__ bool active() const { return true; }
  __device__ int count() const { return k; }
  __device__ const VT *base(int) const { return V; }
  __device__ St init(long long j) const { return {w[j]}; }
  __device__ void step(St &s, int i, const VT (&v)[1]) const {
    s.t = sub_rn(s.t, mul_rn((VT)__ldg(h + i * hstride), v[0]));
  }
  __device__ void done(long long j, const St &s, double (&acc)[1]) const {
    w[j] = s.t;
    acc[0] = add_rn(acc[0], mul_rn(widen(s.t), widen(s.t)));
  }
  __device__ void finish(const double (&s)[1]) const {
    if (out) *out = take_sqrt ? sqrt(s[0]) : s[0];
  }
};

}  // namespace ks
