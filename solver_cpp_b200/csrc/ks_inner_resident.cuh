// The inner CG of a VP method with its vectors on chip (sm_100a).
//
// A VP method's inner solve (innerMethods.cpp:71-118, here CG of a fixed
// number of iterations in FP32, or with BF16 matrix values) runs thousands of
// times; launched kernel by kernel, each iteration streams r, p, q and x
// through L2/HBM and pays three kernel boundaries. This kernel runs the whole
// inner solve in one cooperative launch of one CTA per SM. CTA b owns rows
// [b*rpc, (b+1)*rpc); thread t of it owns the rows b*rpc + t + 1024 k:
//   * r and q of its rows live in tensor memory (TMEM, 256 KB per SM, which
//     no tensor-core work needs here): warp w reaches TMEM lanes
//     32 (w % 4) .. +31 and takes columns 64 (w / 4) .. +63 of them, so every
//     thread has 64 private 32-bit words: r_k in the first 32, q_k in the
//     other 32 (k < kIrMaxK),
//   * p and x of the CTA's rows live in shared memory (2 * rpc floats); p is
//     also published to a global array P from which the other CTAs gather it,
//     x is written out once, at the end,
//   * the matrix (the diagonal copy, FP32 or BF16 values, either layout) is
//     read from global memory (L2) every iteration; the registers left free
//     keep the loads of two rows in flight per thread.
// The TMEM columns are allocated once per launch and released on every way
// out of the kernel (a timed-out wait included).
// Per iteration (cg.cpp:184-240):
//   A: q = A p (own p from shared memory, other CTAs' from P), (p, q) summed
//      over the grid -> alpha = (r, r) / (p, q);
//   B: x += alpha p, r -= alpha q, (r, r) summed -> beta, stopping test;
//   C: p = beta p + r, published; a grid barrier.
// Each element sees the FP32 operations of the kernel-per-step loop
// (CgMvEpi, XrUpdOp, XpbyToOp) in the same order; only the order in which
// the dot products add their terms differs (per thread over its rows, a
// fixed tree over the CTA, then the CTAs' partials in index order: the same
// in every run). Every CTA computes alpha, beta and the stopping decision
// from the same sums, so all leave the loop together.
//
// Grid reductions: each CTA adds its partial to a monotonic arrival counter;
// the last to arrive sums the partials in index order and publishes the
// result with a release store of the generation; the others wait for it with
// acquire loads, bounded by the context's wait limit. A wait that runs out
// sets the context's timeout flag and ends the kernel (the caller returns
// KS_TIMEOUT); every CTA is resident (cooperative launch), so the waits end
// as soon as the last CTA arrives.
#pragma once

#include "ks_kernels.cuh"
#include "ks_state.cuh"

namespace ks {

constexpr int kIrThreads = 1024;  // threads per CTA, one CTA per SM
constexpr int kIrMaxK = 32;       // rows per thread (r and q in 64 TMEM columns)
constexpr int kIrWarps = kIrThreads / 32;

// Barrier state in device memory, zeroed before every launch.
struct IrSync {
  unsigned long long count;  // CTA arrivals, all generations
  unsigned long long flag;   // the last completed generation
  double result[2];
};

struct IrArgs {
  const float *rin;  // the inner right-hand side, rounded to FP32 (n)
  float *x;          // the inner solution z (n)
  float *P;          // published directions (n)
  DevState *st;      // the inner method's state
  const int *outer_done;
  double *partials;  // 2 per CTA
  IrSync *sync;
  int *err;
  unsigned long long wait_ns;
  int n;
  int rpc;  // rows per CTA, a multiple of 32
  int K;    // rows per thread: ceil(rpc / kIrThreads) <= kIrMaxK
};

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Sums of two values over the CTA's 1024 threads in a fixed order; the
// result is valid in thread 0.
__device__ __forceinline__ void ir_block_sum(double (&v)[2], double (*sh)[kIrWarps]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < 2; d++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[d] += __shfl_down_sync(0xffffffffu, v[d], o);
  }
  if (lane == 0) {
    sh[0][w] = v[0];
    sh[1][w] = v[1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int i = 0; i < kIrWarps; i++) {
      s0 += sh[0][i];
      s1 += sh[1][i];
    }
    v[0] = s0;
    v[1] = s1;
  }
}

// Grid-wide sums of (v0, v1), the same in every CTA; also a barrier (every
// store the CTA's threads made before it is visible to every CTA after it).
// Returns false when a wait ran out (the timeout flag is then set).
__device__ __forceinline__ bool ir_allreduce(const IrArgs &a, unsigned long long gen, double (&v)[2]) {
  __shared__ double sh[2][kIrWarps];
  __shared__ double s_res[2];
  __shared__ int s_state;  // 1: last to arrive, 2: waited, 0: timed out
  ir_block_sum(v, sh);
  const unsigned G = gridDim.x;
  if (threadIdx.x == 0) {
    a.partials[2 * blockIdx.x] = v[0];
    a.partials[2 * blockIdx.x + 1] = v[1];
    __threadfence();
    const unsigned long long old = atomicAdd(&a.sync->count, 1ull);
    s_state = (old + 1 == gen * (unsigned long long)G) ? 1 : 2;
  }
  __syncthreads();
  if (s_state == 1) {
    if (threadIdx.x < 32) {
      __threadfence();
      double s0 = 0.0, s1 = 0.0;
      for (unsigned b = threadIdx.x; b < G; b += 32) {
        s0 += __ldcg(&a.partials[2 * b]);
        s1 += __ldcg(&a.partials[2 * b + 1]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
      }
      if (threadIdx.x == 0) {
        s_res[0] = s0;
        s_res[1] = s1;
        a.sync->result[0] = s0;
        a.sync->result[1] = s1;
        __threadfence();
        st_release_u64(&a.sync->flag, gen);
      }
    }
  } else if (threadIdx.x == 0) {
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u64(&a.sync->flag) < gen) {
      if (global_ns() - t0 > a.wait_ns) {
        atomicExch(a.err, 1);
        s_state = 0;
        break;
      }
    }
    if (s_state) {
      s_res[0] = __ldcg(&a.sync->result[0]);
      s_res[1] = __ldcg(&a.sync->result[1]);
    }
  }
  __syncthreads();
  if (!s_state) return false;
  v[0] = s_res[0];
  v[1] = s_res[1];
  return true;
}

template <class MT>
__device__ __forceinline__ MT ir_ld(const MT *p) {
  return __ldg(p);
}
template <>
__device__ __forceinline__ __nv_bfloat16 ir_ld<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __ushort_as_bfloat16(__ldg(reinterpret_cast<const unsigned short *>(p)));
}

// ---------------------------------------------------------------- TMEM access
__device__ __forceinline__ void tm_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tm_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tm_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tm_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 2 consecutive columns of this warp's 32 lanes (one word per column per thread)
__device__ __forceinline__ void tm_st2(uint32_t taddr, float a, float b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(__float_as_uint(a)),
               "r"(__float_as_uint(b))
               : "memory");
}
__device__ __forceinline__ void tm_ld2(uint32_t taddr, float &a, float &b) {
  uint32_t u0, u1;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(u0), "=r"(u1) : "r"(taddr) : "memory");
  // the registers are valid only after the wait; passing them through it
  // keeps every use behind it
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(u0), "+r"(u1)::"memory");
  a = __uint_as_float(u0);
  b = __uint_as_float(u1);
}
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

constexpr uint32_t kIrTmemCols = 512;

// y_row = sum_d A[row][row + off_d] * p[row + off_d] for one row, p from the
// CTA's shared copy or, for other CTAs' rows, from P (every diagonal's value
// loaded, zeros where the row has none: FP32 sums as in the SpMV kernel).
template <class MT, int NDG>
struct IrRow {
  MT av[NDG > 0 ? NDG : kMaxDiag];
  float pv[NDG > 0 ? NDG : kMaxDiag];
  __device__ __forceinline__ void load(const DiaT<MT> &D, const IrArgs &a, const float *sp, int r0, int nr, int i,
                                       int nd) {
    constexpr int KD = NDG > 0 ? NDG : kMaxDiag;
#pragma unroll
    for (int d = 0; d < KD; d++) {
      if (NDG > 0 || d < nd) {
        av[d] = ir_ld(D.vb[d] + (i + D.vs[d]));
        const int c = min(max(i + D.off[d], D.cmin), D.cmax - 1);
        const int lc = c - r0;
        pv[d] = (lc >= 0 && lc < nr) ? sp[lc] : __ldcg(a.P + c);
      }
    }
  }
  __device__ __forceinline__ float sum(int nd) const {
    constexpr int KD = NDG > 0 ? NDG : kMaxDiag;
    float q = 0.f;
#pragma unroll
    for (int d = 0; d < KD; d++)
      if (NDG > 0 || d < nd) q = add_rn(q, mul_rn(mval<float>(av[d]), pv[d]));
    return q;
  }
};

// The inner solve (see the top of this file). Returns the stopping code, or
// -1 when a wait ran out; *xw: x was written (one update at least).
template <class MT, int NDG>
__device__ __forceinline__ int ir_body(const DiaT<MT> &D, const IrArgs &a, float *sp, float *sx, uint32_t tm,
                                       long long *Lout, double *alpha_out, double *beta_out, double *rr_out,
                                       bool *xw) {
  const int nd = NDG > 0 ? NDG : D.nd;
  const int t = threadIdx.x;
  const int r0 = blockIdx.x * a.rpc;
  const int nr = max(0, min(a.rpc, a.n - r0));
  DevState *st = a.st;
  const double eps = st->k.s[S_EPS];
  const double bnorm = st->k.s[S_BNORM];
  const long long maxloop = st->k.aux[A_MAXLOOP];
  double rr = st->k.s[S_RR];
  const int K2 = (a.K + 1) / 2;  // row pairs per thread
  const uint32_t tr = tm, tq = tm + 32;  // this thread's r_k at column tr + k, q_k at tq + k

  // start: r = b (TMEM), p = r (shared memory and P), x = 0
  for (int j = 0; j < K2; j++) {
    float v[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int li = t + (2 * j + u) * kIrThreads;
      v[u] = 0.f;
      if (li < nr) {
        v[u] = __ldcg(a.rin + r0 + li);
        sp[li] = v[u];
        sx[li] = 0.f;
        __stcg(a.P + r0 + li, v[u]);
      }
    }
    tm_st2(tr + 2 * j, v[0], v[1]);
  }
  tm_wait_st();
  unsigned long long gen = 0;
  double v[2] = {0.0, 0.0};
  if (!ir_allreduce(a, ++gen, v)) return -1;  // every p published

  int code = kRunning;
  double alpha = 0.0, beta = 0.0;
  long long L = 1;
  for (; L <= maxloop; L++) {
    // A: q = A p (two rows' loads in flight per thread), (p, q)
    double acc = 0.0;
    for (int j = 0; j < K2; j++) {
      const int l0 = t + 2 * j * kIrThreads, l1 = l0 + kIrThreads;
      IrRow<MT, NDG> R0, R1;
      if (l0 < nr) R0.load(D, a, sp, r0, nr, r0 + l0, nd);
      if (l1 < nr) R1.load(D, a, sp, r0, nr, r0 + l1, nd);
      float q0 = 0.f, q1 = 0.f;
      if (l0 < nr) {
        q0 = R0.sum(nd);
        acc = add_rn(acc, mul_rn(widen(sp[l0]), widen(q0)));
      }
      if (l1 < nr) {
        q1 = R1.sum(nd);
        acc = add_rn(acc, mul_rn(widen(sp[l1]), widen(q1)));
      }
      tm_st2(tq + 2 * j, q0, q1);
    }
    tm_wait_st();
    v[0] = acc;
    v[1] = 0.0;
    if (!ir_allreduce(a, ++gen, v)) return -1;
    // alpha = rr / (p, q)   (rdiv: a zero denominator is a breakdown)
    if (v[0] == 0.0) {
      code = kBreakdown;
      alpha = 0.0;
      break;
    }
    alpha = div_rn(rr, v[0]);
    if (!isfinite(alpha)) {
      code = kNaN;
      break;
    }
    // B: x += alpha p, r -= alpha q, (r, r)
    const float af = (float)alpha;
    acc = 0.0;
    for (int j = 0; j < K2; j++) {
      float rv[2], qv[2];
      tm_ld2(tr + 2 * j, rv[0], rv[1]);
      tm_ld2(tq + 2 * j, qv[0], qv[1]);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int li = t + (2 * j + u) * kIrThreads;
        if (li < nr) {
          sx[li] = add_rn(mul_rn(af, sp[li]), sx[li]);
          rv[u] = add_rn(mul_rn(-af, qv[u]), rv[u]);
          acc = add_rn(acc, mul_rn(widen(rv[u]), widen(rv[u])));
        }
      }
      tm_st2(tr + 2 * j, rv[0], rv[1]);
    }
    tm_wait_st();
    *xw = true;
    v[0] = acc;
    v[1] = 0.0;
    if (!ir_allreduce(a, ++gen, v)) return -1;
    // beta = (r, r)_new / (r, r); then the stopping test at the top of
    // iteration L + 1 (check_top), whose verdict overrides beta's
    const double rr2 = v[0];
    if (rr == 0.0) {
      code = kBreakdown;
      beta = 0.0;
    } else {
      beta = div_rn(rr2, rr);
      if (!isfinite(beta)) code = kNaN;
    }
    rr = rr2;
    const double err = sqrt(rr2) / bnorm;
    if (L + 1 > maxloop)
      code = kMaxLoop;
    else if (err <= eps)
      code = kConverged;
    else if (err != err)
      code = kNaN;
    if (code != kRunning) break;
    // C: p = beta p + r, published
    const float bf = (float)beta;
    for (int j = 0; j < K2; j++) {
      float rv[2];
      tm_ld2(tr + 2 * j, rv[0], rv[1]);
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int li = t + (2 * j + u) * kIrThreads;
        if (li < nr) {
          const float pn = add_rn(mul_rn(bf, sp[li]), rv[u]);
          sp[li] = pn;
          __stcg(a.P + r0 + li, pn);
        }
      }
    }
    if (!ir_allreduce(a, ++gen, v)) return -1;
  }
  *Lout = L;
  *alpha_out = alpha;
  *beta_out = beta;
  *rr_out = rr;
  return code;
}

template <class MT, int NDG>
__global__ void __launch_bounds__(kIrThreads, 1) k_inner_cg_resident(DiaT<MT> D, IrArgs a) {
  extern __shared__ __align__(16) float ir_smem[];
  __shared__ uint32_t s_tmem;
  float *sp = ir_smem;          // p of the CTA's rows
  float *sx = ir_smem + a.rpc;  // x of the CTA's rows
  const int t = threadIdx.x;
  DevState *st = a.st;
  // The start conditions come from kernels that completed before this one,
  // so every CTA reads the same values and all of them return here together.
  if (*(volatile const int *)a.outer_done) return;
  if (*(volatile const int *)&st->k.done != kRunning) return;  // x stays 0 (A_XZERO)
  if (t < 32) {
    tm_alloc(&s_tmem, kIrTmemCols);
    tm_relinquish();
    tm_fence_before();
  }
  __syncthreads();
  tm_fence_after();
  const uint32_t w = t >> 5;
  const uint32_t tm = s_tmem + ((32u * (w & 3u)) << 16) + 64u * (w >> 2);
  long long L = 0;
  double alpha = 0.0, beta = 0.0, rr = 0.0;
  bool xw = false;
  const int code = ir_body<MT, NDG>(D, a, sp, sx, tm, &L, &alpha, &beta, &rr, &xw);
  if (code >= 0) {
    // x out; the state the kernel-per-step loop leaves (nothing pending)
    const int r0 = blockIdx.x * a.rpc;
    const int nr = max(0, min(a.rpc, a.n - r0));
    if (xw)
      for (int li = t; li < nr; li += kIrThreads) __stcg(a.x + r0 + li, sx[li]);
    if (blockIdx.x == 0 && t == 0) {
      st->k.done = code == kRunning ? kMaxLoop : code;
      st->k.loop = code == kBreakdown || code == kNaN ? L : L + 1;
      st->k.s[S_ALPHA] = alpha;
      st->k.s[S_BETA] = beta;
      st->k.s[S_RR] = rr;
      st->k.aux[A_PENDING] = 0;
      st->k.aux[A_XZERO] = xw ? 0 : 1;
    }
  }
  // every thread's TMEM accesses are complete (each waited on its own); the
  // columns go back on every path out of the body
  tm_fence_before();
  __syncthreads();
  if (t < 32) {
    tm_fence_after();
    tm_dealloc(s_tmem, kIrTmemCols);
  }
}

// Launch shape: one CTA per SM, rows per CTA a multiple of 32.
struct IrShape {
  int G = 0, rpc = 0, K = 0;
  size_t smem = 0;
};

// False when the system does not fit: r of a thread's rows in registers
// (K <= kIrMaxK), p and q of a CTA's rows in shared memory.
inline bool ir_shape(const ks_ctx *ctx, long long n, IrShape *s) {
  if (n < 1) return false;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  const long long G = ctx->num_sms;
  const long long rpc = ((n + G - 1) / G + 31) / 32 * 32;
  const long long K = (rpc + kIrThreads - 1) / kIrThreads;
  const size_t smem = sizeof(float) * 2 * (size_t)rpc;
  if (K > kIrMaxK || smem + 2048 > (size_t)optin) return false;  // room for the static shared arrays
  s->G = (int)G;
  s->rpc = (int)rpc;
  s->K = (int)K;
  s->smem = smem;
  return true;
}

// Cooperative launch of one CTA per SM; `probe`: only check that the grid
// can be co-resident (sets *fits).
template <class MT, int NDG>
inline cudaError_t ir_launch_n(ks_ctx *ctx, const CsrDev &A, const IrArgs &a, const IrShape &sh, bool probe,
                               bool *fits) {
  auto fn = k_inner_cg_resident<MT, NDG>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem);
  if (e != cudaSuccess) return e;
  if (probe) {
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kIrThreads, sh.smem);
    *fits = e == cudaSuccess && b >= 1;
    return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sh.G);
  cfg.blockDim = dim3(kIrThreads);
  cfg.dynamicSmemBytes = sh.smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ctx->launches++;
  ProfLaunch pl(ctx, kOther);  // a whole inner solve: SpMVs, dots and updates
  return cudaLaunchKernelEx(&cfg, fn, dview<MT>(A), a);
}

template <class MT>
inline cudaError_t ir_launch(ks_ctx *ctx, const CsrDev &A, const IrArgs &a, const IrShape &sh, bool probe,
                             bool *fits) {
  if (A.dia_nd == 7) return ir_launch_n<MT, 7>(ctx, A, a, sh, probe, fits);
  if (A.dia_nd == 5) return ir_launch_n<MT, 5>(ctx, A, a, sh, probe, fits);
  return ir_launch_n<MT, 0>(ctx, A, a, sh, probe, fits);
}

}  // namespace ks
