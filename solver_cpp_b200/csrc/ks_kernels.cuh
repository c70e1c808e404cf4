// Kernel templates and launchers: the TMA-staged CSR SpMV with fused
// epilogues (ks_spmv_tma.cuh), fused vector (BLAS-1) passes with
// deterministic single-pass grid reductions, and single-thread scalar steps.
#pragma once

#include <atomic>
#include <type_traits>

#include "ks_common.cuh"
#include "ks_dist.cuh"
#include "ks_spmv_dia.cuh"
#include "ks_spmv_tma.cuh"

namespace ks {

// SpMV epilogue concept (see spmv_tma_kernel):
//   using acc_t = double|float;   // row-sum type
//   static constexpr int ND;      // number of fused reductions (0..kMaxDots)
//   __device__ void row(int r, acc_t y, double (&acc)[ND?ND:1]) const;        (one vector)
//   __device__ void row(int r, acc_t y0, acc_t y1, double (&acc)[...]) const; (two vectors)
//   __device__ void finish(const double (&sums)[ND?ND:1]) const;  // thread 0 of last CTA

// Op concept for vec_kernel:
//   static constexpr int ND;
//   __device__ void finish(const double (&sums)[ND?ND:1]) const;
// and either
//   __device__ void elem(long long i, double (&acc)[ND?ND:1]) const;
// or the two-phase form, which lets every thread keep kVecUnroll elements'
// loads in flight before its first store (an op's stores might alias its
// loads, so the compiler cannot reorder a one-phase elem() that way):
//   using Regs = ...;
//   __device__ Regs load(long long i) const;
//   __device__ void store(long long i, const Regs &r, double (&acc)[...]) const;
constexpr int kVecUnroll = 4;

template <class Op, class = void>
struct has_two_phase : std::false_type {};
template <class Op>
struct has_two_phase<Op, std::void_t<typename Op::Regs>> : std::true_type {};

template <class Op>
__global__ void __launch_bounds__(kThreads)
    vec_kernel(Op op, long long n, Stop stop, Red red) {
  pdl_wait();
  if (stop()) return;
  constexpr int ND = Op::ND > 0 ? Op::ND : 1;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const long long stride = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if constexpr (has_two_phase<Op>::value) {
    for (; i < n; i += stride * kVecUnroll) {
      typename Op::Regs r[kVecUnroll];
#pragma unroll
      for (int u = 0; u < kVecUnroll; u++)
        if (i + u * stride < n) r[u] = op.load(i + u * stride);
#pragma unroll
      for (int u = 0; u < kVecUnroll; u++)
        if (i + u * stride < n) op.store(i + u * stride, r[u], acc);
    }
  } else {
#pragma unroll 4
    for (; i < n; i += stride) op.elem(i, acc);
  }
  pdl_trigger();  // the next kernel may be scheduled as this one drains
  if constexpr (Op::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) op.finish(acc);
  }
}

// Tall-skinny basis combination: every element j runs a sequential chain over
// k basis vectors (GMRES's w -= sum h_i v_i, the deferred x += sum alpha_i
// p_i, the GMRES/GCR solution and direction updates), so the order of the
// terms, and with it every rounding, is the reference's per-element loop.
// Each thread walks its elements one at a time; the loads of the next chunk
// of basis vectors are issued before the current chunk is consumed, which
// keeps enough bytes in flight to stream the basis at HBM speed despite the
// chain.
// Op concept:
//   using vt = element type; static constexpr int NB (1 or 2 bases), ND;
//   long long ld;                               // stride between basis vectors
//   struct St;                                  // per-element state
//   __device__ bool active() const;             // uniform gate (device state)
//   __device__ int count() const;               // k (may read device memory)
//   __device__ const vt *base(int b) const;
//   __device__ St init(long long j) const;
//   __device__ void step(St &, int i, const vt (&v)[NB]) const;
//   __device__ void done(long long j, const St &, double (&acc)[ND ? ND : 1]) const;
//   __device__ void finish(const double (&sums)[ND ? ND : 1]) const;
//   static constexpr bool kFinishOnly;          // ND == 0 and finish() still runs
// Loads in flight per element: kBasisLoads (split over the NB bases).
constexpr int kBasisLoads = 8;

template <class Op, class = void>
struct finish_only : std::false_type {};
template <class Op>
struct finish_only<Op, std::void_t<decltype(Op::kFinishOnly)>> : std::integral_constant<bool, Op::kFinishOnly> {};

template <class Op>
__global__ void __launch_bounds__(kThreads) basis_kernel(Op op, long long n, Stop stop, Red red) {
  using VT = typename Op::vt;
  constexpr int NB = Op::NB, C = kBasisLoads / NB;
  constexpr int ND = Op::ND > 0 ? Op::ND : 1;
  pdl_wait();
  if (stop() || !op.active()) return;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const int k = op.count();
  const VT *B[NB];
#pragma unroll
  for (int b = 0; b < NB; b++) B[b] = op.base(b);
  const long long ld = op.ld;
  const long long estride = (long long)gridDim.x * kThreads;
  for (long long j = (long long)blockIdx.x * kThreads + threadIdx.x; j < n; j += estride) {
    // the next element's first chunk heads for L2 while this one runs
    if (j + estride < n) {
#pragma unroll
      for (int u = 0; u < C; u++)
#pragma unroll
        for (int b = 0; b < NB; b++)
          if (u < k) prefetch_l2(B[b] + (long long)u * ld + j + estride);
    }
    typename Op::St s = op.init(j);
    VT cur[C][NB], nxt[C][NB];
#pragma unroll
    for (int u = 0; u < C; u++)
#pragma unroll
      for (int b = 0; b < NB; b++) cur[u][b] = u < k ? B[b][(long long)u * ld + j] : (VT)0;
    for (int i0 = 0; i0 < k; i0 += C) {
#pragma unroll
      for (int u = 0; u < C; u++)
#pragma unroll
        for (int b = 0; b < NB; b++)
          nxt[u][b] = i0 + C + u < k ? B[b][(long long)(i0 + C + u) * ld + j] : (VT)0;
#pragma unroll
      for (int u = 0; u < C; u++)
        if (i0 + u < k) op.step(s, i0 + u, cur[u]);
#pragma unroll
      for (int u = 0; u < C; u++)
#pragma unroll
        for (int b = 0; b < NB; b++) cur[u][b] = nxt[u][b];
    }
    op.done(j, s, acc);
  }
  pdl_trigger();
  if constexpr (Op::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) op.finish(acc);
  } else if constexpr (finish_only<Op>::value) {
    if (grid_last(red.counter) && threadIdx.x == 0) op.finish(acc);
  }
}

// Scalar step run by a single thread (recurrences that need no vector data).
template <class Op>
__global__ void scalar_kernel(Op op, Stop stop) {
  pdl_wait();
  if (stop()) return;
  if (threadIdx.x == 0 && blockIdx.x == 0) op.run();
  pdl_trigger();
}

// ------------------------------------------------------------------ launchers
inline Red red_of(ks_ctx *ctx, int slot = 0) {
  return Red{ctx->partials, ctx->counters + slot};
}

// With ks_params.profile: events around one launch, recorded with its class
// (every launch of a profiled solve goes through this, launch_k or not).
struct ProfLaunch {
  ks_ctx *ctx;
  long long i = -1;
  int cls;
  ProfLaunch(ks_ctx *c, int k) : ctx(c), cls(k) {
    if (!ctx->prof_on) return;
    const size_t n = ctx->prof_class.size();
    while (ctx->prof_events.size() < 2 * n + 2) {
      cudaEvent_t e = nullptr;
      if (cudaEventCreate(&e) != cudaSuccess) {  // no more events: stop recording
        (void)cudaGetLastError();
        ctx->prof_on = 0;
        return;
      }
      ctx->prof_events.push_back(e);
    }
    i = (long long)n;
    cudaEventRecord(ctx->prof_events[2 * n], ctx->stream);
  }
  ~ProfLaunch() {
    if (i < 0) return;
    cudaEventRecord(ctx->prof_events[2 * i + 1], ctx->stream);
    ctx->prof_class.push_back((unsigned char)cls);
  }
};

// Launch on the context's stream with programmatic stream serialization:
// the kernel may be scheduled while the previous one finishes, and reads the
// previous kernels' results only after its griddepcontrol.wait (pdl_wait).
template <class... KArgs, class... Args>
inline void launch_k(ks_ctx *ctx, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ctx->launches++;
  const int cls = ctx->next_class;
  ctx->next_class = kOther;
  ProfLaunch pl(ctx, cls);
  cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <class MT>
inline const MT *values_of(const CsrDev &A);
template <>
inline const double *values_of<double>(const CsrDev &A) {
  return A.val;
}
template <>
inline const float *values_of<float>(const CsrDev &A) {
  return A.val32;
}
template <>
inline const __nv_bfloat16 *values_of<__nv_bfloat16>(const CsrDev &A) {
  return A.val16;
}

template <class MT, class IT>
inline CsrT<MT, IT> tview(const CsrDev &A) {
  const IT *col;
  if constexpr (sizeof(IT) == 2)
    col = A.col16;
  else
    col = A.col;
  return {A.ptr, col, values_of<MT>(A), A.rbi, A.nrb, A.n};
}

// One-time per device and instantiation: opt in to the stage buffers' shared
// memory and record how many CTAs fit on an SM.
template <int NV, class MT, class IT, class GX, class Epi>
inline int spmv_tma_ctas_per_sm(int device) {
  static std::atomic<unsigned long long> configured{0};
  static int per_sm[64] = {0};
  const unsigned long long bit = 1ull << (device & 63);
  if (!(configured.load() & bit)) {
    auto fn = spmv_tma_kernel<NV, MT, IT, GX, Epi>;
    constexpr int smem = (int)spmv_tma_smem<MT, IT>();
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreads, smem) != cudaSuccess || b < 1) b = 1;
    per_sm[device & 63] = b;
    configured.fetch_or(bit);
  }
  return per_sm[device & 63];
}

template <class Op>
inline void launch_scalar(ks_ctx *ctx, const Op &op, Stop stop) {
  launch_k(ctx, scalar_kernel<Op>, dim3(1), dim3(32), 0, op, stop);
}

// ------------------------------------------------------------------ split solves
// In a row-split solve (ctx->red_comm set) a kernel's reductions cover this
// rank's rows only. The kernel then leaves its sums in ctx->d_stage instead of
// running its scalar step; the sums are added over the ranks on the stream,
// and the scalar step runs afterwards on every rank with the same totals, so
// every rank takes the same decisions.
template <class Op>
struct StageSums : Op {
  double *stage;
  __device__ void finish(const double (&s)[Op::ND > 0 ? Op::ND : 1]) const {
#pragma unroll
    for (int d = 0; d < Op::ND; d++) stage[d] = s[d];
  }
};

template <class Op>
struct FinishSummed {
  Op op;
  const double *stage;
  __device__ void run() const {
    double s[Op::ND > 0 ? Op::ND : 1];
#pragma unroll
    for (int d = 0; d < Op::ND; d++) s[d] = stage[d];
    op.finish(s);
  }
};

inline void note_dist(ks_ctx *ctx, ks_status s) {
  if (s != KS_OK && ctx->dist_status == KS_OK) ctx->dist_status = s;
}

template <class Op, class F>
inline void with_rank_sums(ks_ctx *ctx, const Op &op, Stop stop, F &&launch) {
  if constexpr (Op::ND > 0) {
    if (ctx->red_comm) {
      StageSums<Op> w;
      static_cast<Op &>(w) = op;
      w.stage = ctx->d_stage;
      launch(w);
      note_dist(ctx, ctx->red_comm->allreduce(ctx->d_stage, Op::ND));
      launch_scalar(ctx, FinishSummed<Op>{op, ctx->d_stage}, stop);
      return;
    }
  }
  launch(op);
}

template <class MT>
inline const MT *dia_values_of(const CsrDev &A);
template <>
inline const double *dia_values_of<double>(const CsrDev &A) {
  return A.dia_val;
}
template <>
inline const float *dia_values_of<float>(const CsrDev &A) {
  return A.dia_val32;
}
template <>
inline const __nv_bfloat16 *dia_values_of<__nv_bfloat16>(const CsrDev &A) {
  return A.dia_val16;
}

template <class MT>
inline DiaT<MT> dview(const CsrDev &A) {
  DiaT<MT> d;
  const MT *v = dia_values_of<MT>(A);
  const int nd = A.dia_nd, h = nd / 2;
  for (int k = 0; k < kMaxDiag; k++) {
    d.vb[k] = v;
    d.vs[k] = 0;
    if (k >= nd) continue;
    if (!A.dia_sym) {
      d.vb[k] = v + (long long)k * A.dia_ds;
    } else if (k >= h) {  // main and upper diagonals: stored rows
      d.vb[k] = v + (long long)(k - h) * A.dia_ds + A.dia_pad;
    } else {  // lower diagonal k: its mirror nd-1-k, shifted back by the offset
      d.vb[k] = v + (long long)(nd - 1 - k - h) * A.dia_ds + A.dia_pad;
      d.vs[k] = A.dia_off[k];
    }
  }
  // FP64 sums add only the entries the row has (bit-exact also for
  // non-finite x); FP32/BF16 add the stored zeros (see ks_spmv_dia.cuh).
  d.mask = std::is_same<MT, double>::value ? A.dia_mask : nullptr;
  d.n = A.n;
  d.nd = nd;
  d.cmin = A.dia_cmin;
  d.cmax = A.dia_cmax;
  for (int k = 0; k < kMaxDiag; k++) d.off[k] = A.dia_off[k];
  d.quad = 0;
  return d;
}

// Whether a plain SpMV (x read directly, y stored) may take the DIA kernel's
// quad path: 5 or 7 diagonals at offsets 0, -1, +1 and pairs -o, +o with o a
// multiple of 4, stored diagonals of a multiple of 4 elements (their vector
// loads aligned), over the whole x (one GPU), x and y aligned for 4-element
// vector accesses.
template <class XT, class YT>
inline bool dia_quad_ok(const CsrDev &A, const XT *x, const YT *y) {
  const int nd = A.dia_nd;
  if ((nd != 5 && nd != 7) || A.dia_cmin != 0 || A.dia_cmax != A.n) return false;
  if (A.dia_ds % 4 != 0) return false;  // every stored diagonal starts on a 4-element boundary
  const int h = nd / 2;
  if (A.dia_off[h] != 0 || A.dia_off[h - 1] != -1 || A.dia_off[h + 1] != 1) return false;
  for (int k = 0; k < h - 1; k++)
    if (A.dia_off[k] % 4 != 0 || A.dia_off[k] != -A.dia_off[nd - 1 - k]) return false;
  return reinterpret_cast<uintptr_t>(x) % (4 * sizeof(XT)) == 0 && reinterpret_cast<uintptr_t>(y) % (4 * sizeof(YT)) == 0;
}

template <int NV, int NDG, class MT, class GX, class Epi>
inline int spmv_dia_ctas_per_sm(int device) {
  static std::atomic<unsigned long long> configured{0};
  static int per_sm[64] = {0};
  const unsigned long long bit = 1ull << (device & 63);
  if (!(configured.load() & bit)) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, spmv_dia_kernel<NV, NDG, MT, GX, Epi>, kThreads, 0) !=
            cudaSuccess ||
        b < 1)
      b = 1;
    per_sm[device & 63] = std::min(b, 8);
    configured.fetch_or(bit);
  }
  return per_sm[device & 63];
}

template <int NV, int NDG, class MT, class GX, class Epi>
inline void launch_spmv_dn(ks_ctx *ctx, const CsrDev &A, const GX &g0, const GX &g1, const Epi &epi, Stop stop,
                           int slot) {
  const long long need = ((long long)A.n + kThreads - 1) / kThreads;
  const long long wave = (long long)ctx->num_sms * spmv_dia_ctas_per_sm<NV, NDG, MT, GX, Epi>(ctx->device);
  const int grid = (int)std::max<long long>(1, std::min(need, wave));
  ctx->next_class = std::is_same<MT, double>::value ? kMv : kMvLow;
  DiaT<MT> dv = dview<MT>(A);
  if constexpr (NV == 1 && Epi::ND == 0 && (NDG == 5 || NDG == 7) && GX::kPlain && has_row4<Epi>::value &&
                !std::is_same<MT, double>::value)
    dv.quad = dia_quad_ok(A, g0.x, epi.y) ? 1 : 0;
  launch_k(ctx, spmv_dia_kernel<NV, NDG, MT, GX, Epi>, dim3(grid), dim3(kThreads), 0, dv, g0, g1, epi, stop,
           red_of(ctx, slot));
}

// SpMV over the diagonal copy: one thread per row, one resident wave of CTAs;
// 5 and 7 diagonals (2-D and 3-D stencils) compiled for their count.
template <int NV, class MT, class GX, class Epi>
inline void launch_spmv_d(ks_ctx *ctx, const CsrDev &A, const GX &g0, const GX &g1, const Epi &epi_in, Stop stop,
                          int slot) {
  with_rank_sums(ctx, epi_in, stop, [&](const auto &epi) {
    using E = std::decay_t<decltype(epi)>;
    if (A.dia_nd == 7)
      launch_spmv_dn<NV, 7, MT, GX, E>(ctx, A, g0, g1, epi, stop, slot);
    else if (A.dia_nd == 5)
      launch_spmv_dn<NV, 5, MT, GX, E>(ctx, A, g0, g1, epi, stop, slot);
    else
      launch_spmv_dn<NV, 0, MT, GX, E>(ctx, A, g0, g1, epi, stop, slot);
  });
}

template <int NV, class MT, class IT, class GX, class Epi>
inline void launch_spmv_k(ks_ctx *ctx, const CsrDev &A, const GX &g0, const GX &g1, const Epi &epi, Stop stop,
                          int slot) {
  const int per_sm = spmv_tma_ctas_per_sm<NV, MT, IT, GX, Epi>(ctx->device);
  const int grid = std::max(1, std::min(ctx->num_sms * per_sm, A.nrb));
  ctx->next_class = std::is_same<MT, double>::value ? kMv : kMvLow;
  launch_k(ctx, spmv_tma_kernel<NV, MT, IT, GX, Epi>, dim3(grid), dim3(kThreads), spmv_tma_smem<MT, IT>(),
           tview<MT, IT>(A), g0, g1, epi, stop, red_of(ctx, slot), ctx->d_err, ctx->wait_ns);
}

template <int NV, class MT, class IT, class GX, class Epi>
inline void launch_spmv_i(ks_ctx *ctx, const CsrDev &A, const GX &g0, const GX &g1, const Epi &epi_in, Stop stop,
                          int slot) {
  with_rank_sums(ctx, epi_in, stop, [&](const auto &epi) {
    launch_spmv_k<NV, MT, IT, GX, std::decay_t<decltype(epi)>>(ctx, A, g0, g1, epi, stop, slot);
  });
}

// The diagonal copy when the matrix has one for these values, else CSR with
// 16-bit column offsets when it has them, else CSR with int32 columns.
template <int NV, class MT, class GX, class Epi>
inline void launch_spmv_g(ks_ctx *ctx, const CsrDev &A, const GX &g0, const GX &g1, const Epi &epi, Stop stop,
                          int slot = 0) {
  if (A.dia_nd && dia_values_of<MT>(A))
    launch_spmv_d<NV, MT, GX, Epi>(ctx, A, g0, g1, epi, stop, slot);
  else if (A.col16)
    launch_spmv_i<NV, MT, short, GX, Epi>(ctx, A, g0, g1, epi, stop, slot);
  else
    launch_spmv_i<NV, MT, int, GX, Epi>(ctx, A, g0, g1, epi, stop, slot);
}

template <class MT, class XT, class Epi>
inline void launch_spmv(ks_ctx *ctx, const CsrDev &A, const XT *x, const Epi &epi, Stop stop, int slot = 0) {
  launch_spmv_g<1, MT, GPtr<XT>, Epi>(ctx, A, GPtr<XT>{x}, GPtr<XT>{x}, epi, stop, slot);
}

template <class MT, class XT, class Epi>
inline void launch_spmv2(ks_ctx *ctx, const CsrDev &A, const XT *x0, const XT *x1, const Epi &epi, Stop stop,
                         int slot = 0) {
  launch_spmv_g<2, MT, GPtr<XT>, Epi>(ctx, A, GPtr<XT>{x0}, GPtr<XT>{x1}, epi, stop, slot);
}

// Class of a vector pass in the times report: a pass with reductions is a
// dot (most also update vectors: the reductions are fused into them), one
// marked kMemset (ZeroOp) a memset, any other pass "other".
template <class Op, class = void>
struct is_memset_op : std::false_type {};
template <class Op>
struct is_memset_op<Op, std::void_t<decltype(Op::kMemset)>> : std::integral_constant<bool, Op::kMemset> {};

template <class O>
constexpr int vec_class() {
  return is_memset_op<O>::value ? kMemset : (O::ND > 0 ? kDot : kOther);
}

template <class Op>
inline void launch_vec(ks_ctx *ctx, long long n, const Op &op_in, Stop stop, int slot = 0) {
  long long need = (n + kThreads - 1) / kThreads;
  int grid = red_grid(ctx);
  if (need < grid) grid = (int)(need > 0 ? need : 1);
  with_rank_sums(ctx, op_in, stop, [&](const auto &op) {
    using O = std::decay_t<decltype(op)>;
    ctx->next_class = vec_class<O>();
    launch_k(ctx, vec_kernel<O>, dim3(grid), dim3(kThreads), 0, op, n, stop, red_of(ctx, slot));
  });
}

// k_hint: the number of basis vectors, or a bound when the kernel reads it
// from the device. Short chains run at least one full-occupancy wave of CTAs
// and at most two elements per thread (measured best at 128^3: fewer CTAs
// keep the final reduction short, but each element's loads are a round trip
// the next element waits behind, even with its basis prefetched into L2).
// Long chains (measured: from 64 vectors) stream fastest with one thread per
// element, the reduction's cost then being small beside the pass.
template <class Op>
inline void launch_basis(ks_ctx *ctx, long long n, int k_hint, const Op &op, Stop stop, int slot = 0) {
  long long grid = (n + kThreads - 1) / kThreads;
  const long long cap = k_hint >= 64 ? (long long)(ctx->partials_len / (Op::ND > 0 ? Op::ND : 1))
                                     : std::max((long long)ctx->num_sms * 8, (grid + 1) / 2);
  grid = std::max(1LL, std::min(grid, cap));
  with_rank_sums(ctx, op, stop, [&](const auto &o) {
    using O = std::decay_t<decltype(o)>;
    launch_k(ctx, basis_kernel<O>, dim3((unsigned)grid), dim3(kThreads), 0, o, n, stop, red_of(ctx, slot));
  });
}

}  // namespace ks
