// Kernel templates: row-blocked CSR SpMV with fused epilogues, and fused
// vector (BLAS-1) passes with deterministic single-pass grid reductions.
#pragma once

#include "ks_common.cuh"

namespace ks {

// One SpMV row block (CSR-Adaptive style binning, chosen per block):
//  * "stream" blocks hold up to kRowsPerBlock rows and kNnzPerBlock nonzeros.
//    The CTA streams the block's col/val with 128-bit loads (int4 columns,
//    double2/float4 values), gathers x, and parks the products in shared
//    memory. Rows of up to 16 nonzeros on average are then summed one thread
//    per row, in index order from 0.0, exactly as blas::MtxVec_mult
//    (blas.cpp:56-62) does -- the FP64 result equals the reference's bit for
//    bit. Denser blocks sum one warp per row.
//  * "long" blocks hold a single row with more than kNnzPerBlock nonzeros,
//    reduced by the whole CTA.
// NV right-hand vectors share one pass over the block's col/val (NV = 2 for
// the k-skip matrix powers). On return rowsum[v*kRowsPerBlock + t] holds row
// r0+t of product v, visible to all threads.
template <int NV, class MT, class XT, class AT>
__device__ __forceinline__ void spmv_block(const CsrK<MT> &A, int blk,
                                           const XT *const *x,
                                           AT *__restrict__ rowsum,
                                           AT *__restrict__ prod, int &r0_out,
                                           int &nrows_out) {
  const int r0 = A.rb[blk], r1 = A.rb[blk + 1];
  const int nrows = r1 - r0;
  const int j0 = A.ptr[r0], j1 = A.ptr[r1];
  const int t = threadIdx.x;
  int rs = 0, re = 0;
  if (t < nrows) {
    rs = A.ptr[r0 + t];
    re = A.ptr[r0 + t + 1];
  }
  const int nnz = j1 - j0;
  r0_out = r0;
  nrows_out = nrows;
  if (nnz <= kNnzPerBlock) {
    const int a0 = j0 & ~(kChunk - 1);
    const int nch = (j1 - a0 + kChunk - 1) / kChunk;
    for (int c = t; c < nch; c += kThreads) {
      const int j = a0 + c * kChunk;
      const int4 cc = ld_stream(reinterpret_cast<const int4 *>(A.col + j));
      MT v[4];
      ld_vals4(A.val + j, v);
      const int cols[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int jj = j + q;
        if (jj >= j0 && jj < j1) {
#pragma unroll
          for (int u = 0; u < NV; u++)
            prod[u * kNnzPerBlock + jj - j0] =
                mul_rn(mval<AT>(v[q]), (AT)__ldg(x[u] + cols[q]));
        }
      }
    }
    __syncthreads();
    if (nnz <= 16 * nrows) {
      if (t < nrows) {
#pragma unroll
        for (int u = 0; u < NV; u++) {
          const AT *pp = prod + u * kNnzPerBlock;
          AT s = (AT)0;
          for (int e = rs - j0; e < re - j0; e++) s = add_rn(s, pp[e]);
          rowsum[u * kRowsPerBlock + t] = s;
        }
      }
    } else {
      const int lane = t & 31, w = t >> 5;
      for (int rr = w; rr < nrows; rr += kThreads / 32) {
        const int a = A.ptr[r0 + rr] - j0, b = A.ptr[r0 + rr + 1] - j0;
#pragma unroll
        for (int u = 0; u < NV; u++) {
          const AT *pp = prod + u * kNnzPerBlock;
          AT s = (AT)0;
          for (int e = a + lane; e < b; e += 32) s += pp[e];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == 0) rowsum[u * kRowsPerBlock + rr] = s;
        }
      }
    }
    __syncthreads();
  } else {
    // A single long row: the CTA strides over it.
    double v[NV];
#pragma unroll
    for (int u = 0; u < NV; u++) {
      AT s = (AT)0;
      for (int j = j0 + t; j < j1; j += kThreads)
        s += mval<AT>(A.val[j]) * (AT)__ldg(x[u] + A.col[j]);
      v[u] = (double)s;
    }
    block_sum<NV>(v);
    if (t == 0) {
#pragma unroll
      for (int u = 0; u < NV; u++) rowsum[u * kRowsPerBlock] = (AT)v[u];
    }
    __syncthreads();
  }
}

// Epilogue concept for spmv_kernel:
//   using acc_t = double|float;   // row-sum type
//   static constexpr int ND;      // number of fused reductions (0..kMaxDots)
//   __device__ void row(int r, acc_t y, double (&acc)[ND?ND:1]) const;
//   __device__ void finish(const double (&sums)[ND?ND:1]) const;  // thread 0 of last CTA
template <class MT, class XT, class Epi>
__global__ void __launch_bounds__(kThreads)
    spmv_kernel(CsrK<MT> A, const XT *__restrict__ x, Epi epi, Stop stop,
                Red red) {
  using AT = typename Epi::acc_t;
  __shared__ AT prod[kNnzPerBlock];
  __shared__ AT rowsum[kRowsPerBlock];
  if (stop()) return;
  constexpr int ND = Epi::ND > 0 ? Epi::ND : 1;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const XT *xs[1] = {x};
  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x) {
    int r0, nrows;
    spmv_block<1, MT, XT, AT>(A, blk, xs, rowsum, prod, r0, nrows);
    if (threadIdx.x < nrows) epi.row(r0 + threadIdx.x, rowsum[threadIdx.x], acc);
    __syncthreads();
  }
  if constexpr (Epi::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) epi.finish(acc);
  }
}

// Two SpMVs sharing one pass over A (k-skip matrix powers: r and p chains).
// Epi::row(r, y0, y1, acc).
template <class MT, class XT, class Epi>
__global__ void __launch_bounds__(kThreads)
    spmv2_kernel(CsrK<MT> A, const XT *__restrict__ x0,
                 const XT *__restrict__ x1, Epi epi, Stop stop, Red red) {
  using AT = typename Epi::acc_t;
  __shared__ AT prod[2 * kNnzPerBlock];
  __shared__ AT rowsum[2 * kRowsPerBlock];
  if (stop()) return;
  constexpr int ND = Epi::ND > 0 ? Epi::ND : 1;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const XT *xs[2] = {x0, x1};
  for (int blk = blockIdx.x; blk < A.nrb; blk += gridDim.x) {
    int r0, nrows;
    spmv_block<2, MT, XT, AT>(A, blk, xs, rowsum, prod, r0, nrows);
    if (threadIdx.x < nrows)
      epi.row(r0 + threadIdx.x, rowsum[threadIdx.x], rowsum[kRowsPerBlock + threadIdx.x], acc);
    __syncthreads();
  }
  if constexpr (Epi::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) epi.finish(acc);
  }
}

// Op concept for vec_kernel:
//   static constexpr int ND;
//   __device__ void elem(long long i, double (&acc)[ND?ND:1]) const;
//   __device__ void finish(const double (&sums)[ND?ND:1]) const;
template <class Op>
__global__ void __launch_bounds__(kThreads)
    vec_kernel(Op op, long long n, Stop stop, Red red) {
  if (stop()) return;
  constexpr int ND = Op::ND > 0 ? Op::ND : 1;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const long long stride = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
#pragma unroll 4
  for (; i < n; i += stride) op.elem(i, acc);
  if constexpr (Op::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) op.finish(acc);
  }
}

// Scalar step run by a single thread (recurrences that need no vector data).
template <class Op>
__global__ void scalar_kernel(Op op, Stop stop) {
  if (stop()) return;
  if (threadIdx.x == 0 && blockIdx.x == 0) op.run();
}

// ------------------------------------------------------------------ launchers
inline Red red_of(ks_ctx *ctx, int slot = 0) {
  return Red{ctx->partials, ctx->counters + slot};
}

template <class MT, class XT, class Epi>
inline void launch_spmv(ks_ctx *ctx, const CsrDev &A, const XT *x, const Epi &epi,
                        Stop stop, int slot = 0) {
  const int grid = spmv_grid(ctx, A);
  ctx->launches++;
  spmv_kernel<MT, XT, Epi><<<grid, kThreads, 0, ctx->stream>>>(view<MT>(A), x, epi, stop,
                                                              red_of(ctx, slot));
}

template <class MT, class XT, class Epi>
inline void launch_spmv2(ks_ctx *ctx, const CsrDev &A, const XT *x0, const XT *x1,
                         const Epi &epi, Stop stop, int slot = 0) {
  const int grid = spmv_grid(ctx, A);
  ctx->launches++;
  spmv2_kernel<MT, XT, Epi><<<grid, kThreads, 0, ctx->stream>>>(view<MT>(A), x0, x1, epi,
                                                               stop, red_of(ctx, slot));
}

template <class Op>
inline void launch_vec(ks_ctx *ctx, long long n, const Op &op, Stop stop, int slot = 0) {
  long long need = (n + kThreads - 1) / kThreads;
  int grid = red_grid(ctx);
  if (need < grid) grid = (int)(need > 0 ? need : 1);
  ctx->launches++;
  vec_kernel<Op><<<grid, kThreads, 0, ctx->stream>>>(op, n, stop, red_of(ctx, slot));
}

template <class Op>
inline void launch_scalar(ks_ctx *ctx, const Op &op, Stop stop) {
  ctx->launches++;
  scalar_kernel<Op><<<1, 32, 0, ctx->stream>>>(op, stop);
}

}  // namespace ks
