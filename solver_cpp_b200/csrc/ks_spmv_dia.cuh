// SpMV over the diagonal copy of a stencil-like matrix (sm_100a).
//
// Matrices of structured grids (5- and 7-point stencils, upwind
// convection-diffusion) hold every row's columns at a handful of fixed
// offsets from the row. Stored diagonal-major, the SpMV needs no column
// indices or row offsets at all: per nonzero only its value (plus, for FP64,
// one mask byte per row), against value + int16 offset + a share of the row
// offsets in CSR. A symmetric matrix keeps only its main and upper diagonals:
// a lower term A[i][i-o] is read as its mirror A[i-o][i], the same stream
// shifted back by o rows, which the CTAs working o rows behind have just
// pulled into L2 (4 instead of 7 value streams for a 7-point stencil).
// Thread i computes row i: for each diagonal d it adds val[d][i] *
// x[i + off[d]], diagonals in ascending offset order, which is the row's CSR
// column order, from 0.0 with separately rounded products and sums: the same
// sums as blas::MtxVec_mult (blas.cpp:56-62), bit for bit. FP64 adds only the
// terms the row's mask names. FP32 and BF16 add every diagonal: an absent
// entry is a stored zero, and 0 * x (x finite) added to a sum that started at
// +0.0 leaves it unchanged bit for bit, so the mask byte is not read. A warp
// reads 32 consecutive values of each diagonal and 32 consecutive entries of
// x per diagonal (coalesced; x is shared by the diagonals through L1/L2).
// Matrix data is read with the streaming hint, so the Krylov vectors keep
// their place in L2.
#pragma once

#include "ks_spmv_tma.cuh"

namespace ks {

template <class MT>
struct DiaT {
  // Diagonal d's element of row i is vb[d][i + vs[d]]: the full layout has
  // vs = 0; the symmetric half reads a lower diagonal from its upper mirror,
  // shifted by the (negative) offset into its zero pad.
  const MT *vb[kMaxDiag];
  int vs[kMaxDiag];
  const unsigned char *__restrict__ mask;  // n; null: every diagonal's term is added
  int n;
  int nd;
  int cmin, cmax;  // columns that exist in x (a split rank's window: beyond its rows)
  int off[kMaxDiag];
};

template <class MT>
__device__ __forceinline__ MT ld_stream(const MT *p) {
  return __ldcs(p);
}
template <>
__device__ __forceinline__ __nv_bfloat16 ld_stream<__nv_bfloat16>(const __nv_bfloat16 *p) {
  const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
  return __ushort_as_bfloat16(u);
}

// One thread per row, rows i, i + stride, ... of a grid-stride loop. NDG is
// the number of diagonals when known at compile time (5, 7), else 0 and the
// count comes from D.nd. Every diagonal's value is loaded (zeros stand where
// the row has no entry) and x at every diagonal's column, clamped into the
// columns that exist; a term whose mask bit is clear is computed but not
// added (a select, not a branch), so no load waits for the mask.
template <int NV, int NDG, class MT, class GX, class Epi>
__global__ void __launch_bounds__(kThreads) spmv_dia_kernel(DiaT<MT> D, GX gx0, GX gx1, Epi epi, Stop stop, Red red) {
  using AT = typename Epi::acc_t;
  constexpr int ND = Epi::ND > 0 ? Epi::ND : 1;
  constexpr int K = NDG > 0 ? NDG : kMaxDiag;
  const int nd = NDG > 0 ? NDG : D.nd;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const int stride = (int)(gridDim.x * blockDim.x);
  pdl_wait();  // x, the stop flags and the scalars come from earlier kernels
  if (stop()) return;
  const GX g0 = gx0.prep(), g1 = gx1.prep();
  for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < D.n; i += stride) {
    const unsigned m = D.mask ? (unsigned)__ldcs(D.mask + i) : 0xffu;
    MT a[K];
    AT x0[K], x1[NV == 2 ? K : 1];
#pragma unroll
    for (int d = 0; d < K; d++) {
      if (NDG > 0 || d < nd) {
        a[d] = ld_stream(D.vb[d] + (i + D.vs[d]));
        const int c = min(max(i + D.off[d], D.cmin), D.cmax - 1);
        x0[d] = g0.template get<AT>(c);
        if constexpr (NV == 2) x1[d] = g1.template get<AT>(c);
      }
    }
    // the row's sum over the diagonals it has, in ascending offset order
    AT y0 = (AT)0, y1 = (AT)0;
#pragma unroll
    for (int d = 0; d < K; d++) {
      if (NDG > 0 || d < nd) {
        const bool has = (m >> d) & 1u;
        const AT v = mval<AT>(a[d]);
        const AT t0 = add_rn(y0, mul_rn(v, x0[d]));
        y0 = has ? t0 : y0;
        if constexpr (NV == 2) {
          const AT t1 = add_rn(y1, mul_rn(v, x1[d]));
          y1 = has ? t1 : y1;
        }
      }
    }
    if constexpr (NV == 1)
      epi.row(i, y0, acc);
    else
      epi.row(i, y0, y1, acc);
  }
  __syncthreads();
  pdl_trigger();  // the next kernel may be scheduled as this one drains
  if constexpr (Epi::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) epi.finish(acc);
  }
}

}  // namespace ks
