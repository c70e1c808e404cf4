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
  int quad;  // 1: the launcher enabled the quad path (spmv_dia_kernel; dia_quad_ok)
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
// The quad path of a plain SpMV (no reduction in its epilogue, x read
// directly, one GPU): thread t takes the quads of 4 consecutive rows
// 4 (t + k stride) .. +3 and loads each stored diagonal's values for them as
// one aligned vector (the symmetric layout's -1 diagonal: the +1 vector
// shifted by a row and one scalar), x of the +-1 diagonals as its own quad
// shifted by a row plus x[i0-1] and x[i0+4], each far diagonal's x as one
// aligned quad. A column outside [0, n) reads 0 where the row loop reads a
// clamped column; its value is 0 (the row has no entry there), and adding a
// zero term to a sum that starts at +0 leaves it unchanged, so each row's sum
// has the same terms in the same order and the same bits. Launched only
// where dia_quad_ok holds (5 or 7 diagonals at 0, +-1 and pairs of multiples
// of 4, the whole x, 16-byte aligned x and y), for FP32 and BF16 values: with
// FP64 values the quad path's registers cost the kernel occupancy, and the
// row path is faster (C4: 34.7 against 37.1 us).
template <class E, class = void>
struct has_row4 : std::false_type {};
template <class E>
struct has_row4<E, std::void_t<decltype(&E::row4)>> : std::true_type {};

template <class T>
__device__ __forceinline__ void dq_ld4(const T *p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 u = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
  } else {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
  }
}
template <class MT, class AT>
__device__ __forceinline__ void dq_vals(const MT *p, AT (&v)[4]) {
  if constexpr (std::is_same<MT, __nv_bfloat16>::value) {
    const uint2 u = ld_stream(reinterpret_cast<const uint2 *>(p));
    v[0] = __uint_as_float(u.x << 16), v[1] = __uint_as_float(u.x & 0xffff0000u);
    v[2] = __uint_as_float(u.y << 16), v[3] = __uint_as_float(u.y & 0xffff0000u);
  } else if constexpr (sizeof(MT) == 4) {
    const float4 u = ld_stream(reinterpret_cast<const float4 *>(p));
    v[0] = u.x, v[1] = u.y, v[2] = u.z, v[3] = u.w;
  } else {
    const double2 a = ld_stream(reinterpret_cast<const double2 *>(p)),
                  b = ld_stream(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
  }
}

template <int NDG, class MT, class AT, class XT, class Epi>
__device__ __forceinline__ void dia_quads(const DiaT<MT> &D, const XT *x, const Epi &epi, int stride) {
  constexpr int H = NDG / 2;
  constexpr bool kMask = std::is_same<MT, double>::value;
  const int nq = D.n / 4;
  const bool sym = D.vs[H - 1] != 0;
  for (int qi = (int)(blockIdx.x * blockDim.x + threadIdx.x); qi < nq; qi += stride) {
    const int i0 = 4 * qi;
    unsigned m = 0xffffffffu;
    if constexpr (kMask) m = __ldcs(reinterpret_cast<const unsigned *>(D.mask + i0));
    AT y[4] = {(AT)0, (AT)0, (AT)0, (AT)0};
    auto term = [&](int k, const AT (&v)[4], const AT (&xv)[4]) {
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const AT t = add_rn(y[e], mul_rn(v[e], xv[e]));
        if constexpr (kMask)
          y[e] = ((m >> (8 * e + k)) & 1u) ? t : y[e];
        else
          y[e] = t;
      }
    };
    auto xq = [&](int c, AT (&xv)[4]) {  // x[c .. c+3], c a multiple of 4
      if (c >= 0 && c + 4 <= D.n) {
        XT t[4];
        dq_ld4<XT>(x + c, t);
#pragma unroll
        for (int e = 0; e < 4; e++) xv[e] = (AT)t[e];
      } else {
#pragma unroll
        for (int e = 0; e < 4; e++) xv[e] = (c + e >= 0 && c + e < D.n) ? (AT)__ldg(x + c + e) : (AT)0;
      }
    };
    auto far = [&](int k) {
      AT v[4], xv[4];
      dq_vals<MT, AT>(D.vb[k] + (i0 + D.vs[k]), v);
      xq(i0 + D.off[k], xv);
      term(k, v, xv);
    };
    AT xo[4], v1[4];
    xq(i0, xo);
    const AT xm1 = i0 >= 1 ? (AT)__ldg(x + i0 - 1) : (AT)0;
    const AT xp4 = i0 + 4 < D.n ? (AT)__ldg(x + i0 + 4) : (AT)0;
    dq_vals<MT, AT>(D.vb[H + 1] + i0, v1);
#pragma unroll
    for (int k = 0; k < H - 1; k++) far(k);
    {
      AT v[4];
      if (sym) {
        v[0] = mval<AT>(ld_stream(D.vb[H + 1] + (i0 - 1)));
        v[1] = v1[0], v[2] = v1[1], v[3] = v1[2];
      } else {
        dq_vals<MT, AT>(D.vb[H - 1] + i0, v);
      }
      const AT xv[4] = {xm1, xo[0], xo[1], xo[2]};
      term(H - 1, v, xv);
    }
    {
      AT v[4];
      dq_vals<MT, AT>(D.vb[H] + i0, v);
      term(H, v, xo);
    }
    {
      const AT xv[4] = {xo[1], xo[2], xo[3], xp4};
      term(H + 1, v1, xv);
    }
#pragma unroll
    for (int k = H + 2; k < NDG; k++) far(k);
    epi.row4(i0, y);
  }
}

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
  int row0 = 0;  // the rows the quad path leaves to the loop below start here
  if constexpr (NV == 1 && Epi::ND == 0 && (NDG == 5 || NDG == 7) && GX::kPlain && has_row4<Epi>::value &&
                !std::is_same<MT, double>::value) {
    if (D.quad) {
      dia_quads<NDG, MT, AT>(D, g0.x, epi, stride);
      row0 = D.n / 4 * 4;
    }
  }
  for (int i = row0 + (int)(blockIdx.x * blockDim.x + threadIdx.x); i < D.n; i += stride) {
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

// BiCG's two products q = A p and t = A^T p* in one pass (FP64, one GPU):
// thread i sums row i of A against p and row i of A^T against p*, the
// latter read from A's own diagonal copy through DT, a view in which A^T's
// diagonal k (offset o) is A's diagonal -o shifted by o rows
// (A^T[i][i+o] = A[i+o][i]); DT's row masks are A^T's. Both rows add their
// terms in ascending offset order from +0, so q and t are the bits of the
// two separate SpMVs. The shifted reads of A's diagonals meet the lines that
// the CTAs working o rows away load for their own q (|o| is a grid plane at
// most; plain loads, not evict-first ones, so that those lines stay), so A
// streams from HBM about once for both products. In the full
// layout (nd arrays of n values back to back) a shifted read of a lower
// diagonal runs into the next array and one of an upper diagonal into the
// previous one: every address stays inside the copy, and those terms are
// masked out. epi.row(i, q, t, acc).
template <int NDG, class GX, class Epi>
__global__ void __launch_bounds__(kThreads)
    spmv_dia_pair_kernel(DiaT<double> DA, DiaT<double> DT, GX gx0, GX gx1, Epi epi, Stop stop, Red red) {
  constexpr int ND = Epi::ND > 0 ? Epi::ND : 1;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const int stride = (int)(gridDim.x * blockDim.x);
  pdl_wait();
  if (stop()) return;
  const GX g0 = gx0.prep(), g1 = gx1.prep();
  for (int i = (int)(blockIdx.x * blockDim.x + threadIdx.x); i < DA.n; i += stride) {
    const unsigned ma = (unsigned)__ldcs(DA.mask + i), mt = (unsigned)__ldcs(DT.mask + i);
    double a[NDG], b[NDG], x0[NDG], x1[NDG];
#pragma unroll
    for (int d = 0; d < NDG; d++) {
      a[d] = __ldg(DA.vb[d] + (i + DA.vs[d]));
      b[d] = __ldg(DT.vb[d] + (i + DT.vs[d]));
      x0[d] = g0.template get<double>(min(max(i + DA.off[d], DA.cmin), DA.cmax - 1));
      x1[d] = g1.template get<double>(min(max(i + DT.off[d], DT.cmin), DT.cmax - 1));
    }
    double y0 = 0.0, y1 = 0.0;
#pragma unroll
    for (int d = 0; d < NDG; d++) {
      const double t0 = add_rn(y0, mul_rn(a[d], x0[d]));
      y0 = ((ma >> d) & 1u) ? t0 : y0;
      const double t1 = add_rn(y1, mul_rn(b[d], x1[d]));
      y1 = ((mt >> d) & 1u) ? t1 : y1;
    }
    epi.row(i, y0, y1, acc);
  }
  __syncthreads();
  pdl_trigger();
  if constexpr (Epi::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && threadIdx.x == 0) epi.finish(acc);
  }
}

}  // namespace ks
