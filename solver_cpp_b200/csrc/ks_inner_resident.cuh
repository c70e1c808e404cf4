// The inner CG of a VP method with its vectors on chip (sm_100a).
//
// A VP method's inner solve (innerMethods.cpp:71-118, here CG of a fixed
// number of iterations in FP32, or with BF16 matrix values) runs thousands of
// times; launched kernel by kernel, each iteration streams r, p, q and x
// through L2/HBM and pays three kernel boundaries. This kernel runs the whole
// inner solve in one cooperative launch of one CTA per SM. CTA b owns rows
// [b*rpc, (b+1)*rpc); thread t of it owns the quads of 4 consecutive rows
// b*rpc + 4096 j + 4 t .. +3 (j = 0, 1, ...):
//   * r and q of its rows live in tensor memory (TMEM, 256 KB per SM, which
//     no tensor-core work needs here): warp w reaches TMEM lanes
//     32 (w % 4) .. +31 and takes columns 64 (w / 4) .. +63 of them, so every
//     thread has 64 private 32-bit words: r_k in the first 32, q_k in the
//     other 32 (k < kIrMaxK),
//   * p and x of the CTA's rows live in shared memory (2 * rpc floats); p is
//     also published to a global array P from which the other CTAs gather it,
//     x is written out once, at the end,
//   * the matrix (the diagonal copy, FP32 or BF16 values, either layout) is
//     read from global memory (L2) every iteration, one vector load per
//     diagonal and quad where aligned.
// The TMEM columns are allocated once per launch and released on every way
// out of the kernel (a timed-out wait included).
// Per iteration (cg.cpp:184-240):
//   A: q = A p (own p from shared memory, other CTAs' from P), (p, q) summed
//      over the grid -> alpha = (r, r) / (p, q);
//   B: r -= alpha q, (r, r) summed -> beta, stopping test; x += alpha p
//      while the sum travels;
//   C: p = beta p + r, published; each CTA then waits only for the CTAs
//      whose rows its own rows read (release/acquire flags per CTA).
// Each element sees the FP32 operations of the kernel-per-step loop
// (CgMvEpi, XrUpdOp, XpbyToOp) in the same order; only the order in which
// the dot products add their terms differs (per thread over its rows, a
// fixed tree over the CTA, then the CTAs' partials in index order: the same
// in every run). Every CTA computes alpha, beta and the stopping decision
// from the same sums, so all leave the loop together.
//
// Grid reductions: each CTA writes its partial sums and adds itself to a
// monotonic arrival counter, waits with acquire loads until every CTA has
// arrived, then adds all the partials itself in one fixed order (the same
// bits in every CTA). Every wait is bounded by the context's wait limit; one
// that runs out sets the context's timeout flag and ends the kernel (the
// caller returns KS_TIMEOUT). Every CTA is resident (cooperative launch), so
// the waits end as soon as the last CTA arrives.
#pragma once

#include "ks_kernels.cuh"
#include "ks_state.cuh"

namespace ks {

constexpr int kIrThreads = 1024;  // threads per CTA, one CTA per SM
constexpr int kIrMaxK = 32;       // rows per thread (r and q in 64 TMEM columns)
constexpr int kIrWarps = kIrThreads / 32;

// Barrier state in device memory, zeroed before every launch: the grid
// reductions' counter, generation and result, then one publication flag per
// CTA (ir_sync_bytes).
struct IrSync {
  unsigned long long count;  // CTA arrivals at the reductions, all generations
  unsigned long long reserved;
};
static_assert(sizeof(IrSync) % 8 == 0, "the publication flags follow IrSync");

// Flag of CTA q right after IrSync: the last generation of p it has published.
__device__ __forceinline__ unsigned long long *ir_pub(IrSync *s, int q) {
  return reinterpret_cast<unsigned long long *>(s + 1) + q;
}

inline size_t ir_sync_bytes(int G) { return sizeof(IrSync) + sizeof(unsigned long long) * (size_t)G; }

struct IrArgs {
  const void *rin;  // inner solve: r rounded to FP32; whole solve: b (FP64); n entries
  void *x;          // the solution (the kernel's precision), n
  void *P;          // published directions (the kernel's precision), n
  DevState *st;     // the method's state
  const int *outer_done;  // inner solve: the outer method's done; whole solve: null
  double *partials;  // 2 kIrMaxSums per CTA (two generations)
  IrSync *sync;
  int *err;
  unsigned long long wait_ns;
  int n;
  int rpc;    // rows per CTA, a multiple of 32
  int K;      // rows per thread: ceil(rpc / kIrThreads) <= kIrMaxK (half for FP64)
  int whole;  // 1: a whole CG solve (|b|, the stopping state and the history of the method)
  int stencil;  // 1: full quads take ir_quad_mv_st (ir_stencil_ok holds, P is zero-padded)
  void *P2;     // BiCG: the published p* (zero-padded as P)
};

// P's zero pad on each side for the stencil path: beyond the largest offset
// plus a quad, a multiple of 8 elements (keeps P's vector alignment).
inline long long ir_p_pad(const CsrDev &A) {
  int m = 0;
  for (int k = 0; k < A.dia_nd; k++) m = std::max(m, std::abs(A.dia_off[k]));
  return ((long long)m + 8 + 7) / 8 * 8;
}

// Whether a matrix takes the stencil path of the on-chip SpMV: 5 or 7
// diagonals at offsets 0, -1, +1 and further pairs -o, +o with o a multiple
// of 4, stored diagonals of a multiple of 4 elements (the vector loads of
// their values aligned), over the system's own columns (one GPU).
inline bool ir_stencil_ok(const CsrDev &A, long long n) {
  const int nd = A.dia_nd;
  if ((nd != 5 && nd != 7) || A.dia_cmin != 0 || A.dia_cmax != n) return false;
  if (A.dia_ds % 4 != 0) return false;  // every stored diagonal starts on a 4-element boundary
  const int h = nd / 2;
  if (A.dia_off[h] != 0 || A.dia_off[h - 1] != -1 || A.dia_off[h + 1] != 1) return false;
  for (int k = 0; k < h - 1; k++)
    if (A.dia_off[k] % 4 != 0 || A.dia_off[k] != -A.dia_off[nd - 1 - k]) return false;
  return true;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// A reduction with release semantics at GPU scope: the thread's earlier
// writes, and those of the CTA ordered before it by __syncthreads, are
// visible to any thread whose acquire load reads this add's result or that
// of a later add to the same counter. (Cheaper than a sequentially
// consistent __threadfence followed by a relaxed atomic: C5 BiCG 28.46 ->
// 28.10 ms, C5 CG 76.3 -> 75.2 ms.)
__device__ __forceinline__ void red_release_add_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Sums of N values over the CTA's 1024 threads in a fixed order; the result
// is valid in thread 0.
template <int N>
__device__ __forceinline__ void ir_block_sum(double (&v)[N], double (*sh)[kIrWarps]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < N; d++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[d] += __shfl_down_sync(0xffffffffu, v[d], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < N; d++) sh[d][w] = v[d];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < N; d++) {
      double s0 = 0.0;
      for (int i = 0; i < kIrWarps; i++) s0 += sh[d][i];
      v[d] = s0;
    }
  }
}

// Grid-wide sums of N values, the same in every CTA; also a barrier (every
// store the CTA's threads made before it is visible to every CTA after it).
// Each CTA writes its partials, counts itself in, waits (bounded) until all G
// have, then sums all partials itself, every load issued before the first
// add and the terms added in one fixed order, so every CTA obtains the same
// bits. Returns false when a wait ran out (the timeout flag is then set).
constexpr int kIrMaxGrid = 256;  // CTAs a reduction takes (one per SM)
constexpr int kIrMaxSums = 2;    // values one reduction carries

// A grid reduction in two halves, so that work which does not need the sums
// runs while the other CTAs arrive: ir_red_post adds the CTA's values (a
// block-wide step: every thread calls it) and counts the CTA in; ir_red_wait
// (every thread) waits for all CTAs and returns the sums.
template <int N>
__device__ __forceinline__ void ir_red_post(const IrArgs &a, unsigned long long gen, double (&v)[N]) {
  static_assert(N >= 1 && N <= kIrMaxSums, "values per reduction");
  __shared__ double sh[kIrMaxSums][kIrWarps];
  ir_block_sum<N>(v, sh);
  if (threadIdx.x == 0) {
    const unsigned G = gridDim.x;
    // Two sets of partials, by the parity of the generation: a CTA writes
    // generation g + 2's only after every CTA has arrived at g + 1, i.e.
    // after every CTA has read generation g's.
    double *part = a.partials + (size_t)(gen & 1) * kIrMaxSums * G;
#pragma unroll
    for (int d = 0; d < N; d++) part[(size_t)d * G + blockIdx.x] = v[d];
    red_release_add_u64(&a.sync->count, 1ull);
  }
}

// Returns false when the wait ran out (the timeout flag is then set).
template <int N>
__device__ __forceinline__ bool ir_red_wait(const IrArgs &a, unsigned long long gen, double (&v)[N]) {
  __shared__ double s_res[kIrMaxSums];
  __shared__ int s_ok;
  const unsigned G = gridDim.x;
  const double *part = a.partials + (size_t)(gen & 1) * kIrMaxSums * G;
  if (threadIdx.x == 0) {
    s_ok = 1;
    const unsigned long long want = gen * (unsigned long long)G;
    const unsigned long long t0 = global_ns();
    while (ld_acquire_u64(&a.sync->count) < want) {
      if (global_ns() - t0 > a.wait_ns) {
        atomicExch(a.err, 1);
        s_ok = 0;
        break;
      }
    }
  }
  __syncthreads();
  if (!s_ok) return false;
  if (threadIdx.x < 32) {
    constexpr int U = kIrMaxGrid / 32;
#pragma unroll
    for (int d = 0; d < N; d++) {
      double pv[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const unsigned b = threadIdx.x + 32u * u;
        pv[u] = b < G ? __ldcg(&part[(size_t)d * G + b]) : 0.0;
      }
      double s0 = 0.0;
#pragma unroll
      for (int u = 0; u < U; u++) s0 += pv[u];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s0 += __shfl_down_sync(0xffffffffu, s0, o);
      if (threadIdx.x == 0) s_res[d] = s0;
    }
  }
  __syncthreads();
#pragma unroll
  for (int d = 0; d < N; d++) v[d] = s_res[d];
  return true;
}

template <int N>
__device__ __forceinline__ bool ir_allreduce(const IrArgs &a, unsigned long long gen, double (&v)[N]) {
  ir_red_post<N>(a, gen, v);
  return ir_red_wait<N>(a, gen, v);
}

// After publishing its rows of p: release this CTA's flag, then wait until
// the CTAs owning the columns its rows read ([bl, bh]) have published the same
// generation. Replaces a grid barrier where only neighbours' values are read.
// Returns false when a wait ran out (the timeout flag is then set).
__device__ __forceinline__ bool ir_publish_sync(const IrArgs &a, unsigned long long gen, int bl, int bh) {
  __shared__ int s_ok;
  __syncthreads();  // every thread's stores of p are ordered before thread 0's release
  if (threadIdx.x == 0) {
    st_release_u64(ir_pub(a.sync, blockIdx.x), gen);
    s_ok = 1;
    const unsigned long long t0 = global_ns();
    for (int q = bl; q <= bh && s_ok; q++) {
      if (q == (int)blockIdx.x) continue;
      while (ld_acquire_u64(ir_pub(a.sync, q)) < gen) {
        if (global_ns() - t0 > a.wait_ns) {
          atomicExch(a.err, 1);
          s_ok = 0;
          break;
        }
      }
    }
  }
  __syncthreads();
  return s_ok != 0;
}

// The matrix values (and FP64 row masks) are loaded with an L2 evict_last
// policy: between two inner solves the outer method's kernels stream its
// FP64 matrix and vectors through L2, and the diagonal copy, read 20 times
// per inner solve, then stays in L2 ahead of them (measured: the inner solve
// ran 425 us with L2 flushed before it and 570 us after the outer kernels,
// without the hint). After the solve ir_l2_release lowers it again.
__device__ __forceinline__ uint64_t ir_pol() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ldl(const float *p) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ double ldl(const double *p) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ unsigned short ldl(const unsigned short *p) {
  unsigned short v;
  asm("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ unsigned ldl(const unsigned *p) {
  unsigned v;
  asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ uint2 ldl2(const void *p) {
  uint2 v;
  asm("ld.global.nc.L2::cache_hint.v2.u32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ float4 ldl4(const float *p) {
  float4 v;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p), "l"(ir_pol()));
  return v;
}
__device__ __forceinline__ double2 ldl2d(const double *p) {
  double2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(ir_pol()));
  return v;
}

template <class MT>
__device__ __forceinline__ MT ir_ld(const MT *p) {
  return ldl(p);
}
template <>
__device__ __forceinline__ __nv_bfloat16 ir_ld<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __ushort_as_bfloat16(ldl(reinterpret_cast<const unsigned short *>(p)));
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
// N consecutive columns of this warp's 32 lanes (one word per column per thread)
__device__ __forceinline__ void tm_st4(uint32_t taddr, const uint32_t (&w)[4]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(w[0]), "r"(w[1]),
               "r"(w[2]), "r"(w[3])
               : "memory");
}
__device__ __forceinline__ void tm_ld4(uint32_t taddr, uint32_t (&w)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
               : "r"(taddr)
               : "memory");
}
// The registers of a load are valid only after the wait; passing them
// through it keeps every use behind it.
__device__ __forceinline__ void tm_wait_ld4(uint32_t (&w)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(w[0]), "+r"(w[1]), "+r"(w[2]), "+r"(w[3])::"memory");
}
__device__ __forceinline__ void tm_wait_ld8(uint32_t (&w)[4], uint32_t (&v)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(w[0]), "+r"(w[1]), "+r"(w[2]), "+r"(w[3]), "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3])::"memory");
}
__device__ __forceinline__ void tm_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

constexpr uint32_t kIrTmemCols = 512;
constexpr int kIrQ = 4;                     // consecutive rows a thread takes at a time
constexpr int kIrTile = kIrThreads * kIrQ;  // rows of one pass of the CTA

// A quad of a thread's rows in TMEM: 4 words per quad in FP32 (16 in the
// thread's 32-word region, so 8 quads), 8 words in FP64 (4 quads).
template <class VT>
struct IrWords {
  static constexpr int W = kIrQ * (int)sizeof(VT) / 4;  // words per quad
  static constexpr int MaxQuads = 32 / W;
  __device__ static void put(uint32_t taddr, const VT (&v)[kIrQ]) {
    if constexpr (sizeof(VT) == 4) {
      const uint32_t w[4] = {__float_as_uint(v[0]), __float_as_uint(v[1]), __float_as_uint(v[2]),
                             __float_as_uint(v[3])};
      tm_st4(taddr, w);
    } else {
      uint32_t w[4], x[4];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const unsigned long long u0 = (unsigned long long)__double_as_longlong(v[e]);
        const unsigned long long u1 = (unsigned long long)__double_as_longlong(v[2 + e]);
        w[2 * e] = (uint32_t)u0;
        w[2 * e + 1] = (uint32_t)(u0 >> 32);
        x[2 * e] = (uint32_t)u1;
        x[2 * e + 1] = (uint32_t)(u1 >> 32);
      }
      tm_st4(taddr, w);
      tm_st4(taddr + 4, x);
    }
  }
  // Two quads (r and q) loaded together, one wait.
  __device__ static void get2(uint32_t ta, VT (&a)[kIrQ], uint32_t tb, VT (&b)[kIrQ]) {
    if constexpr (sizeof(VT) == 4) {
      uint32_t w[4], x[4];
      tm_ld4(ta, w);
      tm_ld4(tb, x);
      tm_wait_ld8(w, x);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        a[e] = __uint_as_float(w[e]);
        b[e] = __uint_as_float(x[e]);
      }
    } else {
      uint32_t w[4], x[4];
      tm_ld4(ta, w);
      tm_ld4(ta + 4, x);
      tm_wait_ld8(w, x);
      a[0] = __longlong_as_double((long long)(((unsigned long long)w[1] << 32) | w[0]));
      a[1] = __longlong_as_double((long long)(((unsigned long long)w[3] << 32) | w[2]));
      a[2] = __longlong_as_double((long long)(((unsigned long long)x[1] << 32) | x[0]));
      a[3] = __longlong_as_double((long long)(((unsigned long long)x[3] << 32) | x[2]));
      tm_ld4(tb, w);
      tm_ld4(tb + 4, x);
      tm_wait_ld8(w, x);
      b[0] = __longlong_as_double((long long)(((unsigned long long)w[1] << 32) | w[0]));
      b[1] = __longlong_as_double((long long)(((unsigned long long)w[3] << 32) | w[2]));
      b[2] = __longlong_as_double((long long)(((unsigned long long)x[1] << 32) | x[0]));
      b[3] = __longlong_as_double((long long)(((unsigned long long)x[3] << 32) | x[2]));
    }
  }
  __device__ static void get(uint32_t ta, VT (&a)[kIrQ]) {
    if constexpr (sizeof(VT) == 4) {
      uint32_t w[4];
      tm_ld4(ta, w);
      tm_wait_ld4(w);
#pragma unroll
      for (int e = 0; e < 4; e++) a[e] = __uint_as_float(w[e]);
    } else {
      uint32_t w[4], x[4];
      tm_ld4(ta, w);
      tm_ld4(ta + 4, x);
      tm_wait_ld8(w, x);
      a[0] = __longlong_as_double((long long)(((unsigned long long)w[1] << 32) | w[0]));
      a[1] = __longlong_as_double((long long)(((unsigned long long)w[3] << 32) | w[2]));
      a[2] = __longlong_as_double((long long)(((unsigned long long)x[1] << 32) | x[0]));
      a[3] = __longlong_as_double((long long)(((unsigned long long)x[3] << 32) | x[2]));
    }
  }
};

// The largest K (rows per thread) the 64 TMEM words of a thread hold, r and q.
template <class VT>
constexpr int ir_max_k() {
  return IrWords<VT>::MaxQuads * kIrQ;
}

// 4 consecutive elements, p[0..3] of one 16-byte-aligned (FP32) or 32-byte-
// aligned (FP64) address; matrix values the same from an 8-byte (BF16) one.
template <class T>
__device__ __forceinline__ void ld4(const T *p, T (&v)[kIrQ], bool global_cg);
template <>
__device__ __forceinline__ void ld4<float>(const float *p, float (&v)[kIrQ], bool cg) {
  const float4 u = cg ? __ldcg(reinterpret_cast<const float4 *>(p)) : ldl4(p);
  v[0] = u.x;
  v[1] = u.y;
  v[2] = u.z;
  v[3] = u.w;
}
template <>
__device__ __forceinline__ void ld4<double>(const double *p, double (&v)[kIrQ], bool cg) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
  const double2 a = cg ? __ldcg(q) : ldl2d(p), b = cg ? __ldcg(q + 1) : ldl2d(p + 2);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}
template <>
__device__ __forceinline__ void ld4<__nv_bfloat16>(const __nv_bfloat16 *p, __nv_bfloat16 (&v)[kIrQ], bool) {
  const uint2 u = ldl2(p);
  v[0] = __ushort_as_bfloat16((unsigned short)(u.x & 0xffffu));
  v[1] = __ushort_as_bfloat16((unsigned short)(u.x >> 16));
  v[2] = __ushort_as_bfloat16((unsigned short)(u.y & 0xffffu));
  v[3] = __ushort_as_bfloat16((unsigned short)(u.y >> 16));
}
template <class T>
__device__ __forceinline__ void lds4(const T *p, T (&v)[kIrQ]) {  // shared memory, aligned as ld4
  if constexpr (sizeof(T) == 4) {
    const float4 u = *reinterpret_cast<const float4 *>(p);
    v[0] = u.x;
    v[1] = u.y;
    v[2] = u.z;
    v[3] = u.w;
  } else {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
  }
}
template <class T>
__device__ __forceinline__ void sts4(T *p, const T (&v)[kIrQ]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  }
}
template <class T>
__device__ __forceinline__ void stcg4(T *p, const T (&v)[kIrQ]) {
  if constexpr (sizeof(T) == 4) {
    __stcg(reinterpret_cast<float4 *>(p), make_float4(v[0], v[1], v[2], v[3]));
  } else {
    __stcg(reinterpret_cast<double2 *>(p), make_double2(v[0], v[1]));
    __stcg(reinterpret_cast<double2 *>(p) + 1, make_double2(v[2], v[3]));
  }
}

// A quad of matrix values as loaded: packed where MT is narrower than 4
// bytes (BF16: two per register, unpacked at use).
template <class MT>
struct IrVals {
  MT v[kIrQ];
  __device__ __forceinline__ float get(int e) const { return mval<float>(v[e]); }
};
template <>
struct IrVals<__nv_bfloat16> {
  uint2 u;
  __device__ __forceinline__ float get(int e) const {
    const unsigned w = e < 2 ? u.x : u.y;
    return __uint_as_float((e & 1) ? (w & 0xffff0000u) : (w << 16));
  }
};

// The values of diagonal d for rows i0 .. i0+3: one vector load where all 4
// rows are present and the address is aligned, else one load per row.
template <class MT>
__device__ __forceinline__ void ir_vals(const MT *vp, bool full, int li0, int nr, IrVals<MT> &a) {
  const bool aligned = (reinterpret_cast<uintptr_t>(vp) & (kIrQ * sizeof(MT) - 1)) == 0;
  if constexpr (std::is_same<MT, __nv_bfloat16>::value) {
    if (full && aligned) {
      a.u = ldl2(vp);
    } else {
      unsigned short h[kIrQ];
#pragma unroll
      for (int e = 0; e < kIrQ; e++) h[e] = li0 + e < nr ? ldl(reinterpret_cast<const unsigned short *>(vp) + e) : 0;
      a.u = make_uint2(h[0] | ((unsigned)h[1] << 16), h[2] | ((unsigned)h[3] << 16));
    }
  } else {
    if (full && aligned) {
      ld4<MT>(vp, a.v, false);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++) a.v[e] = li0 + e < nr ? ldl(vp + e) : (MT)0;
    }
  }
}

// A thread's own quad of a shared-memory vector: one vector access for a full
// quad (a scalar one per row would hit 4 threads on one bank), else per row.
template <class VT>
__device__ __forceinline__ void ir_own4(const VT *v, int li0, int nr, VT (&o)[kIrQ]) {
  if (li0 + kIrQ <= nr) {
    lds4<VT>(v + li0, o);
  } else {
#pragma unroll
    for (int e = 0; e < kIrQ; e++) o[e] = li0 + e < nr ? v[li0 + e] : (VT)0;
  }
}

// p[c .. c+3] for an aligned column c: one vector load from the CTA's shared
// copy or from P when the 4 columns are all on one side of the CTA's rows and
// inside [cmin, cmax); else per column, clamped into the window (whose terms
// have zero matrix values).
template <class VT>
__device__ __forceinline__ void ir_p4(const VT *sp, const VT *P, int r0, int nr, int cmin, int cmax, int c,
                                      VT (&p)[kIrQ]) {
  const int lc = c - r0;
  if (lc >= 0 && lc + kIrQ <= nr) {
    lds4<VT>(sp + lc, p);
  } else if (c >= cmin && c + kIrQ <= cmax && (lc + kIrQ <= 0 || lc >= nr)) {
    ld4<VT>(P + c, p, true);
  } else {
#pragma unroll
    for (int e = 0; e < kIrQ; e++) {
      const int cc = min(max(c + e, cmin), cmax - 1);
      const int l = cc - r0;
      p[e] = (l >= 0 && l < nr) ? sp[l] : __ldcg(P + cc);
    }
  }
}

// q = A p for the 4 consecutive rows i0 .. i0+3 (local li0 .. li0+3, i0 a
// multiple of 4) of a thread, diagonals in ascending offset order (the
// row's CSR order), in batches whose loads are all issued before the batch
// is summed. p at an offset o: the aligned quad when 4 divides o, else the
// two aligned quads around it and a funnel by o mod 4 (uniform across the
// warp). Every diagonal's value is loaded (zeros where a row has none); FP64
// adds only the terms the row's mask names, FP32 adds every one.
template <class VT, class MT, int NDG>
__device__ __forceinline__ void ir_quad_mv(const DiaT<MT> &D, const VT *P, const VT *sp, int r0, int nr, int li0,
                                           int nd, VT (&q)[kIrQ]) {
  constexpr int KD = NDG > 0 ? NDG : kMaxDiag;
  constexpr int B = sizeof(MT) == 2 ? KD : (sizeof(MT) == 4 ? 4 : 2);  // diagonals per batch
  constexpr bool kMask = std::is_same<MT, double>::value;
  const int i0 = r0 + li0;
  const bool full = li0 + kIrQ <= nr;
  unsigned m = 0xffffffffu;  // the rows' mask bytes, row e in byte e
  if constexpr (kMask) {
    if (full) {
      m = ldl(reinterpret_cast<const unsigned *>(D.mask + i0));
    } else {
      m = 0;
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) m |= (unsigned)__ldg(D.mask + i0 + e) << (8 * e);
    }
  }
#pragma unroll
  for (int e = 0; e < kIrQ; e++) q[e] = (VT)0;
#pragma unroll
  for (int d0 = 0; d0 < KD; d0 += B) {
    IrVals<MT> av[B];
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int d = d0 + u;
      if (d < KD && (NDG > 0 || d < nd)) ir_vals<MT>(D.vb[d] + (i0 + D.vs[d]), full, li0, nr, av[u]);
    }
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int d = d0 + u;
      if (d < KD && (NDG > 0 || d < nd)) {
        const int c0 = i0 + D.off[d];
        const int sh = c0 & (kIrQ - 1);
        VT pv[kIrQ];
        if (sh == 0) {
          ir_p4<VT>(sp, P, r0, nr, D.cmin, D.cmax, c0, pv);
        } else {
          VT lo[kIrQ], hi[kIrQ];
          ir_p4<VT>(sp, P, r0, nr, D.cmin, D.cmax, c0 - sh, lo);
          ir_p4<VT>(sp, P, r0, nr, D.cmin, D.cmax, c0 - sh + kIrQ, hi);
#pragma unroll
          for (int e = 0; e < kIrQ; e++) {
            const int k = e + sh;  // 1 .. 6
            pv[e] = k == 1 ? lo[1] : k == 2 ? lo[2] : k == 3 ? lo[3] : k == 4 ? hi[0] : k == 5 ? hi[1] : hi[2];
          }
        }
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          VT val;
          if constexpr (std::is_same<MT, __nv_bfloat16>::value)
            val = av[u].get(e);
          else
            val = (VT)av[u].v[e];
          const VT t = add_rn(q[e], mul_rn(val, pv[e]));
          if constexpr (kMask)
            q[e] = ((m >> (8 * e + d)) & 1u) ? t : q[e];
          else
            q[e] = t;
        }
      }
    }
  }
}

// Matrix values of one stored diagonal for 4 rows from an aligned address.
template <class MT>
__device__ __forceinline__ void ir_vals4(const MT *vp, IrVals<MT> &a) {
  if constexpr (std::is_same<MT, __nv_bfloat16>::value)
    a.u = ldl2(vp);
  else
    ld4<MT>(vp, a.v, false);
}
template <class VT, class MT>
__device__ __forceinline__ VT ir_val(const IrVals<MT> &a, int e) {
  if constexpr (std::is_same<MT, __nv_bfloat16>::value)
    return a.get(e);
  else
    return (VT)a.v[e];
}

// q = A p for a full quad (rows i0 .. i0+3 all in the CTA) of a 5- or
// 7-point stencil whose diagonals lie at 0, +-1 and (+-b, +-c) with b and c
// multiples of 4, P zero-padded beyond [0, n) by more than the largest
// offset (ir_stencil_ok). Without per-diagonal alignment tests or clamps:
//   * p of the +-1 diagonals is the own quad pv shifted by one row, plus
//     p[i0-1] and p[i0+4]; each far diagonal's 4 columns are one aligned
//     quad, from shared memory when inside the CTA's rows, else from P;
//   * matrix values are one aligned vector per diagonal; in the symmetric
//     layout the -1 diagonal of rows i0 .. i0+3 is the +1 diagonal of rows
//     i0-1 .. i0+2: the +1 vector shifted by one row and one scalar.
// A column outside [0, n) has a zero value and reads a zero of P's pad
// (ir_quad_mv reads a clamped column instead): the term adds a zero to a sum
// that starts at +0, which leaves it unchanged, so the terms and their order
// are ir_quad_mv's and so are the results.
template <class VT, class MT, int NDG>
__device__ __forceinline__ void ir_quad_mv_st(const DiaT<MT> &D, const VT *P, const VT *sp, int r0, int nr, int li0,
                                              const VT (&pv)[kIrQ], VT (&q)[kIrQ]) {
  static_assert(NDG == 5 || NDG == 7, "stencil path: 5 or 7 diagonals");
  constexpr int H = NDG / 2;  // the main diagonal
  constexpr bool kMask = std::is_same<MT, double>::value;
  const int i0 = r0 + li0;
  const bool sym = D.vs[H - 1] != 0;  // -1 diagonal read from its +1 mirror
  unsigned m = 0xffffffffu;
  if constexpr (kMask) m = ldl(reinterpret_cast<const unsigned *>(D.mask + i0));
  // p: the -1 / +1 neighbours of the quad, then the far diagonals' quads
  const VT pm1 = li0 >= 1 ? sp[li0 - 1] : __ldcg(P + (i0 - 1));
  const VT pp4 = li0 + kIrQ < nr ? sp[li0 + kIrQ] : __ldcg(P + (i0 + kIrQ));
  IrVals<MT> vm1, v1;
  ir_vals4<MT>(D.vb[H + 1] + i0, v1);
  MT m1s = (MT)0;
  if (sym)
    m1s = ir_ld<MT>(D.vb[H + 1] + (i0 - 1));
  else
    ir_vals4<MT>(D.vb[H - 1] + i0, vm1);
#pragma unroll
  for (int e = 0; e < kIrQ; e++) q[e] = (VT)0;
  auto term = [&](int k, const VT (&val)[kIrQ], const VT (&p)[kIrQ]) {
#pragma unroll
    for (int e = 0; e < kIrQ; e++) {
      const VT t = add_rn(q[e], mul_rn(val[e], p[e]));
      if constexpr (kMask)
        q[e] = ((m >> (8 * e + k)) & 1u) ? t : q[e];
      else
        q[e] = t;
    }
  };
  auto far = [&](int k) {
    const int off = D.off[k];
    IrVals<MT> av;
    ir_vals4<MT>(D.vb[k] + (i0 + D.vs[k]), av);
    VT p[kIrQ], val[kIrQ];
    const int lc = li0 + off;
    if (lc >= 0 && lc + kIrQ <= nr)
      lds4<VT>(sp + lc, p);
    else
      ld4<VT>(P + (i0 + off), p, true);
#pragma unroll
    for (int e = 0; e < kIrQ; e++) val[e] = ir_val<VT, MT>(av, e);
    term(k, val, p);
  };
  // ascending offsets: the far lower diagonals, -1, 0, +1, the far upper ones
#pragma unroll
  for (int k = 0; k < H - 1; k++) far(k);
  {
    VT val[kIrQ];
    const VT p[kIrQ] = {pm1, pv[0], pv[1], pv[2]};
    if (sym) {
      val[0] = (VT)mval<VT>(m1s);
#pragma unroll
      for (int e = 1; e < kIrQ; e++) val[e] = ir_val<VT, MT>(v1, e - 1);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++) val[e] = ir_val<VT, MT>(vm1, e);
    }
    term(H - 1, val, p);
  }
  {
    IrVals<MT> v0;
    ir_vals4<MT>(D.vb[H] + i0, v0);
    VT val[kIrQ];
#pragma unroll
    for (int e = 0; e < kIrQ; e++) val[e] = ir_val<VT, MT>(v0, e);
    term(H, val, pv);
  }
  {
    VT val[kIrQ];
    const VT p[kIrQ] = {pv[1], pv[2], pv[3], pp4};
#pragma unroll
    for (int e = 0; e < kIrQ; e++) val[e] = ir_val<VT, MT>(v1, e);
    term(H + 1, val, p);
  }
#pragma unroll
  for (int k = H + 2; k < NDG; k++) far(k);
}

// The solve (see the top of this file). Returns the stopping code, or -1
// when a wait ran out; *xw: x was written (one update at least).
template <class VT, class MT, int NDG>
__device__ __forceinline__ int ir_body(const DiaT<MT> &D, const IrArgs &a, VT *sp, VT *sx, uint32_t tm,
                                       long long *Lout, double *alpha_out, double *beta_out, double *rr_out,
                                       bool *xw) {
  using TW = IrWords<VT>;
  const int nd = NDG > 0 ? NDG : D.nd;
  const int t = threadIdx.x;
  const int r0 = blockIdx.x * a.rpc;
  const int nr = max(0, min(a.rpc, a.n - r0));
  const bool lead = blockIdx.x == 0 && t == 0;  // keeps the method's state (whole solve)
  DevState *st = a.st;
  VT *P = (VT *)a.P;
  const double eps = st->k.s[S_EPS];
  const long long maxloop = st->k.aux[A_MAXLOOP];
  const int quads = (a.rpc + kIrTile - 1) / kIrTile;  // quads per thread
  const uint32_t tr = tm, tq = tm + 32;  // this thread's r at column tr + W j, q at tq + W j
  // the CTAs owning the columns this CTA's rows read
  int bl = blockIdx.x, bh = blockIdx.x;
  if (nr > 0) {
    const int lo = max(r0 + D.off[0], D.cmin), hi = min(r0 + nr - 1 + D.off[nd - 1], D.cmax - 1);
    bl = min(bl, lo / a.rpc);
    bh = max(bh, hi / a.rpc);
  }

  // start: r = b (TMEM), p = r (shared memory and P), x = 0
  double acc = 0.0;
  for (int j = 0; j < quads; j++) {
    const int li0 = j * kIrTile + kIrQ * t;
    VT v[kIrQ];
#pragma unroll
    for (int e = 0; e < kIrQ; e++) {
      const int li = li0 + e;
      v[e] = li < nr ? __ldcg((const VT *)a.rin + r0 + li) : (VT)0;
      if (li < nr) acc = add_rn(acc, mul_rn(widen(v[e]), widen(v[e])));
    }
    if (li0 + kIrQ <= nr) {
      const VT z[kIrQ] = {(VT)0, (VT)0, (VT)0, (VT)0};
      sts4<VT>(sp + li0, v);
      sts4<VT>(sx + li0, z);
      stcg4<VT>(P + r0 + li0, v);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++) {
        const int li = li0 + e;
        if (li < nr) {
          sp[li] = v[e];
          sx[li] = (VT)0;
          __stcg(P + r0 + li, v[e]);
        }
      }
    }
    TW::put(tr + TW::W * j, v);
  }
  tm_wait_st();
  unsigned long long gen = 0, pgen = 1;  // reductions, publications of p
  double v[1] = {0.0};
  double rr, bnorm;
  int code = kRunning;
  if (a.whole) {
    // |b| and the stopping test at the top of iteration 1 (NormBOp, StartZeroOp)
    v[0] = acc;
    if (!ir_allreduce(a, ++gen, v)) return -1;
    rr = v[0];
    bnorm = sqrt(rr);
    const double err = sqrt(rr) / bnorm;
    if (1 > maxloop)
      code = kMaxLoop;
    else if (err <= eps)
      code = kConverged;
    else if (err != err)
      code = kNaN;
    if (lead) {
      st->k.s[S_BNORM] = bnorm;
      st->k.s[S_RR] = rr;
      check_top(st, 1, err);
    }
    if (code != kRunning) return code;
  } else {
    rr = st->k.s[S_RR];
    bnorm = st->k.s[S_BNORM];
  }
  if (!ir_publish_sync(a, pgen, bl, bh)) return -1;

  double alpha = 0.0, beta = 0.0;
  long long L = 1;
  for (; L <= maxloop; L++) {
    // A: q = A p, (p, q)
    acc = 0.0;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      VT q[kIrQ], pv[kIrQ];
      ir_own4(sp, li0, nr, pv);
      bool st_done = false;
      if constexpr (NDG == 5 || NDG == 7) {
        if (a.stencil && li0 + kIrQ <= nr) {
          ir_quad_mv_st<VT, MT, NDG>(D, P, sp, r0, nr, li0, pv, q);
          st_done = true;
        }
      }
      if (!st_done) ir_quad_mv<VT, MT, NDG>(D, P, sp, r0, nr, li0, nd, q);
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) acc = add_rn(acc, mul_rn(widen(pv[e]), widen(q[e])));
      TW::put(tq + TW::W * j, q);
    }
    tm_wait_st();
    v[0] = acc;
    if (!ir_allreduce(a, ++gen, v)) return -1;
    // alpha = rr / (p, q)   (rdiv: a zero denominator is a breakdown)
    if (v[0] == 0.0) {
      code = kBreakdown;
      alpha = 0.0;
    } else {
      alpha = div_rn(rr, v[0]);
      if (!isfinite(alpha)) code = kNaN;
    }
    if (code != kRunning) {
      if (lead && a.whole) set_done(st, code);
      break;
    }
    // B: r -= alpha q and (r, r), whose sum is posted; then x += alpha p
    // (nothing waits for it) while the other CTAs arrive
    const VT av = (VT)alpha;
    acc = 0.0;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      VT rv[kIrQ], qv[kIrQ];
      TW::get2(tr + TW::W * j, rv, tq + TW::W * j, qv);
#pragma unroll
      for (int e = 0; e < kIrQ; e++) {
        rv[e] = add_rn(mul_rn((VT)(-av), qv[e]), rv[e]);  // rows past nr: unused words
        if (li0 + e < nr) acc = add_rn(acc, mul_rn(widen(rv[e]), widen(rv[e])));
      }
      TW::put(tr + TW::W * j, rv);
    }
    tm_wait_st();
    v[0] = acc;
    ir_red_post<1>(a, ++gen, v);
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      if (li0 + kIrQ <= nr) {  // vector accesses: the 4 rows of a thread are one aligned quad
        VT pv[kIrQ], xv[kIrQ];
        lds4<VT>(sp + li0, pv);
        lds4<VT>(sx + li0, xv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) xv[e] = add_rn(mul_rn(av, pv[e]), xv[e]);
        sts4<VT>(sx + li0, xv);
      } else {
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          const int li = li0 + e;
          if (li < nr) sx[li] = add_rn(mul_rn(av, sp[li]), sx[li]);
        }
      }
    }
    *xw = true;
    if (!ir_red_wait<1>(a, gen, v)) return -1;
    // beta = (r, r)_new / (r, r); then the stopping test at the top of
    // iteration L + 1 (check_top), whose verdict overrides beta's
    const double rr2 = v[0];
    int bcode = kRunning;
    if (rr == 0.0) {
      bcode = kBreakdown;
      beta = 0.0;
    } else {
      beta = div_rn(rr2, rr);
      if (!isfinite(beta)) bcode = kNaN;
    }
    rr = rr2;
    const double err = sqrt(rr2) / bnorm;
    code = bcode;
    if (L + 1 > maxloop)
      code = kMaxLoop;
    else if (err <= eps)
      code = kConverged;
    else if (err != err)
      code = kNaN;
    if (lead && a.whole) {
      if (bcode != kRunning) set_done(st, bcode);
      check_top(st, L + 1, err);
    }
    if (code != kRunning) break;
    // C: p = beta p + r, published
    const VT bv = (VT)beta;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      VT rv[kIrQ];
      TW::get(tr + TW::W * j, rv);
      if (li0 + kIrQ <= nr) {
        VT pv[kIrQ];
        lds4<VT>(sp + li0, pv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) pv[e] = add_rn(mul_rn(bv, pv[e]), rv[e]);
        sts4<VT>(sp + li0, pv);
        stcg4<VT>(P + r0 + li0, pv);
      } else {
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          const int li = li0 + e;
          if (li < nr) {
            const VT pn = add_rn(mul_rn(bv, sp[li]), rv[e]);
            sp[li] = pn;
            __stcg(P + r0 + li, pn);
          }
        }
      }
    }
    if (!ir_publish_sync(a, ++pgen, bl, bh)) return -1;
  }
  *Lout = L;
  *alpha_out = alpha;
  *beta_out = beta;
  *rr_out = rr;
  return code;
}

template <class VT, class MT, int NDG>
__global__ void __launch_bounds__(kIrThreads, 1) k_cg_onchip(DiaT<MT> D, IrArgs a) {
  extern __shared__ __align__(16) unsigned char ir_smem_raw[];
  __shared__ uint32_t s_tmem;
  VT *sp = reinterpret_cast<VT *>(ir_smem_raw);  // p of the CTA's rows
  VT *sx = sp + a.rpc;                           // x of the CTA's rows
  const int t = threadIdx.x;
  DevState *st = a.st;
  // The start conditions come from kernels that completed before this one,
  // so every CTA reads the same values and all of them return here together.
  if (a.outer_done && *(volatile const int *)a.outer_done) return;
  if (*(volatile const int *)&st->k.done != kRunning) return;  // inner: x stays 0 (A_XZERO)
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
  const int code = ir_body<VT, MT, NDG>(D, a, sp, sx, tm, &L, &alpha, &beta, &rr, &xw);
  if (code >= 0) {
    // x out (a whole solve writes its zeros too): thread t reads rows other
    // threads updated last (the loop may end right after an update pass), so
    // the CTA synchronises first; code is the same in every thread
    __syncthreads();
    const int r0 = blockIdx.x * a.rpc;
    const int nr = max(0, min(a.rpc, a.n - r0));
    VT *x = (VT *)a.x;
    if (xw || a.whole)
      for (int li = t; li < nr; li += kIrThreads) __stcg(x + r0 + li, xw ? sx[li] : (VT)0);
    if (blockIdx.x == 0 && t == 0) {
      st->k.s[S_ALPHA] = alpha;
      st->k.s[S_BETA] = beta;
      if (!a.whole) {  // the state the kernel-per-step inner loop leaves (nothing pending)
        st->k.done = code == kRunning ? kMaxLoop : code;
        st->k.loop = code == kBreakdown || code == kNaN ? L : L + 1;
        st->k.s[S_RR] = rr;
        st->k.aux[A_PENDING] = 0;
        st->k.aux[A_XZERO] = xw ? 0 : 1;
      }
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


// ---------------------------------------------------------------- BiCG on chip
// BiCG (bicg.cpp:148-260) as one cooperative launch of one CTA per SM, for
// FP64 systems above the thread-block-cluster limit whose six vectors fit in
// shared memory with one quad of rows per thread (rpc <= kIrTile: up to
// about 606K rows), A and A^T with a diagonal copy (the stencil quad path
// where ir_stencil_ok holds for both, else the generic one): x, r, r*, p, p*
// and q = A p of the CTA's rows in shared
// memory; p and p* also published to P and P* (zero-padded), from which the
// other CTAs gather the columns their rows reach. Per iteration, in the
// engine's order:
//   A: q = A p, (p*, q) summed over the grid -> alpha = (r*, r) / (p*, q);
//   B: x += alpha p, r -= alpha q, r* -= alpha A^T p*, then (r, r) and
//      (r*, r) in one reduction -> the stopping test on |r| / |b| at the top
//      of iteration L + 1 (the engine's XrUpdOp) and, unless it stops, beta =
//      (r*, r)_new / (r*, r);
//   C: p = beta p + r, p* = beta p* + r*, published; each CTA then waits for
//      the CTAs owning the columns its rows read through A or A^T.
// Element operations are the engine's (CgMvEpi, XrUpdOp, BicgMvTEpi,
// Xpby2PlainOp) in the same order; only the dot products add their terms in
// another order (per thread, a fixed tree over the CTA, the CTAs' partials in
// index order). Every wait is bounded (ir_allreduce, ir_publish_sync).
constexpr int kIbVecs = 6;

template <int NDG>
__global__ void __launch_bounds__(kIrThreads, 1) k_bicg_onchip(DiaT<double> DA, DiaT<double> DT, IrArgs a) {
  extern __shared__ __align__(16) unsigned char ir_smem_raw[];
  double *sx = reinterpret_cast<double *>(ir_smem_raw);
  double *sr = sx + a.rpc, *srs = sr + a.rpc, *sp = srs + a.rpc, *sps = sp + a.rpc, *sq = sps + a.rpc;
  const int t = threadIdx.x;
  const int r0 = blockIdx.x * a.rpc;
  const int nr = max(0, min(a.rpc, a.n - r0));
  const int li0 = kIrQ * t;  // the thread's quad of rows (rpc <= kIrTile)
  const bool mine = li0 < nr, full = li0 + kIrQ <= nr;
  const bool lead = blockIdx.x == 0 && t == 0;
  DevState *st = a.st;
  double *P = (double *)a.P, *Ps = (double *)a.P2;
  const double eps = st->k.s[S_EPS];
  const long long maxloop = st->k.aux[A_MAXLOOP];
  // the CTAs owning the columns this CTA's rows read through A or A^T
  int bl = blockIdx.x, bh = blockIdx.x;
  if (nr > 0) {
    const int nda = NDG > 0 ? NDG : DA.nd, ndt = NDG > 0 ? NDG : DT.nd;
    const int lo = max(r0 + min(DA.off[0], DT.off[0]), 0);
    const int hi = min(r0 + nr - 1 + max(DA.off[nda - 1], DT.off[ndt - 1]), a.n - 1);
    bl = min(bl, lo / a.rpc);
    bh = max(bh, hi / a.rpc);
  }
  // one quad of a shared-memory vector in / out (vector access where full)
  auto get = [&](const double *v, double (&o)[kIrQ]) { ir_own4(v, li0, nr, o); };
  auto put = [&](double *v, const double (&o)[kIrQ]) {
    if (full) {
      sts4<double>(v + li0, o);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) v[li0 + e] = o[e];
    }
  };
  auto publish = [&](double *G, const double (&o)[kIrQ]) {
    if (full) {
      stcg4<double>(G + r0 + li0, o);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) __stcg(G + r0 + li0 + e, o[e]);
    }
  };
  auto mv = [&](const DiaT<double> &D, const double *G, const double *sv, const double (&own)[kIrQ],
                double (&y)[kIrQ]) {
    bool done = false;
    if constexpr (NDG == 5 || NDG == 7) {
      if (a.stencil && full) {
        ir_quad_mv_st<double, double, NDG>(D, G, sv, r0, nr, li0, own, y);
        done = true;
      }
    }
    if (!done) ir_quad_mv<double, double, NDG>(D, G, sv, r0, nr, li0, NDG > 0 ? NDG : D.nd, y);
  };

  // start (x0 = 0): r = r* = p = p* = b, x = 0; (r, r) -> |b| and the
  // stopping test at the top of iteration 1 (NormBOp, StartEpi)
  double acc = 0.0;
  if (mine) {
    double v[kIrQ], z[kIrQ];
#pragma unroll
    for (int e = 0; e < kIrQ; e++) {
      const int li = li0 + e;
      v[e] = li < nr ? __ldcg((const double *)a.rin + r0 + li) : 0.0;
      z[e] = 0.0;
      if (li < nr) acc = add_rn(acc, mul_rn(v[e], v[e]));
    }
    put(sx, z);
    put(sr, v);
    put(srs, v);
    put(sp, v);
    put(sps, v);
    publish(P, v);
    publish(Ps, v);
  }
  unsigned long long gen = 0, pgen = 1;
  double s1[1] = {acc};
  if (!ir_allreduce(a, ++gen, s1)) return;
  double rr = s1[0];
  const double bnorm = sqrt(rr);
  int code = kRunning;
  {
    const double err = sqrt(rr) / bnorm;
    if (1 > maxloop)
      code = kMaxLoop;
    else if (err <= eps)
      code = kConverged;
    else if (err != err)
      code = kNaN;
    if (lead) {
      st->k.s[S_BNORM] = bnorm;
      st->k.s[S_RR] = rr;
      check_top(st, 1, err);
    }
  }
  bool xw = false;
  double alpha = 0.0, beta = 0.0;
  if (code == kRunning) {
    if (!ir_publish_sync(a, pgen, bl, bh)) return;
    for (long long L = 1; L <= maxloop; L++) {
      // A: q = A p, (p*, q) -> alpha
      acc = 0.0;
      if (mine) {
        double pv[kIrQ], psv[kIrQ], q[kIrQ];
        get(sp, pv);
        mv(DA, P, sp, pv, q);
        get(sps, psv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++)
          if (li0 + e < nr) acc = add_rn(acc, mul_rn(psv[e], q[e]));
        put(sq, q);
      }
      s1[0] = acc;
      if (!ir_allreduce(a, ++gen, s1)) return;
      if (s1[0] == 0.0) {
        code = kBreakdown;
        alpha = 0.0;
      } else {
        alpha = div_rn(rr, s1[0]);
        if (!isfinite(alpha)) code = kNaN;
      }
      if (code != kRunning) {
        if (lead) set_done(st, code);
        break;
      }
      // B: x += alpha p, r -= alpha q, r* -= alpha A^T p*; (r, r), (r*, r)
      double s2[2] = {0.0, 0.0};
      if (mine) {
        double psv[kIrQ], w[kIrQ];
        get(sps, psv);
        mv(DT, Ps, sps, psv, w);
        double pv[kIrQ], qv[kIrQ], xv[kIrQ], rv[kIrQ], rsv[kIrQ];
        get(sp, pv);
        get(sq, qv);
        get(sx, xv);
        get(sr, rv);
        get(srs, rsv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          xv[e] = add_rn(mul_rn(alpha, pv[e]), xv[e]);
          rv[e] = add_rn(mul_rn(-alpha, qv[e]), rv[e]);
          rsv[e] = add_rn(mul_rn(-alpha, w[e]), rsv[e]);
          if (li0 + e < nr) {
            s2[0] = add_rn(s2[0], mul_rn(rv[e], rv[e]));
            s2[1] = add_rn(s2[1], mul_rn(rsv[e], rv[e]));
          }
        }
        put(sx, xv);
        put(sr, rv);
        put(srs, rsv);
      }
      xw = true;
      if (!ir_allreduce(a, ++gen, s2)) return;
      // the stopping test at the top of iteration L + 1 comes first; beta
      // only where the method goes on
      const double err = sqrt(s2[0]) / bnorm;
      if (L + 1 > maxloop)
        code = kMaxLoop;
      else if (err <= eps)
        code = kConverged;
      else if (err != err)
        code = kNaN;
      if (lead) check_top(st, L + 1, err);
      if (code != kRunning) break;
      if (rr == 0.0) {
        code = kBreakdown;
        beta = 0.0;
      } else {
        beta = div_rn(s2[1], rr);
        if (!isfinite(beta)) code = kNaN;
      }
      rr = s2[1];
      if (lead) {
        st->k.s[S_BETA] = beta;
        st->k.s[S_RR] = rr;
        if (code != kRunning) set_done(st, code);
      }
      if (code != kRunning) break;
      // C: p = beta p + r, p* = beta p* + r*, published
      if (mine) {
        double pv[kIrQ], rv[kIrQ], psv[kIrQ], rsv[kIrQ];
        get(sp, pv);
        get(sr, rv);
        get(sps, psv);
        get(srs, rsv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          pv[e] = add_rn(mul_rn(beta, pv[e]), rv[e]);
          psv[e] = add_rn(mul_rn(beta, psv[e]), rsv[e]);
        }
        put(sp, pv);
        put(sps, psv);
        publish(P, pv);
        publish(Ps, psv);
      }
      if (!ir_publish_sync(a, ++pgen, bl, bh)) return;
    }
  }
  // x out (zeros if the method stopped before its first update); thread t
  // reads rows other threads updated last
  __syncthreads();
  double *x = (double *)a.x;
  for (int li = t; li < nr; li += kIrThreads) __stcg(x + r0 + li, xw ? sx[li] : 0.0);
  if (lead) {
    st->k.s[S_ALPHA] = alpha;
    if (code == kRunning) st->k.done = kMaxLoop;
  }
}

template <int NDG>
inline cudaError_t ib_launch_n(ks_ctx *ctx, const CsrDev &A, const CsrDev &T, const IrArgs &a, size_t smem,
                               int G, bool probe, bool *fits) {
  auto fn = k_bicg_onchip<NDG>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (probe) {
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kIrThreads, smem);
    *fits = e == cudaSuccess && b >= 1;
    return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G);
  cfg.blockDim = dim3(kIrThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ctx->launches++;
  ctx->ir_used = true;  // its matrix lines are evict_last in L2 (ir_l2_release)
  ProfLaunch pl(ctx, kMv);  // a profiled solve counts the whole solve as one SpMV-class launch
  return cudaLaunchKernelEx(&cfg, fn, dview<double>(A), dview<double>(T), a);
}


// ---------------------------------------------------------------- CR on chip
// CR (cr.cpp:151-250) as one cooperative launch of one CTA per SM, for FP64
// stencil systems above the cluster limit up to ~2.1M rows (ir_shape<double>):
// r and p of the CTA's rows in shared memory, q = A p and s = A r in TMEM
// (lanes and columns as in k_cg_onchip), x in global memory, updated in
// place with streaming (evict-first) accesses. r, the SpMV's input, is also
// published to a zero-padded array R.
// Per iteration, in the engine's order (XrUpdOp, CrMvEpi, Xpby2ToOp):
//   B: r -= alpha q, stored and published, (r, r) posted; x += alpha p in the
//      reduction's shadow -> the stopping test at the top of iteration L + 1;
//      the reduction is also the barrier after which every CTA reads R;
//   A: s = A r, (r, s) -> beta = (r, s) / rs, rs = (r, s);
//   C: p = beta p + r, q = beta q + s, (q, q) -> alpha = rs / (q, q).
// Three grid reductions and no publication wait per iteration; element
// operations are the engine's, only the dot sums' order differs.
template <int NDG>
__global__ void __launch_bounds__(kIrThreads, 1) k_cr_onchip(DiaT<double> D, IrArgs a) {
  using TW = IrWords<double>;
  extern __shared__ __align__(16) unsigned char ir_smem_raw[];
  __shared__ uint32_t s_tmem;
  double *sr = reinterpret_cast<double *>(ir_smem_raw);  // r of the CTA's rows
  double *sp = sr + a.rpc;                                // p of the CTA's rows
  const int t = threadIdx.x;
  const int r0 = blockIdx.x * a.rpc;
  const int nr = max(0, min(a.rpc, a.n - r0));
  const int quads = (a.rpc + kIrTile - 1) / kIrTile;
  const bool lead = blockIdx.x == 0 && t == 0;
  DevState *st = a.st;
  double *R = (double *)a.P, *x = (double *)a.x;
  const double eps = st->k.s[S_EPS];
  const long long maxloop = st->k.aux[A_MAXLOOP];
  if (t < 32) {
    tm_alloc(&s_tmem, kIrTmemCols);
    tm_relinquish();
    tm_fence_before();
  }
  __syncthreads();
  tm_fence_after();
  const uint32_t w = t >> 5;
  const uint32_t tm = s_tmem + ((32u * (w & 3u)) << 16) + 64u * (w >> 2);
  const uint32_t tq = tm, ts = tm + 32;  // q and s of the thread's quads, TW::W words apart
  auto own = [&](const double *v, int li0, double (&o)[kIrQ]) { ir_own4(v, li0, nr, o); };
  auto put = [&](double *v, int li0, const double (&o)[kIrQ]) {
    if (li0 + kIrQ <= nr) {
      sts4<double>(v + li0, o);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) v[li0 + e] = o[e];
    }
  };
  auto gput = [&](double *G, int li0, const double (&o)[kIrQ]) {
    if (li0 + kIrQ <= nr) {
      stcg4<double>(G + r0 + li0, o);
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) __stcg(G + r0 + li0 + e, o[e]);
    }
  };
  // x is read and written once per iteration: streamed (evict-first), so
  // that its lines do not push the matrix and R out of L2
  auto xget = [&](int li0, double (&o)[kIrQ]) {
    if (li0 + kIrQ <= nr) {
      const double2 *q2 = reinterpret_cast<const double2 *>(x + r0 + li0);
      const double2 u = __ldcs(q2), v = __ldcs(q2 + 1);
      o[0] = u.x;
      o[1] = u.y;
      o[2] = v.x;
      o[3] = v.y;
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++) o[e] = li0 + e < nr ? __ldcs(x + r0 + li0 + e) : 0.0;
    }
  };
  auto xput = [&](int li0, const double (&o)[kIrQ]) {
    if (li0 + kIrQ <= nr) {
      double2 *q2 = reinterpret_cast<double2 *>(x + r0 + li0);
      __stcs(q2, make_double2(o[0], o[1]));
      __stcs(q2 + 1, make_double2(o[2], o[3]));
    } else {
#pragma unroll
      for (int e = 0; e < kIrQ; e++)
        if (li0 + e < nr) __stcs(x + r0 + li0 + e, o[e]);
    }
  };
  auto mv = [&](int li0, const double (&own4)[kIrQ], double (&y)[kIrQ]) {
    bool done = false;
    if constexpr (NDG == 5 || NDG == 7) {
      if (a.stencil && li0 + kIrQ <= nr) {
        ir_quad_mv_st<double, double, NDG>(D, R, sr, r0, nr, li0, own4, y);
        done = true;
      }
    }
    if (!done) ir_quad_mv<double, double, NDG>(D, R, sr, r0, nr, li0, NDG > 0 ? NDG : D.nd, y);
  };
  unsigned long long gen = 0;
  int code = kRunning;
  double alpha = 0.0, beta = 0.0, rs = 0.0, bnorm = 0.0;
  bool ok = true;  // no wait ran out
  // start (x0 = 0): r = b, p = r, x = 0, R published; (r, r) -> |b| and the
  // stopping test at the top of iteration 1
  double acc = 0.0;
  for (int j = 0; j < quads; j++) {
    const int li0 = j * kIrTile + kIrQ * t;
    if (li0 >= nr) continue;
    double v[kIrQ];
    const double z[kIrQ] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int e = 0; e < kIrQ; e++) {
      const int li = li0 + e;
      v[e] = li < nr ? __ldcg((const double *)a.rin + r0 + li) : 0.0;
      if (li < nr) acc = add_rn(acc, mul_rn(v[e], v[e]));
    }
    put(sr, li0, v);
    put(sp, li0, v);
    gput(R, li0, v);
    xput(li0, z);
  }
  double s1[1] = {acc};
  ok = ir_allreduce(a, ++gen, s1);
  if (ok) {
    const double rr = s1[0];
    bnorm = sqrt(rr);
    const double err = sqrt(rr) / bnorm;
    if (1 > maxloop)
      code = kMaxLoop;
    else if (err <= eps)
      code = kConverged;
    else if (err != err)
      code = kNaN;
    if (lead) {
      st->k.s[S_BNORM] = bnorm;
      check_top(st, 1, err);
    }
  }
  // q = A p (p = r) = s; rs = (r, s), alpha = rs / (q, q)   (CrStartMvEpi)
  if (ok && code == kRunning) {
    double s2[2] = {0.0, 0.0};
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      double rv[kIrQ], y[kIrQ] = {0.0, 0.0, 0.0, 0.0};
      if (li0 < nr) {
        own(sr, li0, rv);
        mv(li0, rv, y);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          if (li0 + e < nr) {
            s2[0] = add_rn(s2[0], mul_rn(rv[e], y[e]));
            s2[1] = add_rn(s2[1], mul_rn(y[e], y[e]));
          }
        }
      }
      TW::put(tq + TW::W * j, y);
      TW::put(ts + TW::W * j, y);
    }
    tm_wait_st();
    ok = ir_allreduce(a, ++gen, s2);
    if (ok) {
      rs = s2[0];
      if (s2[1] == 0.0) {
        code = kBreakdown;
      } else {
        alpha = div_rn(rs, s2[1]);
        if (!isfinite(alpha)) code = kNaN;
      }
      if (lead) {
        st->k.s[S_RR] = rs;
        st->k.s[S_ALPHA] = alpha;
        if (code != kRunning) set_done(st, code);
      }
    }
  }
  for (long long L = 1; ok && code == kRunning && L <= maxloop; L++) {
    // B: r -= alpha q, stored and published; (r, r) posted; x += alpha p
    acc = 0.0;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      double qv[kIrQ];
      TW::get(tq + TW::W * j, qv);
      if (li0 < nr) {
        double rv[kIrQ];
        own(sr, li0, rv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          rv[e] = add_rn(mul_rn(-alpha, qv[e]), rv[e]);
          if (li0 + e < nr) acc = add_rn(acc, mul_rn(rv[e], rv[e]));
        }
        put(sr, li0, rv);
        gput(R, li0, rv);
      }
    }
    s1[0] = acc;
    ir_red_post<1>(a, ++gen, s1);
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      if (li0 >= nr) continue;
      double pv[kIrQ], xv[kIrQ];
      own(sp, li0, pv);
      xget(li0, xv);
#pragma unroll
      for (int e = 0; e < kIrQ; e++) xv[e] = add_rn(mul_rn(alpha, pv[e]), xv[e]);
      xput(li0, xv);
    }
    if (!(ok = ir_red_wait<1>(a, gen, s1))) break;
    {
      const double err = sqrt(s1[0]) / bnorm;
      if (L + 1 > maxloop)
        code = kMaxLoop;
      else if (err <= eps)
        code = kConverged;
      else if (err != err)
        code = kNaN;
      if (lead) check_top(st, L + 1, err);
      if (code != kRunning) break;
    }
    // A: s = A r; (r, s) -> beta
    acc = 0.0;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      double y[kIrQ] = {0.0, 0.0, 0.0, 0.0};
      if (li0 < nr) {
        double rv[kIrQ];
        own(sr, li0, rv);
        mv(li0, rv, y);
#pragma unroll
        for (int e = 0; e < kIrQ; e++)
          if (li0 + e < nr) acc = add_rn(acc, mul_rn(rv[e], y[e]));
      }
      TW::put(ts + TW::W * j, y);
    }
    tm_wait_st();
    s1[0] = acc;
    if (!(ok = ir_allreduce(a, ++gen, s1))) break;
    if (rs == 0.0) {
      code = kBreakdown;
      beta = 0.0;
    } else {
      beta = div_rn(s1[0], rs);
      if (!isfinite(beta)) code = kNaN;
    }
    rs = s1[0];
    if (lead) {
      st->k.s[S_BETA] = beta;
      st->k.s[S_RR] = rs;
      if (code != kRunning) set_done(st, code);
    }
    if (code != kRunning) break;
    // C: p = beta p + r, q = beta q + s; (q, q) -> alpha
    acc = 0.0;
    for (int j = 0; j < quads; j++) {
      const int li0 = j * kIrTile + kIrQ * t;
      double qv[kIrQ], sv[kIrQ];
      TW::get2(tq + TW::W * j, qv, ts + TW::W * j, sv);
#pragma unroll
      for (int e = 0; e < kIrQ; e++) qv[e] = add_rn(mul_rn(beta, qv[e]), sv[e]);
      if (li0 < nr) {
        double pv[kIrQ], rv[kIrQ];
        own(sp, li0, pv);
        own(sr, li0, rv);
#pragma unroll
        for (int e = 0; e < kIrQ; e++) {
          pv[e] = add_rn(mul_rn(beta, pv[e]), rv[e]);
          if (li0 + e < nr) acc = add_rn(acc, mul_rn(qv[e], qv[e]));
        }
        put(sp, li0, pv);
      }
      TW::put(tq + TW::W * j, qv);
    }
    tm_wait_st();
    s1[0] = acc;
    if (!(ok = ir_allreduce(a, ++gen, s1))) break;
    if (s1[0] == 0.0) {
      code = kBreakdown;
      alpha = 0.0;
    } else {
      alpha = div_rn(rs, s1[0]);
      if (!isfinite(alpha)) code = kNaN;
    }
    if (lead) {
      st->k.s[S_ALPHA] = alpha;
      if (code != kRunning) set_done(st, code);
    }
  }
  if (ok && lead && code == kRunning) set_done(st, kMaxLoop);
  // every thread's TMEM accesses are complete (each waited on its own); the
  // columns go back on every path out of the loop
  tm_fence_before();
  __syncthreads();
  if (t < 32) {
    tm_fence_after();
    tm_dealloc(s_tmem, kIrTmemCols);
  }
}

// Lowers the L2 eviction priority of [p, p + bytes) back to normal (the
// lines stay cached), p 128-byte aligned: after the on-chip kernels' evict_last
// loads, so that the diagonal copy does not keep its place in L2 ahead of
// later work.
__global__ void k_l2_normal(const char *p, unsigned long long bytes) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x * 128ull;
  for (unsigned long long o = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) * 128ull; o < bytes;
       o += stride)
    asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(p + o) : "memory");
}

// The whole diagonal copy (every precision's values and the row masks).
inline void ir_l2_release(ks_ctx *ctx, const CsrDev &A) {
  const long long stored = A.dia_sym ? A.dia_nd / 2 + 1 : A.dia_nd;
  auto one = [&](const void *p, unsigned long long bytes) {
    if (!p || !bytes) return;
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)127;
    ctx->next_class = kMemset;  // cache maintenance, profiled with the memsets
    launch_k(ctx, k_l2_normal, dim3(ctx->num_sms * 2), dim3(256), 0, reinterpret_cast<const char *>(a0),
             bytes + (reinterpret_cast<uintptr_t>(p) - a0));
  };
  const unsigned long long e = (unsigned long long)(stored * A.dia_ds);
  one(A.dia_val, e * sizeof(double));
  one(A.dia_val32, e * sizeof(float));
  one(A.dia_val16, e * sizeof(__nv_bfloat16));
  one(A.dia_mask, (unsigned long long)A.n);
}

// Launch shape: one CTA per SM, rows per CTA a multiple of 32.
struct IrShape {
  int G = 0, rpc = 0, K = 0;
  size_t smem = 0;
};

// False when the system does not fit: r and q of a thread's rows in its 64
// TMEM words (K <= ir_max_k), p and x of a CTA's rows in shared memory.
// `fill`: fewer CTAs than SMs where the system is small, so that every
// thread has at least one quad of rows (fewer arrivals at each grid
// reduction; FP64 CG whole solves, same box, three rounds: 64^3 4.38 -> 3.79
// ms, 256^2 30.7 -> 28.8 ms, 512^2 74.8 -> 72.6 ms; CR, which streams x
// through global memory, got slower: 3.21 -> 4.26 ms).
template <class VT>
inline bool ir_shape(const ks_ctx *ctx, long long n, IrShape *s, bool fill = false) {
  if (n < 1) return false;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  const long long G = fill ? std::min<long long>(ctx->num_sms, std::max<long long>(1, (n + kIrQ * kIrThreads - 1) /
                                                                                         (kIrQ * kIrThreads)))
                           : ctx->num_sms;
  const long long rpc = ((n + G - 1) / G + 31) / 32 * 32;
  const long long K = (rpc + kIrThreads - 1) / kIrThreads;
  const size_t smem = sizeof(VT) * 2 * (size_t)rpc;
  if (K > ir_max_k<VT>() || G > kIrMaxGrid || smem + 2048 > (size_t)optin) return false;  // + the static arrays
  s->G = (int)G;
  s->rpc = (int)rpc;
  s->K = (int)K;
  s->smem = smem;
  return true;
}

// Cooperative launch of one CTA per SM; `probe`: only check that the grid
// can be co-resident (sets *fits). `cls`: its class in a profiled solve.
template <class VT, class MT, int NDG>
inline cudaError_t ir_launch_n(ks_ctx *ctx, const CsrDev &A, const IrArgs &a, const IrShape &sh, bool probe,
                               bool *fits, int cls) {
  auto fn = k_cg_onchip<VT, MT, NDG>;
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
  ctx->ir_used = true;  // its matrix lines are evict_last in L2 (ir_l2_release)
  ProfLaunch pl(ctx, cls);
  return cudaLaunchKernelEx(&cfg, fn, dview<MT>(A), a);
}

template <class VT, class MT>
inline cudaError_t ir_launch(ks_ctx *ctx, const CsrDev &A, const IrArgs &a, const IrShape &sh, bool probe,
                             bool *fits, int cls) {
  if (A.dia_nd == 7) return ir_launch_n<VT, MT, 7>(ctx, A, a, sh, probe, fits, cls);
  if (A.dia_nd == 5) return ir_launch_n<VT, MT, 5>(ctx, A, a, sh, probe, fits, cls);
  return ir_launch_n<VT, MT, 0>(ctx, A, a, sh, probe, fits, cls);
}

template <int NDG>
inline cudaError_t icr_launch_n(ks_ctx *ctx, const CsrDev &A, const IrArgs &a, const IrShape &sh, bool probe,
                                bool *fits) {
  auto fn = k_cr_onchip<NDG>;
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
  ctx->ir_used = true;  // its matrix lines are evict_last in L2 (ir_l2_release)
  ProfLaunch pl(ctx, kMv);  // a profiled solve counts the whole solve as one SpMV-class launch
  return cudaLaunchKernelEx(&cfg, fn, dview<double>(A), a);
}

}  // namespace ks
