// Row-blocked CSR SpMV with TMA bulk staging (sm_100a).
//
// Each CTA walks its row blocks (CSR-Adaptive partition: <= kRowsPerBlock rows
// and <= kNnzPerBlock nonzeros per block; a longer row is a block of its own)
// through a two-stage shared-memory pipeline. One thread issues, per block,
// three 1-D bulk async copies (cp.async.bulk, completing on an mbarrier) of
// the block's column indices (int32, or int16 offsets from the row where the
// matrix allows them), values and row offsets, two blocks ahead of the
// compute, with an evict-first L2 policy so the Krylov vectors keep their
// place in L2. All threads then gather x and sum rows out of shared memory:
// one thread per row, in index order from 0.0 with separately rounded
// products and sums (exactly blas::MtxVec_mult, blas.cpp:56-62), or one warp
// per row when the block's rows average more than 16 nonzeros. Long rows are
// summed straight from global memory by the whole CTA.
//
// Every wait on an mbarrier is bounded by the global timer; a wait that runs
// out sets an error flag (reported as KS_TIMEOUT), waits once more, bounded,
// for the copies in flight and lets the CTA finish without further staging.
// No multicast form of the bulk copy is used.
#pragma once

#include <cstdint>

#include "ks_common.cuh"

namespace ks {

constexpr int kStages = 2;
constexpr int kStageElems = kNnzPerBlock + 16;  // values / columns per stage
constexpr int kStagePtr = kRowsPerBlock + 8;    // row offsets per stage
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

template <class MT, class IT>
struct StageBuf {
  MT val[kStageElems];
  IT col[kStageElems];
  int ptr[kStagePtr];
};

// Elements per 16 bytes of the narrower of the value and index arrays: a row
// block's copies start and end on multiples of this so both stay 16-byte aligned.
template <class MT, class IT>
constexpr int granule() {
  return 16 / (sizeof(MT) < sizeof(IT) ? sizeof(MT) : sizeof(IT));
}

// Column of a stored index: int32 indices are the column itself, int16 ones
// the offset of the column from the row.
template <class IT>
__device__ __forceinline__ int col_of(int row, IT v) {
  if constexpr (sizeof(IT) == 2)
    return row + (int)v;
  else
    return v;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false if the phase did not complete within `limit` ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          unsigned long long limit = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit) return false;
  }
  return true;
}

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
      "%4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <class MT, class IT>
struct CsrT {
  const int *__restrict__ ptr;   // n+1 offsets, padded to n+1+kPad
  const IT *__restrict__ col;    // nnz, padded (int: column; short: column - row)
  const MT *__restrict__ val;    // nnz, padded
  const int4 *__restrict__ rbi;  // per row block: r0, r1, j0, j1
  int nrb;
  int n;
};

// Issue the copies of row block `info` into stage buffer `sb`.
template <class MT, class IT>
__device__ __forceinline__ void stage_issue(const CsrT<MT, IT> &A, int4 info, StageBuf<MT, IT> *sb,
                                            uint64_t *bar, uint64_t pol) {
  constexpr int G = granule<MT, IT>();
  const int a0 = info.z & ~(G - 1);
  const int a1 = (info.w + G - 1) & ~(G - 1);
  const int p0 = info.x & ~3;
  const int p1 = (info.y + 1 + 3) & ~3;
  const uint32_t vb = (uint32_t)(a1 - a0) * sizeof(MT);
  const uint32_t cb = (uint32_t)(a1 - a0) * sizeof(IT);
  const uint32_t pb = (uint32_t)(p1 - p0) * sizeof(int);
  mbar_expect_tx(bar, vb + cb + pb);
  if (vb) bulk_g2s(sb->val, A.val + a0, vb, bar, pol);
  if (cb) bulk_g2s(sb->col, A.col + a0, cb, bar, pol);
  bulk_g2s(sb->ptr, A.ptr + p0, pb, bar, pol);
}

__device__ __forceinline__ bool is_long(int4 info) {
  return info.w - info.z > kNnzPerBlock;
}

// Gather of the right-hand vector (GX concept: prep() once per thread, then
// get<AT>(column)).
template <class XT>
struct GPtr {
  static constexpr bool kPlain = true;  // x read directly (the DIA kernel's quad path)
  const XT *__restrict__ x;
  __device__ __forceinline__ GPtr prep() const { return *this; }
  template <class AT>
  __device__ __forceinline__ AT get(int c) const {
    return (AT)__ldg(x + c);
  }
};

// NV right-hand vectors (1, or 2 for the k-skip matrix powers), gathered by
// GX. Epi::row(r, y) for NV = 1, Epi::row(r, y0, y1) for NV = 2 (with acc).
template <int NV, class MT, class IT, class GX, class Epi>
__global__ void __launch_bounds__(kThreads)
    spmv_tma_kernel(CsrT<MT, IT> A, GX gx0, GX gx1, Epi epi, Stop stop, Red red, int *err,
                    unsigned long long wait_ns) {
  using AT = typename Epi::acc_t;
  using SB = StageBuf<MT, IT>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SB *stage = reinterpret_cast<SB *>(smem_raw);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw + kStages * sizeof(SB));
  constexpr int ND = Epi::ND > 0 ? Epi::ND : 1;
  constexpr int G = granule<MT, IT>();
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) acc[d] = 0.0;
  const int tid = threadIdx.x;
  const uint64_t pol = l2_evict_first_policy();
  if (tid == 0) {
    for (int s = 0; s < kStages; s++) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // Producer state (thread 0): next block of this CTA to stage. The matrix
  // does not depend on the kernels before this one, so the first blocks are
  // staged before waiting for them (programmatic dependent launch).
  int prod_blk = blockIdx.x;
  int staged = 0;  // copies issued
  if (tid == 0) {
    while (staged < kStages && prod_blk < A.nrb) {
      const int4 info = A.rbi[prod_blk];
      if (!is_long(info)) {
        stage_issue(A, info, &stage[staged % kStages], &bars[staged % kStages], pol);
        staged++;
      }
      prod_blk += gridDim.x;
    }
  }
  pdl_wait();  // x, the stop flags and the scalars come from earlier kernels
  if (stop()) {
    if (tid == 0)  // let the copies already issued land before the CTA exits
      for (int c = 0; c < staged; c++) mbar_wait(&bars[c % kStages], (uint32_t)((c / kStages) & 1));
    __syncthreads();
    return;
  }
  const GX g0 = gx0.prep(), g1 = gx1.prep();
  int consumed = 0;
  bool failed = false;
  for (int blk = blockIdx.x; blk < A.nrb && !failed; blk += gridDim.x) {
    const int4 info = A.rbi[blk];
    const int r0 = info.x, nrows = info.y - info.x, j0 = info.z, nnz = info.w - info.z;
    if (is_long(info)) {
      // whole CTA on one long row, straight from global memory
      double v[NV];
#pragma unroll
      for (int u = 0; u < NV; u++) {
        const GX &gu = u == 0 ? g0 : g1;
        AT s = (AT)0;
        for (int j = j0 + tid; j < info.w; j += kThreads)
          s += mval<AT>(A.val[j]) * gu.template get<AT>(col_of(r0, A.col[j]));
        v[u] = (double)s;
      }
      block_sum<NV>(v);
      if (tid == 0) {
        if constexpr (NV == 1)
          epi.row(r0, (AT)v[0], acc);
        else
          epi.row(r0, (AT)v[0], (AT)v[NV - 1], acc);
      }
      __syncthreads();
      continue;
    }
    const int s = consumed % kStages;
    const uint32_t parity = (uint32_t)((consumed / kStages) & 1);
    const bool ok = mbar_wait(&bars[s], parity, wait_ns);
    // One decision for the whole CTA: a thread whose wait ran out must not
    // leave the others behind at a barrier.
    if (__syncthreads_or(!ok)) {
      failed = true;
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    const SB *sb = &stage[s];
    const int a0 = j0 & ~(G - 1);
    const int p0 = r0 & ~3;
    if (nnz <= 16 * nrows) {
      if (tid < nrows) {
        const int row = r0 + tid;
        const int rs = sb->ptr[r0 - p0 + tid] - a0, re = sb->ptr[r0 - p0 + tid + 1] - a0;
        AT y0 = (AT)0, y1 = (AT)0;
#pragma unroll 4
        for (int e = rs; e < re; e++) {
          const AT a = mval<AT>(sb->val[e]);
          const int c = col_of(row, sb->col[e]);
          y0 = add_rn(y0, mul_rn(a, g0.template get<AT>(c)));
          if constexpr (NV == 2) y1 = add_rn(y1, mul_rn(a, g1.template get<AT>(c)));
        }
        if constexpr (NV == 1)
          epi.row(r0 + tid, y0, acc);
        else
          epi.row(r0 + tid, y0, y1, acc);
      }
    } else {
      const int lane = tid & 31, w = tid >> 5;
      for (int rr = w; rr < nrows; rr += kThreads / 32) {
        const int rs = sb->ptr[r0 - p0 + rr] - a0, re = sb->ptr[r0 - p0 + rr + 1] - a0;
        AT y0 = (AT)0, y1 = (AT)0;
        for (int e = rs + lane; e < re; e += 32) {
          const AT a = mval<AT>(sb->val[e]);
          const int c = col_of(r0 + rr, sb->col[e]);
          y0 += a * g0.template get<AT>(c);
          if constexpr (NV == 2) y1 += a * g1.template get<AT>(c);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          y0 += __shfl_xor_sync(0xffffffffu, y0, o);
          if constexpr (NV == 2) y1 += __shfl_xor_sync(0xffffffffu, y1, o);
        }
        if (lane == 0) {
          if constexpr (NV == 1)
            epi.row(r0 + rr, y0, acc);
          else
            epi.row(r0 + rr, y0, y1, acc);
        }
      }
    }
    consumed++;
    __syncthreads();  // every thread is done reading stage s
    if (tid == 0) {
      // refill stage s with the next staged block of this CTA
      while (prod_blk < A.nrb) {
        const int4 nx = A.rbi[prod_blk];
        prod_blk += gridDim.x;
        if (!is_long(nx)) {
          fence_proxy_async_smem();
          stage_issue(A, nx, &stage[staged % kStages], &bars[staged % kStages], pol);
          staged++;
          break;
        }
      }
    }
  }
  if (failed) {
    // copies still in flight: one more bounded wait on each (the default
    // limit, whatever limit ended the loop), then finish
    for (int c = consumed; c < staged; c++) mbar_wait(&bars[c % kStages], (uint32_t)((c / kStages) & 1));
  }
  __syncthreads();
  pdl_trigger();  // the next kernel may be scheduled as this one drains
  if constexpr (Epi::ND > 0) {
    if (grid_sum<ND>(acc, red.partials, red.counter) && tid == 0) epi.finish(acc);
  }
}

template <class MT, class IT>
constexpr size_t spmv_tma_smem() {
  return kStages * sizeof(StageBuf<MT, IT>) + kStages * sizeof(uint64_t) + 16;
}

}  // namespace ks
