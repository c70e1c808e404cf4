// Small systems solved inside one thread-block cluster (CG, CR, BiCG).
//
// Up to 32K rows the kernels of a CG iteration (cg.cpp:184-240) each take a
// few microseconds and the loop is bound by its kernel boundaries (launch,
// drain, the grid reduction's last-CTA step), not by memory. Here the whole
// solve is one launch of one cluster of C <= 16 CTAs:
//
//  * CTA c owns rows [c * 2^shift, (c + 1) * 2^shift) and keeps its slices
//    of x, r and p in shared memory. The SpMV gathers r and p from the owning
//    CTA's shared memory, through distributed shared memory for another CTA's
//    rows. The matrix stays in global memory; its slice is read through L1,
//    where it stays between iterations.
//  * A reduction is a block sum sent to every CTA of the cluster, then the C
//    block sums added in rank order. Every CTA adds the same values in the
//    same order, so all compute the same alpha, beta and stopping decision and
//    leave the loop together; only rank 0's first thread writes the device
//    state (loop counter, history, done code).
//
// The per-element arithmetic (SpMV row sums in column order, the x, r and p
// updates) is the kernel-per-step engine's, operation for operation; only the
// order in which the dot products add their partial sums differs.
//
// The CTAs are co-scheduled by the cluster launch and take the same branch at
// every decision. A CTA waits at the cluster's hardware barrier twice (after
// setting up, before leaving) and otherwise only on its own mbarrier for the
// other CTAs' block sums, a wait bounded in time: if it runs out the CTA sets
// the context's error flag and leaves the loop, and so do the others at
// their next wait.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>

#include "ks_spmv_tma.cuh"
#include "ks_state.cuh"

namespace ks {

namespace cgx = cooperative_groups;

constexpr int kResMaxCluster = 16;        // CTAs of the cluster (16 needs the non-portable size)
constexpr int kResThreads = 512;          // threads per CTA at most (up to 128 registers each)
constexpr int kResMaxRowsPerCta = 2048;   // 512 threads x 4 rows
constexpr int kResTargetRowsPerCta = 256; // preferred slice; larger systems use all 16 CTAs
constexpr long long kResMaxRows = (long long)kResMaxCluster * kResMaxRowsPerCta;

constexpr int kResHist = 256;  // history entries buffered in shared memory between flushes

// The method's scalar steps (check_top, rdiv of ks_state.cuh) evaluated by
// every thread on the same values. `writer` (one thread) keeps the device
// state's loop counter and history length in registers and the history
// entries in a shared-memory ring, and stores them at flushes and at the end:
// a cluster barrier (release) waits for its CTA's outstanding global stores,
// so global stores inside the loop would delay every CTA at every barrier.
struct ResScal {
  DevState *st;
  bool writer;
  double eps;
  long long maxloop;
  double *h_err;     // shared ring, kResHist entries (writer's CTA)
  long long *h_it;
  int done = kRunning;
  long long loop = 0;
  long long hlen = 0, hflushed = 0, hcap = 0;
  bool rec = false;
  __device__ void begin() {
    if (!writer) return;
    rec = st->k.aux[A_RECORD] != 0;
    hlen = hflushed = st->k.hlen;
    hcap = st->k.hcap;
  }
  __device__ void flush() {
    for (long long h = hflushed; h < hlen; h++) {
      if (h < hcap) {
        st->k.hist_err[h] = h_err[h % kResHist];
        st->k.hist_it[h] = h_it[h % kResHist];
      }
    }
    hflushed = hlen;
  }
  __device__ void end() {
    if (!writer) return;
    flush();
    st->k.hlen = hlen;
    st->k.loop = loop;
  }
  __device__ void stop(int code) {
    done = code;
    if (writer) set_done(st, code);
  }
  __device__ void check_top(long long L, double err) {
    loop = L;
    if (L > maxloop) {
      stop(kMaxLoop);
      return;
    }
    if (writer && rec) {
      if (hlen - hflushed == kResHist) flush();
      h_err[hlen % kResHist] = err;
      h_it[hlen % kResHist] = L;
      hlen++;
    }
    if (err <= eps)
      stop(kConverged);
    else if (err != err)
      stop(kNaN);
  }
  __device__ double rdiv(double a, double b) {
    if (b == 0.0) {
      stop(kBreakdown);
      return 0.0;
    }
    const double q = div_rn(a, b);
    if (!isfinite(q)) stop(kNaN);
    return q;
  }
};

// Butterfly sum over groups of W lanes (W a power of two <= 32): every lane
// of a group ends with the same sum, each step adding the same two operands
// in either order.
template <int W>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kResMaxSums = 2;  // values one cluster reduction carries

// Exchange area of one CTA for the cluster reductions: every CTA's block sums
// (two slots, used by alternate reductions), one mbarrier per slot, and the
// outcome of the wait for the CTA.
struct ResXchg {
  double red[2][kResMaxSums][kResMaxCluster];
  uint64_t bar[2];
  int ok;
  double tot[kResMaxSums];
};

__device__ __forceinline__ void xchg_init(cgx::cluster_group cl, ResXchg *xg) {
  if (threadIdx.x == 0) {
    mbar_init(&xg->bar[0], 1);
    mbar_init(&xg->bar[1], 1);
    mbar_fence_init();
  }
  cl.sync();  // every CTA's barriers are initialised before any CTA sends to them
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Sums number m (0, 1, 2, ...) over the cluster of NV values per thread.
// Warp 0 of each CTA adds its CTA's warp sums and stores the NV block sums
// into slot m % 2 of every CTA's exchange area with st.async, each store
// completing 8 bytes on that CTA's mbarrier of the slot (a release at cluster
// scope, so the CTA's earlier shared-memory writes, ordered before it by
// __syncthreads, are visible to the receiver once its wait returns). Every
// thread then runs `shadow` (work that needs neither the sums nor other CTAs'
// data) while the block sums travel; thread 0 expects 8 NV C bytes per use of
// the barrier and waits for them (bounded by kWaitLimitNs) and adds the C
// block sums of each value in rank order, the same on every CTA. warp_s holds
// NV x 32 doubles. Returns false in every thread of the CTA if the wait ran
// out.
//
// Slot reuse: a CTA sends sums m + 2 only after completing sums m + 1, which
// need every CTA's block sums m + 1, which each CTA computes only after it
// has read sums m; so sums m + 2 never land on a slot or barrier phase still
// in use. (A block sum may land before the receiver's own expect for that
// phase; the transaction count then runs negative until it does.)
template <int NV, class F>
__device__ __forceinline__ bool cluster_sums(double (&v)[NV], double *warp_s, ResXchg *xg, int m, int C, int rank,
                                             F &&shadow) {
  static_assert(NV >= 1 && NV <= kResMaxSums, "values per cluster reduction");
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  const int s = m & 1;
  const uint32_t parity = (uint32_t)((m >> 1) & 1);
#pragma unroll
  for (int k = 0; k < NV; k++) {
    v[k] = group_sum<32>(v[k]);
    if (lane == 0) warp_s[k * 32 + w] = v[k];
  }
  __syncthreads();
  if (w == 0) {
    // every group of 8 or 16 lanes adds the same warp sums, so every lane that
    // sends holds the same block sums
    double t[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
      if (nw > 16) {
        t[k] = group_sum<32>(warp_s[k * 32 + lane]);
      } else if (nw > 8) {
        const int g = lane & 15;
        t[k] = group_sum<16>(g < nw ? warp_s[k * 32 + g] : 0.0);
      } else {
        const int g = lane & 7;
        t[k] = group_sum<8>(g < nw ? warp_s[k * 32 + g] : 0.0);
      }
    }
    if (lane == 0) mbar_expect_tx(&xg->bar[s], 8u * (uint32_t)(NV * C));
    if (lane < C) {
      uint32_t rb;
      asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(smem_u32(&xg->bar[s])), "r"(lane));
#pragma unroll
      for (int k = 0; k < NV; k++) {
        uint32_t ra;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                     : "=r"(ra)
                     : "r"(smem_u32(&xg->red[s][k][rank])), "r"(lane));
        asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];" ::"r"(ra),
                     "l"(__double_as_longlong(t[k])), "r"(rb)
                     : "memory");
      }
    }
  }
  shadow();
  if (threadIdx.x == 0) {
    bool ok = mbar_try_wait_cluster(&xg->bar[s], parity);
    if (!ok) {
      const unsigned long long t0 = global_ns();
      while (!(ok = mbar_try_wait_cluster(&xg->bar[s], parity)))
        if (global_ns() - t0 > kWaitLimitNs) break;
    }
    xg->ok = ok ? 1 : 0;
    if (ok) {
#pragma unroll
      for (int k = 0; k < NV; k++) {
        double u = 0.0;
        for (int c = 0; c < C; c++) u += xg->red[s][k][c];  // rank order
        xg->tot[k] = u;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; k++) v[k] = xg->tot[k];
  return xg->ok != 0;
}

// One value: the sum in *out.
template <class F>
__device__ __forceinline__ bool cluster_sum(double v, double *warp_s, ResXchg *xg, int m, int C, int rank,
                                            double *out, F &&shadow) {
  double a[1] = {v};
  const bool ok = cluster_sums<1>(a, warp_s, xg, m, C, rank, shadow);
  *out = a[0];
  return ok;
}

__device__ __forceinline__ void no_shadow() {}

struct ResCgArgs {
  const int *ptr;
  const int *col;
  const short *col16;  // col - row, when the matrix keeps 16-bit offsets
  const double *val;
  const double *b;
  double *x;
  DevState *st;  // reset by InitOp before the launch
  int *err;      // set if a bounded wait ran out
  int n;
  int shift;  // rows per CTA = 2^shift
};

// cg::solve (cg.cpp:148-240) from x = 0 to the stopping test, in one launch,
// with two cluster reductions per iteration and no other synchronisation
// between CTAs. The CTAs publish r (not p): the SpMV of iteration L forms
// p_L = beta p_{L-1} + r_L for every column it gathers, from the owner's
// p_{L-1} and r_L, with the operations of the direction update (so the value
// equals the owner's p_L bit for bit), while each CTA writes its own p_L into
// the other of two p buffers. The reduction after the x/r update then also
// publishes r_{L+1} and p_L. x, r and p live in the CTA's shared memory (a
// thread reads and writes only its own rows of x); q, needed across the (p,q)
// reduction, in registers. With one row per thread the values the next SpMV
// gathers (up to kResPre per row) are loaded right after that reduction, so
// their latency overlaps the beta division and the stopping test.
constexpr int kResPre = 7;

template <int R, bool I16>
__global__ void __launch_bounds__(kResThreads, 1) k_cg_resident(const ResCgArgs a) {
  cgx::cluster_group cl = cgx::this_cluster();
  extern __shared__ double dyn_s[];  // slices of x, r, p (two buffers)
  __shared__ double warp_s[kResMaxSums * 32];
  __shared__ ResXchg xg;
  __shared__ double hist_e[kResHist];
  __shared__ long long hist_i[kResHist];
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int rp = 1 << a.shift, mask = rp - 1;
  double *x_s = dyn_s, *r_s = dyn_s + rp, *p_s0 = dyn_s + 2 * rp, *p_s1 = dyn_s + 3 * rp;
  const int T = blockDim.x;
  const int r0 = rank << a.shift;
  ResScal S{a.st, rank == 0 && threadIdx.x == 0, a.st->k.s[S_EPS], a.st->k.aux[A_MAXLOOP], hist_e, hist_i};
  S.begin();
  xchg_init(cl, &xg);
  int m = 0;  // reductions so far
  bool ok = true;
  double q[R];
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    double ri = 0.0;
    if (i < a.n) {
      ri = sub_rn(a.b[i], 0.0);  // b - A*0 with x = 0 (cg.cpp:79)
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    x_s[li] = 0.0;
    r_s[li] = ri;
    p_s0[li] = ri;  // p_0 := r_1 with beta_0 = 0 gives p_1 = 0*r_1 + r_1 = r_1 (r finite here)
    q[k] = 0.0;
  }
  // the gather of one row (R == 1): its first kResPre columns' p_{L-1}, r_L
  // and matrix values; the rest of a longer row is read in the SpMV itself
  const int i1 = r0 + (int)threadIdx.x;
  const bool row1 = R == 1 && i1 < a.n;
  int j0 = 0, j1 = 0;
  if (row1) {
    j0 = __ldg(a.ptr + i1);
    j1 = __ldg(a.ptr + i1 + 1);
  }
  double pv[kResPre], rv[kResPre], av[kResPre];
  auto gather = [&](const double *p_old) {
#pragma unroll
    for (int t = 0; t < kResPre; t++) {
      if (row1 && t < j1 - j0) {
        const int j = j0 + t;
        const int c = I16 ? i1 + (int)__ldg(a.col16 + j) : __ldg(a.col + j);
        const int o = c >> a.shift, lc = c & mask;
        const double *pp = p_old + lc, *rq = r_s + lc;
        if (o != rank) {  // another CTA's row: its shared memory, through the cluster
          pp = cl.map_shared_rank(pp, (unsigned)o);
          rq = cl.map_shared_rank(rq, (unsigned)o);
        }
        pv[t] = *pp;
        rv[t] = *rq;
        av[t] = __ldg(a.val + j);
      }
    }
  };
  // |b|^2 and (r,r) are the same sum, r being b
  double rr = 0.0;
  ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rr, no_shadow);
  if (R == 1) gather(p_s0);
  const double bnorm = sqrt(rr);
  if (S.writer) a.st->k.s[S_BNORM] = bnorm;
  // The stopping test of iteration L (on (r_L, r_L)) runs in the shadow of
  // the next (p,q) reduction: the SpMV of iteration L runs before the test
  // and is discarded if the test stops the method (it changes only p_new and
  // q, which are then unused). The verdicts and the history are the
  // kernel-per-step engine's.
  double rr_chk = rr;
  long long L = 1;
  double beta = 0.0, alpha = 0.0;
  while (ok) {
    const double *p_old = (L & 1) ? p_s0 : p_s1;  // p_{L-1}
    double *p_new = (L & 1) ? p_s1 : p_s0;        // p_L
    // p_L = beta p_{L-1} + r_L; q = A p_L; (p,q) -> alpha
    acc = 0.0;
    if (R == 1) {
      if (row1) {
        const int li = (int)threadIdx.x;
        const double pk = add_rn(mul_rn(beta, p_old[li]), r_s[li]);
        p_new[li] = pk;
        double sum = 0.0;
#pragma unroll
        for (int t = 0; t < kResPre; t++)
          if (t < j1 - j0) sum = add_rn(sum, mul_rn(av[t], add_rn(mul_rn(beta, pv[t]), rv[t])));
        for (int j = j0 + kResPre; j < j1; j++) {
          const int c = I16 ? i1 + (int)__ldg(a.col16 + j) : __ldg(a.col + j);
          const int o = c >> a.shift, lc = c & mask;
          const double *pp = p_old + lc, *rq = r_s + lc;
          if (o != rank) {
            pp = cl.map_shared_rank(pp, (unsigned)o);
            rq = cl.map_shared_rank(rq, (unsigned)o);
          }
          sum = add_rn(sum, mul_rn(__ldg(a.val + j), add_rn(mul_rn(beta, *pp), *rq)));
        }
        q[0] = sum;
        acc = add_rn(0.0, mul_rn(pk, sum));
      }
    } else {
#pragma unroll
      for (int k = 0; k < R; k++) {
        const int li = threadIdx.x + k * T, i = r0 + li;
        if (i < a.n) {
          const double pk = add_rn(mul_rn(beta, p_old[li]), r_s[li]);
          p_new[li] = pk;
          const int jb = __ldg(a.ptr + i), je = __ldg(a.ptr + i + 1);
          double sum = 0.0;
#pragma unroll 4
          for (int j = jb; j < je; j++) {
            const int c = I16 ? i + (int)__ldg(a.col16 + j) : __ldg(a.col + j);
            const int o = c >> a.shift, lc = c & mask;
            const double *pp = p_old + lc, *rq = r_s + lc;
            if (o != rank) {
              pp = cl.map_shared_rank(pp, (unsigned)o);
              rq = cl.map_shared_rank(rq, (unsigned)o);
            }
            sum = add_rn(sum, mul_rn(__ldg(a.val + j), add_rn(mul_rn(beta, *pp), *rq)));
          }
          q[k] = sum;
          acc = add_rn(acc, mul_rn(pk, sum));
        }
      }
    }
    double pq = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &pq,
                           [&] { S.check_top(L, sqrt(rr_chk) / bnorm); })))
      break;
    if (S.done != kRunning) break;  // iteration L does not run
    alpha = S.rdiv(rr, pq);
    if (S.done != kRunning) break;
    // r -= alpha q (published); (r,r) -> beta; x += alpha p in the shadow
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        const double rk = add_rn(mul_rn(-alpha, q[k]), r_s[li]);
        r_s[li] = rk;
        acc = add_rn(acc, mul_rn(rk, rk));
      }
    }
    double rr2 = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rr2, [&] {
#pragma unroll
          for (int k = 0; k < R; k++) {
            const int li = threadIdx.x + k * T, i = r0 + li;
            if (i < a.n) x_s[li] = add_rn(mul_rn(alpha, p_new[li]), x_s[li]);
          }
        })))
      break;
    if (R == 1) gather(p_new);  // for iteration L + 1, whose p_L is p_new
    beta = S.rdiv(rr2, rr);
    rr = rr2;
    rr_chk = rr2;
    L++;
    if (S.done != kRunning) {  // beta's division stopped the method: the test still runs
      S.check_top(L, sqrt(rr_chk) / bnorm);
      break;
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    if (i < a.n) a.x[i] = x_s[li];
  }
  S.end();
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

struct ResBicgArgs {
  const int *ptr, *col;  // A
  const short *col16;
  const double *val;
  const int *tptr, *tcol;  // A^T
  const short *tcol16;
  const double *tval;
  const double *b;
  double *x;
  DevState *st;  // reset by InitOp before the launch
  int *err;      // set if a bounded wait ran out
  int n;
  int shift;  // rows per CTA = 2^shift
};

// Row i of M times the direction formed on the fly, beta d_old + v, from the
// owners' slices (this CTA's shared memory, or another CTA's through the
// cluster); the direction update's operations, the row's CSR order.
template <bool I16>
__device__ __forceinline__ double row_times_dir(cgx::cluster_group cl, const int *ptr, const int *col,
                                                const short *col16, const double *val, int i, int shift,
                                                int rank, double beta, const double *d_old, const double *v_s) {
  const int mask = (1 << shift) - 1;
  const int j0 = __ldg(ptr + i), j1 = __ldg(ptr + i + 1);
  double s = 0.0;
#pragma unroll 4
  for (int j = j0; j < j1; j++) {
    const int c = I16 ? i + (int)__ldg(col16 + j) : __ldg(col + j);
    const int o = c >> shift, lc = c & mask;
    const double *pp = d_old + lc, *vq = v_s + lc;
    if (o != rank) {
      pp = cl.map_shared_rank(pp, (unsigned)o);
      vq = cl.map_shared_rank(vq, (unsigned)o);
    }
    s = add_rn(s, mul_rn(__ldg(val + j), add_rn(mul_rn(beta, *pp), *vq)));
  }
  return s;
}

// bicg::solve (bicg.cpp:162-277) from x = 0 to the stopping test, in one
// launch (as k_cg_resident; x, r, r* and two buffers each of p and p* in
// shared memory). Per iteration both SpMVs, q = A p and t = A^T p*, form
// their directions in their reads from the published r and r*; then two
// cluster reductions: (p*, q) -> alpha, with the stopping test of the
// previous iteration in its shadow, and ((r,r), (r*,r)) after r -= alpha q,
// r* -= alpha t, with x += alpha p in its shadow. The decisions come in the
// kernel-per-step engine's order: the stopping test on (r,r), then beta =
// (r*,r)/(r*,r)_old; when beta's division stops the method the test still
// runs and its verdict wins, as there.
template <int R, bool IA16, bool IT16>
__global__ void __launch_bounds__(kResThreads, 1) k_bicg_resident(const ResBicgArgs a) {
  cgx::cluster_group cl = cgx::this_cluster();
  extern __shared__ double dyn_s[];  // slices of x, r, r*, p (two), p* (two)
  __shared__ double warp_s[kResMaxSums * 32];
  __shared__ ResXchg xg;
  __shared__ double hist_e[kResHist];
  __shared__ long long hist_i[kResHist];
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int rp = 1 << a.shift;
  double *x_s = dyn_s, *r_s = dyn_s + rp, *rs_s = dyn_s + 2 * rp;
  double *p_s0 = dyn_s + 3 * rp, *p_s1 = dyn_s + 4 * rp, *ps_s0 = dyn_s + 5 * rp, *ps_s1 = dyn_s + 6 * rp;
  const int T = blockDim.x;
  const int r0 = rank << a.shift;
  ResScal S{a.st, rank == 0 && threadIdx.x == 0, a.st->k.s[S_EPS], a.st->k.aux[A_MAXLOOP], hist_e, hist_i};
  S.begin();
  xchg_init(cl, &xg);
  int m = 0;
  bool ok = true;
  double q[R], t[R];
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    double ri = 0.0;
    if (i < a.n) {
      ri = sub_rn(a.b[i], 0.0);  // b - A*0 with x = 0; r* = r (bicg.cpp:181-183)
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    x_s[li] = 0.0;
    r_s[li] = ri;
    rs_s[li] = ri;
    p_s0[li] = ri;  // p_0 := r_1, p*_0 := r*_1 with beta_0 = 0: p_1 = r_1, p*_1 = r*_1
    ps_s0[li] = ri;
    q[k] = t[k] = 0.0;
  }
  // |b|^2, (r,r) and (r*,r) are the same sum, r* and r being b
  double rr = 0.0;
  ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rr, no_shadow);
  const double bnorm = sqrt(rr);
  if (S.writer) a.st->k.s[S_BNORM] = bnorm;
  double rr_chk = rr;  // (r,r) of the pending stopping test
  long long L = 1;
  double beta = 0.0, alpha = 0.0;
  while (ok) {
    const double *p_old = (L & 1) ? p_s0 : p_s1, *ps_old = (L & 1) ? ps_s0 : ps_s1;
    double *p_new = (L & 1) ? p_s1 : p_s0, *ps_new = (L & 1) ? ps_s1 : ps_s0;
    // p = beta p + r, p* = beta p* + r*; q = A p, t = A^T p*; (p*, q) -> alpha
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        p_new[li] = add_rn(mul_rn(beta, p_old[li]), r_s[li]);
        const double psk = add_rn(mul_rn(beta, ps_old[li]), rs_s[li]);
        ps_new[li] = psk;
        q[k] = row_times_dir<IA16>(cl, a.ptr, a.col, a.col16, a.val, i, a.shift, rank, beta, p_old, r_s);
        t[k] = row_times_dir<IT16>(cl, a.tptr, a.tcol, a.tcol16, a.tval, i, a.shift, rank, beta, ps_old, rs_s);
        acc = add_rn(acc, mul_rn(psk, q[k]));
      }
    }
    double pq = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &pq,
                           [&] { S.check_top(L, sqrt(rr_chk) / bnorm); })))
      break;
    if (S.done != kRunning) break;  // iteration L does not run
    alpha = S.rdiv(rr, pq);
    if (S.done != kRunning) break;
    // r -= alpha q; r* -= alpha t (published); (r,r), (r*,r); x += alpha p in the shadow
    double sums[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        const double rk = add_rn(mul_rn(-alpha, q[k]), r_s[li]);
        const double rsk = add_rn(mul_rn(-alpha, t[k]), rs_s[li]);
        r_s[li] = rk;
        rs_s[li] = rsk;
        sums[0] = add_rn(sums[0], mul_rn(rk, rk));
        sums[1] = add_rn(sums[1], mul_rn(rsk, rk));
      }
    }
    if (!(ok = cluster_sums<2>(sums, warp_s, &xg, m++, C, rank, [&] {
#pragma unroll
          for (int k = 0; k < R; k++) {
            const int li = threadIdx.x + k * T, i = r0 + li;
            if (i < a.n) x_s[li] = add_rn(mul_rn(alpha, p_new[li]), x_s[li]);
          }
        })))
      break;
    rr_chk = sums[0];
    L++;
    // the stopping test on (r,r) runs first in the engine; it is deferred to
    // the next reduction's shadow here, so beta's division comes first, and
    // when that stops the method the test runs at once (its verdict wins)
    beta = S.rdiv(sums[1], rr);
    rr = sums[1];
    if (S.done != kRunning) {
      S.check_top(L, sqrt(rr_chk) / bnorm);
      break;
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    if (i < a.n) a.x[i] = x_s[li];
  }
  S.end();
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Row i of M times the vector v, read from the owners' slices (this CTA's
// shared memory, or another CTA's through the cluster), in the row's CSR order.
template <bool I16>
__device__ __forceinline__ double row_times(cgx::cluster_group cl, const int *ptr, const int *col,
                                            const short *col16, const double *val, int i, int shift, int rank,
                                            const double *v_s) {
  const int mask = (1 << shift) - 1;
  const int j0 = __ldg(ptr + i), j1 = __ldg(ptr + i + 1);
  double s = 0.0;
#pragma unroll 4
  for (int j = j0; j < j1; j++) {
    const int c = I16 ? i + (int)__ldg(col16 + j) : __ldg(col + j);
    const int o = c >> shift, lc = c & mask;
    const double *vq = v_s + lc;
    if (o != rank) vq = cl.map_shared_rank(vq, (unsigned)o);
    s = add_rn(s, mul_rn(__ldg(val + j), *vq));
  }
  return s;
}

// cr::solve (cr.cpp:152-263) from x = 0 to the stopping test, in one launch
// (as k_cg_resident; x and r in shared memory, p, q = A p and s = A r of the
// thread's rows in registers). The SpMV reads r only, so r is the one vector
// the CTAs publish; an iteration has three cluster reductions, in the
// engine's order: (r,r) after x += alpha p, r -= alpha q (the stopping test;
// it also publishes r), (r,s) after s = A r (beta), and (q,q) after p = beta
// p + r, q = beta q + s (alpha).
template <int R, bool I16>
__global__ void __launch_bounds__(kResThreads, 1) k_cr_resident(const ResCgArgs a) {
  cgx::cluster_group cl = cgx::this_cluster();
  extern __shared__ double dyn_s[];  // slices of x and r
  __shared__ double warp_s[kResMaxSums * 32];
  __shared__ ResXchg xg;
  __shared__ double hist_e[kResHist];
  __shared__ long long hist_i[kResHist];
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int rp = 1 << a.shift;
  double *x_s = dyn_s, *r_s = dyn_s + rp;
  const int T = blockDim.x;
  const int r0 = rank << a.shift;
  ResScal S{a.st, rank == 0 && threadIdx.x == 0, a.st->k.s[S_EPS], a.st->k.aux[A_MAXLOOP], hist_e, hist_i};
  S.begin();
  xchg_init(cl, &xg);
  int m = 0;
  bool ok = true;
  double p[R], q[R], sv[R];
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    double ri = 0.0;
    if (i < a.n) {
      ri = sub_rn(a.b[i], 0.0);  // b - A*0 with x = 0; p = r (cr.cpp:79-86)
      acc = add_rn(acc, mul_rn(ri, ri));
    }
    x_s[li] = 0.0;
    r_s[li] = ri;
    p[k] = ri;
    q[k] = sv[k] = 0.0;
  }
  // |b|^2 and (r,r) are the same sum, r being b; the reduction also publishes r
  double rr = 0.0;
  ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rr, no_shadow);
  const double bnorm = sqrt(rr);
  if (S.writer) a.st->k.s[S_BNORM] = bnorm;
  if (ok) S.check_top(1, sqrt(rr) / bnorm);
  double rs = 0.0, alpha = 0.0, beta = 0.0;
  if (ok && S.done == kRunning) {
    // q = A p (p = r), s = q; (r,s) and (q,q) -> rs, alpha
    double sums[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int i = r0 + threadIdx.x + k * T;
      if (i < a.n) {
        const double v = row_times<I16>(cl, a.ptr, a.col, a.col16, a.val, i, a.shift, rank, r_s);
        q[k] = v;
        sv[k] = v;
        sums[0] = add_rn(sums[0], mul_rn(p[k], v));
        sums[1] = add_rn(sums[1], mul_rn(v, v));
      }
    }
    ok = cluster_sums<2>(sums, warp_s, &xg, m++, C, rank, no_shadow);
    if (ok) {
      rs = sums[0];
      alpha = S.rdiv(sums[0], sums[1]);
    }
  }
  long long L = 1;
  while (ok && S.done == kRunning) {
    // x += alpha p; r -= alpha q (published); (r,r) -> stopping test
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        x_s[li] = add_rn(mul_rn(alpha, p[k]), x_s[li]);
        const double rk = add_rn(mul_rn(-alpha, q[k]), r_s[li]);
        r_s[li] = rk;
        acc = add_rn(acc, mul_rn(rk, rk));
      }
    }
    double rr2 = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rr2, no_shadow))) break;
    S.check_top(L + 1, sqrt(rr2) / bnorm);
    L++;
    if (S.done != kRunning) break;
    // s = A r; (r,s) -> beta
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        sv[k] = row_times<I16>(cl, a.ptr, a.col, a.col16, a.val, i, a.shift, rank, r_s);
        acc = add_rn(acc, mul_rn(r_s[li], sv[k]));
      }
    }
    double rs2 = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &rs2, no_shadow))) break;
    beta = S.rdiv(rs2, rs);
    rs = rs2;
    if (S.done != kRunning) break;
    // p = beta p + r; q = beta q + s; (q,q) -> alpha
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        p[k] = add_rn(mul_rn(beta, p[k]), r_s[li]);
        q[k] = add_rn(mul_rn(beta, q[k]), sv[k]);
        acc = add_rn(acc, mul_rn(q[k], q[k]));
      }
    }
    double qq = 0.0;
    if (!(ok = cluster_sum(acc, warp_s, &xg, m++, C, rank, &qq, no_shadow))) break;
    alpha = S.rdiv(rs, qq);
  }
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
#pragma unroll
  for (int k = 0; k < R; k++) {
    const int li = threadIdx.x + k * T, i = r0 + li;
    if (i < a.n) a.x[i] = x_s[li];
  }
  S.end();
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------- host side
struct ResShape {
  int C = 0;      // CTAs (0: the system is too large)
  int T = 0;      // threads per CTA
  int R = 0;      // rows per thread
  int shift = 0;  // rows per CTA = 2^shift = T * R
};

// Rows per CTA: a power of two of at least kResTargetRowsPerCta, more when
// 16 CTAs need more, at most kResMaxRowsPerCta. (CG on the 64 x 64 Poisson
// matrix, 202 iterations on B200: 16 CTAs of 256 rows 0.71 ms, 8 of 512 rows
// 0.74 ms, 4 of 1024 rows 0.98 ms. Above 32K rows the kernel-per-step engine
// is as fast: 256 x 256 Poisson 9.4 ms against 9.6 ms, 40^3 2.7 against 2.4.)
inline ResShape resident_shape(long long n) {
  ResShape sh;
  if (n < 1 || n > kResMaxRows) return sh;
  const long long need = std::max<long long>(
      {32, (n + kResMaxCluster - 1) / kResMaxCluster, std::min<long long>(kResTargetRowsPerCta, n)});
  int shift = 5;
  while ((1LL << shift) < need) shift++;
  const int rp = 1 << shift;
  sh.C = (int)((n + rp - 1) / rp);
  sh.T = std::min(rp, kResThreads);
  sh.R = rp / sh.T;
  sh.shift = shift;
  return sh;
}

// Launches `kern` over one cluster of shape sh with `smem` bytes of dynamic
// shared memory; probe_only: sets *fits to whether one such cluster can be
// resident on the device and launches nothing.
template <class Args>
inline cudaError_t res_launch(void (*kern)(Args), const ResShape &sh, size_t smem, cudaStream_t s,
                              const Args &a, bool probe_only, bool *fits) {
  if (sh.C > 8) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)sh.C);
  cfg.blockDim = dim3((unsigned)sh.T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)sh.C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (probe_only) {
    int clusters = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg);
    *fits = e == cudaSuccess && clusters >= 1;
    if (e != cudaSuccess) (void)cudaGetLastError();
    return cudaSuccess;
  }
  return cudaLaunchKernelEx(&cfg, kern, a);
}

template <int R, bool I16>
inline cudaError_t res_cg_launch(const ResShape &sh, cudaStream_t s, const ResCgArgs &a, bool probe_only,
                                 bool *fits) {
  // x, r and two p slices
  return res_launch(k_cg_resident<R, I16>, sh, (4 * sizeof(double)) << sh.shift, s, a, probe_only, fits);
}

template <int R, bool I16>
inline cudaError_t res_cr_launch(const ResShape &sh, cudaStream_t s, const ResCgArgs &a, bool probe_only,
                                 bool *fits) {
  // x and r slices
  return res_launch(k_cr_resident<R, I16>, sh, (2 * sizeof(double)) << sh.shift, s, a, probe_only, fits);
}

// As res_cg, for CR.
inline cudaError_t res_cr(const ResShape &sh, bool i16, cudaStream_t s, const ResCgArgs &a, bool probe_only,
                          bool *fits) {
  switch (sh.R * 2 + (i16 ? 1 : 0)) {
    case 2: return res_cr_launch<1, false>(sh, s, a, probe_only, fits);
    case 3: return res_cr_launch<1, true>(sh, s, a, probe_only, fits);
    case 4: return res_cr_launch<2, false>(sh, s, a, probe_only, fits);
    case 5: return res_cr_launch<2, true>(sh, s, a, probe_only, fits);
    case 8: return res_cr_launch<4, false>(sh, s, a, probe_only, fits);
    case 9: return res_cr_launch<4, true>(sh, s, a, probe_only, fits);
  }
  return cudaErrorInvalidValue;
}

template <int R, bool IA16, bool IT16>
inline cudaError_t res_bicg_launch(const ResShape &sh, cudaStream_t s, const ResBicgArgs &a, bool probe_only,
                                   bool *fits) {
  // x, r, r*, two p and two p* slices
  return res_launch(k_bicg_resident<R, IA16, IT16>, sh, (7 * sizeof(double)) << sh.shift, s, a, probe_only, fits);
}

template <int R>
inline cudaError_t res_bicg_r(const ResShape &sh, bool ia16, bool it16, cudaStream_t s, const ResBicgArgs &a,
                              bool probe_only, bool *fits) {
  if (ia16)
    return it16 ? res_bicg_launch<R, true, true>(sh, s, a, probe_only, fits)
                : res_bicg_launch<R, true, false>(sh, s, a, probe_only, fits);
  return it16 ? res_bicg_launch<R, false, true>(sh, s, a, probe_only, fits)
              : res_bicg_launch<R, false, false>(sh, s, a, probe_only, fits);
}

// As res_cg, for BiCG (columns of A and of A^T as int16 offsets or int32).
inline cudaError_t res_bicg(const ResShape &sh, bool ia16, bool it16, cudaStream_t s, const ResBicgArgs &a,
                            bool probe_only, bool *fits) {
  switch (sh.R) {
    case 1: return res_bicg_r<1>(sh, ia16, it16, s, a, probe_only, fits);
    case 2: return res_bicg_r<2>(sh, ia16, it16, s, a, probe_only, fits);
    case 4: return res_bicg_r<4>(sh, ia16, it16, s, a, probe_only, fits);
  }
  return cudaErrorInvalidValue;
}

// probe_only: sets *fits to whether one cluster of this shape can be resident
// on the device (launches nothing). Otherwise launches the solve.
inline cudaError_t res_cg(const ResShape &sh, bool i16, cudaStream_t s, const ResCgArgs &a, bool probe_only,
                          bool *fits) {
  switch (sh.R * 2 + (i16 ? 1 : 0)) {
    case 2: return res_cg_launch<1, false>(sh, s, a, probe_only, fits);
    case 3: return res_cg_launch<1, true>(sh, s, a, probe_only, fits);
    case 4: return res_cg_launch<2, false>(sh, s, a, probe_only, fits);
    case 5: return res_cg_launch<2, true>(sh, s, a, probe_only, fits);
    case 8: return res_cg_launch<4, false>(sh, s, a, probe_only, fits);
    case 9: return res_cg_launch<4, true>(sh, s, a, probe_only, fits);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ks
