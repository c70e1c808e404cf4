// Small systems solved inside one thread-block cluster.
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
//  * A reduction is a block sum, one cluster barrier, then the C block sums
//    read and added in a fixed order. Every thread of every CTA adds the same values in the
//    same order, so all compute the same alpha, beta and stopping decision and
//    leave the loop together; only rank 0's first thread writes the device
//    state (loop counter, history, done code).
//
// The per-element arithmetic (SpMV row sums in column order, the x, r and p
// updates) is the kernel-per-step engine's, operation for operation; only the
// order in which the dot products add their partial sums differs.
//
// Nothing here spins: a CTA waits only at the cluster's hardware barrier,
// which every CTA of the cluster reaches (they are co-scheduled by the launch
// and all take the same branch at every decision).
#pragma once

#include <cooperative_groups.h>

#include <algorithm>

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

// Sum over the cluster of one value per thread; every thread of every CTA
// returns the same total: the block sums are added by warp 0 of each CTA, and
// after the cluster barrier warp 0 of every CTA adds the same C block sums in
// the same butterfly and hands the total to its CTA through `tot`. (One warp
// per CTA reads the other CTAs' sums: a read by every warp would queue
// hundreds of distributed-shared-memory requests at each CTA's slot.) `red`
// alternates between two slots: another CTA may still be reading this call's
// slot when this CTA starts the next reduction, but not two reductions on (a
// cluster barrier lies between).
__device__ __forceinline__ double cluster_sum(cgx::cluster_group cl, double v, double *warp_s, double *red,
                                              double *tot, int C) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  v = group_sum<32>(v);
  if (lane == 0) warp_s[w] = v;
  __syncthreads();
  if (w == 0) {
    const double t = group_sum<32>(lane < nw ? warp_s[lane] : 0.0);
    if (lane == 0) *red = t;
  }
  cl.sync();
  if (w == 0) {
    const double u = group_sum<32>(lane < C ? *cl.map_shared_rank(red, (unsigned)lane) : 0.0);
    if (lane == 0) *tot = u;
  }
  __syncthreads();
  return *tot;
}

struct ResCgArgs {
  const int *ptr;
  const int *col;
  const short *col16;  // col - row, when the matrix keeps 16-bit offsets
  const double *val;
  const double *b;
  double *x;
  DevState *st;  // reset by InitOp before the launch
  int n;
  int shift;  // rows per CTA = 2^shift
};

// cg::solve (cg.cpp:148-240) from x = 0 to the stopping test, in one launch,
// with two cluster barriers per iteration. The CTAs publish r (not p): the
// SpMV of iteration L forms p_L = beta p_{L-1} + r_L for every column it
// gathers, from the owner's p_{L-1} and r_L, with the operations of the
// direction update (so the value equals the owner's p_L bit for bit), while
// each CTA writes its own p_L into the other of two p buffers. The reduction
// barrier after the x/r update then also publishes r_{L+1} and p_L, and the
// separate barrier after the direction update is not needed. x, r and p live
// in the CTA's shared memory (a thread reads and writes only its own rows of
// x); q, needed across the (p,q) reduction, in registers.
template <int R, bool I16>
__global__ void __launch_bounds__(kResThreads, 1) k_cg_resident(const ResCgArgs a) {
  cgx::cluster_group cl = cgx::this_cluster();
  extern __shared__ double dyn_s[];  // slices of x, r, p (two buffers)
  __shared__ double warp_s[32];
  __shared__ double red_s[2];
  __shared__ double tot_s;
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
  int red_i = 0;
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
  // |b|^2 and (r,r) are the same sum, r being b
  double rr = cluster_sum(cl, acc, warp_s, red_s + (red_i++ & 1), &tot_s, C);
  const double bnorm = sqrt(rr);
  if (S.writer) a.st->k.s[S_BNORM] = bnorm;
  S.check_top(1, sqrt(rr) / bnorm);
  double beta = 0.0;
  long long L = 1;
  while (S.done == kRunning) {
    const double *p_old = (L & 1) ? p_s0 : p_s1;  // p_{L-1}
    double *p_new = (L & 1) ? p_s1 : p_s0;        // p_L
    // p_L = beta p_{L-1} + r_L; q = A p_L; (p,q) -> alpha
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        const double pk = add_rn(mul_rn(beta, p_old[li]), r_s[li]);
        p_new[li] = pk;
        const int j0 = __ldg(a.ptr + i), j1 = __ldg(a.ptr + i + 1);
        double s = 0.0;
#pragma unroll 4
        for (int j = j0; j < j1; j++) {
          const int c = I16 ? i + (int)__ldg(a.col16 + j) : __ldg(a.col + j);
          const int o = c >> a.shift, lc = c & mask;
          const double *pp = p_old + lc, *rq = r_s + lc;
          if (o != rank) {  // another CTA's row: its shared memory, through the cluster
            pp = cl.map_shared_rank(pp, (unsigned)o);
            rq = cl.map_shared_rank(rq, (unsigned)o);
          }
          s = add_rn(s, mul_rn(__ldg(a.val + j), add_rn(mul_rn(beta, *pp), *rq)));
        }
        q[k] = s;
        acc = add_rn(acc, mul_rn(pk, s));
      }
    }
    const double pq = cluster_sum(cl, acc, warp_s, red_s + (red_i++ & 1), &tot_s, C);
    const double alpha = S.rdiv(rr, pq);
    if (S.done != kRunning) break;
    // x += alpha p; r -= alpha q (published); (r,r) -> beta; stopping test
    acc = 0.0;
#pragma unroll
    for (int k = 0; k < R; k++) {
      const int li = threadIdx.x + k * T, i = r0 + li;
      if (i < a.n) {
        x_s[li] = add_rn(mul_rn(alpha, p_new[li]), x_s[li]);
        const double rk = add_rn(mul_rn(-alpha, q[k]), r_s[li]);
        r_s[li] = rk;
        acc = add_rn(acc, mul_rn(rk, rk));
      }
    }
    const double rr2 = cluster_sum(cl, acc, warp_s, red_s + (red_i++ & 1), &tot_s, C);
    beta = S.rdiv(rr2, rr);
    rr = rr2;
    S.check_top(L + 1, sqrt(rr2) / bnorm);
    L++;
  }
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

template <int R, bool I16>
inline cudaError_t res_cg_launch(const ResShape &sh, cudaStream_t s, const ResCgArgs &a, bool probe_only,
                                 bool *fits) {
  auto kern = k_cg_resident<R, I16>;
  const size_t smem = (4 * sizeof(double)) << sh.shift;  // x, r and two p slices
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
