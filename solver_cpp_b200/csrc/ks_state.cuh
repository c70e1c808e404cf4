// Device-resident state of a running Krylov method: the named scalar slots,
// the stopping test and the residual history, shared by the kernel-per-step
// engine (ks_solvers.cu) and the cluster-resident small-system solves
// (ks_resident.cuh).
#pragma once

#include "ks_common.cuh"

namespace ks {

// ------------------------------------------------------------------ state
enum Slot : int {
  S_BNORM = 0,
  S_EPS = 1,
  S_RR = 2,     // (r,r) / (r*,r) / (r,z) / (r,s) / zaz: the carried product
  S_ALPHA = 3,
  S_BETA = 4,
  S_T = 5,      // GMRES: current norm
  S_GAMMA = 6,  // k-skip
  S_TRUECNT = 8,  // VP methods: FP64 true-residual checks made
  S_TRUERES = 9,  // the last one's |b - A x| / |b|
};
enum Aux : int { A_MAXLOOP = 0, A_RECORD = 1, A_SPMV = 2, A_CONVK = 3, A_FINAL = 4, A_KIDX = 5, A_PENDING = 6, A_XZERO = 7 };

struct DevState {  // KState plus the host-mapped mirror of `done`
  KState k;
  int *host_done;
};

__device__ __forceinline__ void set_done(DevState *st, int code) {
  st->k.done = code;
  if (st->host_done) *(volatile int *)st->host_done = code;
}

__device__ __forceinline__ void record(DevState *st, long long label, double err) {
  if (!st->k.aux[A_RECORD]) return;
  const long long h = st->k.hlen++;
  if (h < st->k.hcap) {
    st->k.hist_err[h] = err;
    st->k.hist_it[h] = label;
  }
}

// Stopping test at the top of iteration L of the CG-type loops
// (cg.cpp:184-198): loop ends after maxloop iterations, records, compares.
__device__ __forceinline__ void check_top(DevState *st, long long L, double err) {
  st->k.loop = L;
  if (L > st->k.aux[A_MAXLOOP]) {
    set_done(st, kMaxLoop);
    return;
  }
  record(st, L, err);
  if (err <= st->k.s[S_EPS])
    set_done(st, kConverged);
  else if (err != err)
    set_done(st, kNaN);
}

// a / b of a recurrence; a zero or non-finite result stops the method.
__device__ __forceinline__ double rdiv(DevState *st, double a, double b) {
  if (b == 0.0) {
    set_done(st, kBreakdown);
    return 0.0;
  }
  const double q = div_rn(a, b);
  if (!isfinite(q)) set_done(st, kNaN);
  return q;
}

__device__ __forceinline__ double rd(const double *p) { return __ldg(p); }

}  // namespace ks
