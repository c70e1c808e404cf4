// Krylov methods with every vector and every recurrence scalar on the device.
//
// Each method is the reference's loop (cg.cpp, cr.cpp, bicg.cpp, gcr.cpp,
// gmres.cpp, kskipcg.cpp, kskipbicg.cpp, vpcg.cpp, vpcr.cpp, vpgcr.cpp,
// vpgmres.cpp) re-cut into fused kernels. Reductions finish in the last CTA
// of their kernel, which also advances the scalar recurrence (alpha, beta,
// the stopping test and the residual history) in device memory. The host
// issues iterations without waiting and only polls a host-mapped `done`
// flag a bounded number of iterations behind; once a method has finished,
// queued kernels see `done` and return at once.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "ks_ops.cuh"
#include "ks_state.cuh"
#include "ks_resident.cuh"
#include "ks_inner_resident.cuh"

namespace ks {

ks_status spmv_any(ks_ctx *ctx, const CsrDev &A, ks_precision vals, ks_precision vt, const void *x,
                   void *y, Stop stop);
ks_status matpow(ks_ctx *ctx, const CsrDev &A, const double *r, const double *p, int k, double *Ar,
                 double *Ap, Stop stop);

// ------------------------------------------------------------------ env
struct Params {
  long long maxloop;
  double eps;
  long long restart;
  int kskip;
  int fix;
  int x_update = 0;       // ks_params.x_update
  int cluster_solve = 0;  // ks_params.cluster_solve
};

template <class VT>
struct Env {
  ks_ctx *ctx = nullptr;
  const CsrDev *A = nullptr;   // operator
  const CsrDev *AT = nullptr;  // its transpose
  ks_precision mvals = KS_FP64;
  DevState *st = nullptr;
  const int *outer_done = nullptr;
  bool record = false;
  bool outer = false;  // drives host polling
  Params sp{};
  bool faithful = false;
  long long n = 0;    // this rank's vector length
  long long ld = 0;   // workspace slot length (n, or the window of a split solve)
  long long off = 0;  // the vector's offset in its slot
  volatile int *hflag = nullptr;  // host view of st->host_done (outer only)
  int lookahead = 8;
  // row-split solve: the transport and the halo plans of A and AT
  ks_comm *comm = nullptr;
  const HaloPlan *planA = nullptr, *planT = nullptr;
  bool true_check = false;  // VP outer methods: FP64 true-residual check before converging
  Stop stop() const { return Stop{&st->k.done, outer_done}; }
  // Fill the halo of an SpMV input from the peers (it is written, though
  // the method treats the vector as read-only: the halo is not its data).
  void halo(const CsrDev &M, const VT *x) const {
    if (comm) note_dist(ctx, comm->exchange(&M == A ? *planA : *planT, (void *)x, sizeof(VT)));
  }
};

__global__ void k_snapshot(const int *done, int *out) { *out = *(volatile const int *)done; }

// Host-side bounded lookahead: after each issued iteration, wait for the one
// `la` iterations back and read the mapped done flag.
struct Poller {
  ks_ctx *ctx;
  volatile int *flag;
  int la;
  long long issued = 0;
  // Row-split solve: every rank must stop issuing after the same iteration,
  // or their collectives would no longer pair up. Every `la` iterations a
  // one-thread kernel copies `done` into a mapped ring; the host decides from
  // the copy one chunk back, which holds the same value on every rank.
  bool step_split() {
    issued++;
    if (issued % la) return false;
    const long long m = issued / la;
    const int R = ctx->nflags;
    ctx->launches++;
    k_snapshot<<<1, 1, 0, ctx->stream>>>(ctx->poll_done, ctx->d_snap + (m % R));
    cudaEventRecord(ctx->flag_events[m % R], ctx->stream);
    if (m < 2) return false;
    cudaEventSynchronize(ctx->flag_events[(m - 1) % R]);
    return ((volatile int *)ctx->h_snap)[(m - 1) % R] != 0;
  }
  bool step() {
    if (!flag) return false;
    if (ctx->red_comm) return step_split();
    const int R = ctx->nflags;
    cudaEventRecord(ctx->flag_events[issued % R], ctx->stream);
    issued++;
    if (*flag) return true;
    if (issued > la) {
      cudaEventSynchronize(ctx->flag_events[(issued - 1 - la) % R]);
      return *flag != 0;
    }
    return false;
  }
};

// SpMV with an epilogue, dispatched on the vector type and value copy.
template <class VT, class Epi>
inline void mv(const Env<VT> &E, const CsrDev &M, const VT *x, const Epi &epi) {
  E.halo(M, x);
  if constexpr (std::is_same<VT, double>::value) {
    launch_spmv<double, double>(E.ctx, M, x, epi, E.stop());
  } else {
    if (E.mvals == KS_BF16)
      launch_spmv<__nv_bfloat16, float>(E.ctx, M, x, epi, E.stop());
    else
      launch_spmv<float, float>(E.ctx, M, x, epi, E.stop());
  }
}

template <class VT, class Op>
inline void vec(const Env<VT> &E, const Op &op) {
  launch_vec(E.ctx, E.n, op, E.stop());
}

// ------------------------------------------------------------------ shared ops
// bnorm = |b|, stored with eps; resets the method's state.
struct InitOp {
  DevState *st;
  double eps;
  long long maxloop;
  int rec;
  __device__ void run() const {
    st->k.done = kRunning;
    st->k.loop = 0;
    st->k.hlen = 0;
    st->k.s[S_EPS] = eps;
    st->k.aux[A_MAXLOOP] = maxloop;
    st->k.aux[A_RECORD] = rec;
    st->k.aux[A_CONVK] = 0;
    st->k.aux[A_FINAL] = 0;
    st->k.aux[A_PENDING] = 0;
    st->k.aux[A_XZERO] = 1;  // x = 0 until the first deferred update lands
    st->k.s[S_BETA] = 0.0;  // first fused direction update: p = 0*r + r = r
    if (st->host_done) *(volatile int *)st->host_done = 0;
  }
};

template <class VT>
struct NormBOp {  // s[BNORM] = |b|
  const VT *b;
  DevState *st;
  static constexpr int ND = 1;
  struct Regs {
    VT b;
  };
  __device__ Regs load(long long i) const { return {b[i]}; }
  __device__ void store(long long, const Regs &g, double (&acc)[1]) const {
    const double v = widen(g.b);
    acc[0] = add_rn(acc[0], mul_rn(v, v));
  }
  __device__ void finish(const double (&s)[1]) const { st->k.s[S_BNORM] = sqrt(s[0]); }
};

template <class VT>
struct ZeroOp {
  VT *x;
  static constexpr int ND = 0;
  static constexpr bool kMemset = true;
  __device__ void elem(long long i, double (&)[1]) const { x[i] = (VT)0; }
  __device__ void finish(const double (&)[1]) const {}
};

template <class VT>
struct CopyOp {
  const VT *a;
  VT *b;
  static constexpr int ND = 0;
  struct Regs {
    VT a;
  };
  __device__ Regs load(long long i) const { return {a[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const { b[i] = g.a; }
  __device__ void finish(const double (&)[1]) const {}
};

// p = (beta * p) + r, beta from a slot (Scalar_axy(beta, p, r, p)).
template <class VT>
struct XpbyOp {
  VT *p;
  const VT *r;
  const double *beta;
  static constexpr int ND = 0;
  struct Regs {
    VT p, r;
  };
  __device__ Regs load(long long i) const { return {p[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const VT b = (VT)rd(beta);
    p[i] = add_rn(mul_rn(b, g.p), g.r);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// Two of them with one beta (p = beta p + r; q = beta q + s), optionally
// followed by (q,q) -> alpha = s[RR] / (q,q) (CR, VPCR).
template <class VT>
struct Xpby2Op {
  VT *p;
  const VT *r;
  VT *q;
  const VT *s;
  DevState *st;
  int alpha_from_qq;
  static constexpr int ND = 1;
  struct Regs {
    VT p, r, q, s;
  };
  __device__ Regs load(long long i) const { return {p[i], r[i], q[i], s[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT b = (VT)rd(&st->k.s[S_BETA]);
    p[i] = add_rn(mul_rn(b, g.p), g.r);
    const VT qi = add_rn(mul_rn(b, g.q), g.s);
    q[i] = qi;
    acc[0] = add_rn(acc[0], mul_rn(widen(qi), widen(qi)));
  }
  __device__ void finish(const double (&sm)[1]) const {
    if (alpha_from_qq) st->k.s[S_ALPHA] = rdiv(st, st->k.s[S_RR], sm[0]);
  }
};

// r = b - A x; out (r,r); optional copies c1 = r, c2 = r. Used by every
// method's start; `mode` picks the scalar step in finish().
enum StartMode : int {
  START_CG = 0,    // rr = (r,r); check_top(1)
  START_CHECK = 1, // check_top(1) only (VP methods: rr comes later)
  START_NORM = 2,  // s[T] = |r| (GMRES cycle start)
  START_GCR = 3,   // GCR cycle start: maxloop test, check(loop)
  START_KSKIP = 4, // nothing (k-skip checks at block start)
};

template <class VT>
struct StartEpi {
  using acc_t = VT;
  const VT *b;
  VT *r;
  VT *c1;
  VT *c2;
  VT *c3;
  DevState *st;
  int mode;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    const VT ri = sub_rn(b[i], v);
    r[i] = ri;
    if (c1) c1[i] = ri;
    if (c2) c2[i] = ri;
    if (c3) c3[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
  }
  __device__ void finish(const double (&s)[1]) const;
};

// GCR's stopping test at the top of step k (gcr.cpp:222-239).
__device__ __forceinline__ void check_gcr(DevState *st, double err) {
  const long long L = st->k.loop;
  record(st, L, err);
  if (err <= st->k.s[S_EPS]) {
    set_done(st, kConverged);
  } else if (L >= st->k.aux[A_MAXLOOP]) {
    set_done(st, kMaxLoop);
  } else if (err != err) {
    set_done(st, kNaN);
  } else {
    st->k.loop = L + 1;
  }
}

template <class VT>
__device__ void StartEpi<VT>::finish(const double (&s)[1]) const {
  const double err = sqrt(s[0]) / st->k.s[S_BNORM];
  switch (mode) {
    case START_CG:
      st->k.s[S_RR] = s[0];
      check_top(st, 1, err);
      break;
    case START_CHECK:
      check_top(st, 1, err);
      break;
    case START_NORM:
      st->k.s[S_T] = sqrt(s[0]);
      break;
    case START_GCR:
      if (st->k.loop >= st->k.aux[A_MAXLOOP])
        set_done(st, kMaxLoop);
      else
        check_gcr(st, err);
      break;
    default:
      break;
  }
}

// The start of a method whose x is zero (every method zeroes x first, as
// cg.cpp:79 does): A*0 is exactly 0, so r = b - A*0 is b bit for bit and the
// SpMV can be skipped; one vector pass does the copies, (r,r) and the same
// scalar step as StartEpi::finish.
template <class VT>
struct StartZeroOp {
  StartEpi<VT> e;
  static constexpr int ND = 1;
  struct Regs {
    VT b;
  };
  __device__ Regs load(long long i) const { return {e.b[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT ri = sub_rn(g.b, (VT)0);
    e.r[i] = ri;
    if (e.c1) e.c1[i] = ri;
    if (e.c2) e.c2[i] = ri;
    if (e.c3) e.c3[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
  }
  __device__ void finish(const double (&s)[1]) const { e.finish(s); }
};

template <class VT>
inline void start_from_zero(const Env<VT> &E, const StartEpi<VT> &epi) {
  vec(E, StartZeroOp<VT>{epi});
}

// ------------------------------------------------------------------ CG
// cg::solve (cg.cpp:148-240), three fused kernels per iteration:
//   q = A p, (p,q) -> alpha;  x += alpha p, r -= alpha q, (r,r) -> beta,
//   check;  p = beta p + r.
template <class VT>
struct CgMvEpi {
  using acc_t = VT;
  const VT *p;
  VT *q;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    q[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(p[i]), widen(v)));
  }
  __device__ void finish(const double (&s)[1]) const {
    st->k.s[S_ALPHA] = rdiv(st, st->k.s[S_RR], s[0]);
  }
};

// x += alpha p; r -= alpha q; (r,r). mode 0: CG (beta = rr2/rr, check);
// mode 1: check only (VP outer: rr carried separately).
template <class VT>
struct XrUpdOp {
  VT *x;
  VT *r;
  const VT *p;
  const VT *q;
  DevState *st;
  int mode;
  static constexpr int ND = 1;
  struct Regs {
    VT x, p, q, r;
  };
  __device__ Regs load(long long i) const { return {x[i], p[i], q[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT a = (VT)rd(&st->k.s[S_ALPHA]);
    x[i] = add_rn(mul_rn(a, g.p), g.x);
    const VT ri = add_rn(mul_rn((VT)(-a), g.q), g.r);
    r[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
  }
  __device__ void finish(const double (&s)[1]) const {
    const long long L = st->k.loop;
    if (mode == 0) {
      st->k.s[S_BETA] = rdiv(st, s[0], st->k.s[S_RR]);
      st->k.s[S_RR] = s[0];
    }
    check_top(st, L + 1, sqrt(s[0]) / st->k.s[S_BNORM]);
  }
};

// ------------------------------------------------------------------ deferred x
// CG, CR and BiCG update x only through x += alpha p (cg.cpp:211,
// cr.cpp:240, bicg.cpp:242), and nothing reads x inside their loops. So the
// update is deferred: iteration L keeps its direction in slot (L-1) % D of a
// ring of D vectors (the direction update writes the next slot instead of
// overwriting p), its r-update kernel records alpha beside it and counts the
// iteration as pending, and every D iterations (and once after the loop) one
// pass applies x += alpha_i p_i over the pending slots in iteration order.
// Each element of x sees the same products and sums in the same order, so x
// is bit-identical, while the r-update no longer reads and writes x and p:
// two fewer vector passes per iteration for one ring pass per D iterations.
// The ring pays where x, r and the direction vectors stream from HBM every
// iteration. When they fit in L2 (here: within 60 % of it) the per-iteration
// x += alpha p is served from L2 and costs less than streaming the ring back
// from HBM: measured on B200, the ring made CG 11 % faster at 160^3 in FP64
// (4 vectors of 32.8 MB) but 3 % slower at 128^3 in FP64 (16.8 MB vectors)
// and the FP32 inner solves at 160^3 (16.4 MB vectors) 8 % slower.
constexpr int kDirRing = 32;

inline int loop_vectors(int method) {  // x, r, p, A p (+ s for CR, + r*, p* for BiCG)
  return method == KS_CG ? 4 : method == KS_CR ? 5 : method == KS_BICG ? 6 : 0;
}

inline bool defer_x(int method, const Params &sp, long long n, size_t elem, size_t l2) {
  if (!loop_vectors(method) || sp.x_update == 1) return false;
  if (sp.x_update == 2) return true;
  return (double)loop_vectors(method) * (double)n * (double)elem > 0.6 * (double)l2;
}

inline int dir_ring(const Params &sp) {
  return (int)std::max<long long>(1, std::min<long long>(kDirRing, sp.maxloop));
}

// Direction slots a method allocates: the ring, or the single in-place p
// (two for CG and BiCG, whose SpMV may form the next direction from the
// previous one while writing it: run_cg, run_bicg; they use the second only
// then).
inline int dir_slots(int method, const Params &sp, long long n, size_t elem, size_t l2) {
  return defer_x(method, sp, n, elem, l2) ? dir_ring(sp) : (method == KS_CG || method == KS_BICG ? 2 : 1);
}

template <class VT>
inline bool defer_x(const Env<VT> &E, int method) {
  return defer_x(method, E.sp, E.n, sizeof(VT), E.ctx->l2_bytes);
}

template <class VT>
struct DirRing {
  VT *P;
  long long ld;  // slot stride
  int D;
  double *alpha;
  VT *slot(long long L) const { return P + ((L - 1) % D) * ld; }
  double *aslot(long long L) const { return alpha + (L - 1) % D; }
};

// r -= alpha q; (r,r); alpha saved to the ring and the iteration counted as
// pending for x. The scalar step is XrUpdOp's (mode 0: CG beta; 1: check).
template <class VT>
struct RUpdOp {
  VT *r;
  const VT *q;
  DevState *st;
  int mode;
  double *aslot;
  static constexpr int ND = 1;
  struct Regs {
    VT q, r;
  };
  __device__ Regs load(long long i) const { return {q[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT a = (VT)rd(&st->k.s[S_ALPHA]);
    const VT ri = add_rn(mul_rn((VT)(-a), g.q), g.r);
    r[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
  }
  __device__ void finish(const double (&s)[1]) const {
    *aslot = st->k.s[S_ALPHA];
    st->k.aux[A_PENDING]++;
    const long long L = st->k.loop;
    if (mode == 0) {
      st->k.s[S_BETA] = rdiv(st, s[0], st->k.s[S_RR]);
      st->k.s[S_RR] = s[0];
    }
    check_top(st, L + 1, sqrt(s[0]) / st->k.s[S_BNORM]);
  }
};

// x += alpha_i p_i for the pending slots i = 0, 1, ... in order (basis_kernel),
// then no iteration is pending. x starts at 0 (cg.cpp:79): the first flush
// starts from 0 instead of reading x, so x needs no zeroing pass. Every
// thread reads the pending count and the zero flag before the last CTA's
// finish() resets them.
template <class VT>
struct FlushXOp {
  using vt = VT;
  static constexpr int NB = 1, ND = 0;
  static constexpr bool kFinishOnly = true;
  VT *x;
  const VT *P;
  long long ld;
  const double *alpha;
  DevState *st;
  struct St {
    VT t;
  };
  __device__ bool active() const { return true; }
  __device__ int count() const { return (int)__ldg(&st->k.aux[A_PENDING]); }
  __device__ const VT *base(int) const { return P; }
  __device__ St init(long long j) const { return {__ldg(&st->k.aux[A_XZERO]) ? (VT)0 : x[j]}; }
  __device__ void step(St &s, int i, const VT (&v)[1]) const {
    s.t = add_rn(mul_rn((VT)__ldg(alpha + i), v[0]), s.t);
  }
  __device__ void done(long long j, const St &s, double (&)[1]) const { x[j] = s.t; }
  __device__ void finish(const double (&)[1]) const {  // last CTA, after every element
    st->k.aux[A_PENDING] = 0;
    st->k.aux[A_XZERO] = 0;
  }
};

// p_next = (beta * p) + r into the next ring slot.
template <class VT>
struct XpbyToOp {
  const VT *p;
  const VT *r;
  VT *out;
  const double *beta;
  static constexpr int ND = 0;
  struct Regs {
    VT p, r;
  };
  __device__ Regs load(long long i) const { return {p[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const VT b = (VT)rd(beta);
    out[i] = add_rn(mul_rn(b, g.p), g.r);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// After iteration L: apply the ring once it is full.
template <class VT>
inline void ring_step(const Env<VT> &E, const DirRing<VT> &R, VT *x, long long L) {
  if (L % R.D == 0) launch_basis(E.ctx, E.n, R.D, FlushXOp<VT>{x, R.P, R.ld, R.alpha, E.st}, E.stop());
}

// After the loop: apply what is pending. Runs after the method has stopped
// (its own done flag set), so only the outer method's flag stops it.
template <class VT>
inline void ring_final(const Env<VT> &E, const DirRing<VT> &R, VT *x) {
  launch_basis(E.ctx, E.n, R.D, FlushXOp<VT>{x, R.P, R.ld, R.alpha, E.st}, Stop{nullptr, E.outer_done});
}

// Carves vectors out of one workspace block: slots of ld entries, the
// vector's own entries at offset `off` (a row-split solve keeps its halo
// around them; on one GPU ld = n, off = 0). Consecutive slots of one take()
// form a basis with stride ld.
template <class VT>
struct Ws {
  VT *base;
  long long ld;
  long long off;
  int used = 0;
  VT *take(int count = 1) {
    VT *p = base + (long long)used * ld + off;
    used += count;
    return p;
  }
};

template <class VT>
ks_status init_state(const Env<VT> &E, const VT *b) {
  launch_scalar(E.ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  launch_vec(E.ctx, E.n, NormBOp<VT>{b, E.st}, Stop{nullptr, E.outer_done});
  return KS_OK;
}

// ------------------------------------------------------------------ true residual
// A VP method that has stopped on its recurrence residual (vpcg.cpp:704-713
// tests r, which drifts from b - A x in finite precision, the more so with an
// FP32 inner solve) checks |b - A x| / |b| in FP64 before its convergence
// stands (ks_params.true_residual). The check's SpMV writes the true residual
// into r (residual replacement). If it passes the eps, the method stays
// converged; otherwise it is marked running again and restarts from its
// current x and r, its iteration count and history carrying on.
template <class VT>
struct TrueChkEpi {
  using acc_t = VT;
  const VT *b;
  VT *r;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    const VT rt = sub_rn(b[i], v);
    r[i] = rt;
    acc[0] = add_rn(acc[0], mul_rn(widen(rt), widen(rt)));
  }
  __device__ void finish(const double (&s)[1]) const {
    if (st->k.done != kConverged) return;
    const double tr = sqrt(s[0]) / st->k.s[S_BNORM];
    st->k.s[S_TRUECNT] += 1.0;
    st->k.s[S_TRUERES] = tr;
    if (!(tr <= st->k.s[S_EPS])) {
      st->k.aux[A_FINAL] = 0;  // GMRES: the next stop assembles x again
      set_done(st, kRunning);
    }
  }
};

struct SetDoneOp {
  DevState *st;
  int code;
  __device__ void run() const {
    if (st->k.done == kRunning) set_done(st, code);
  }
};

// After the method's loop: the check, when it applies. Returns true when the
// method has to go on (the host waits for the answer; this happens only when
// the recurrence test has fired).
template <class VT>
inline bool true_check_continue(const Env<VT> &E, const VT *b, const VT *x, VT *r) {
  if constexpr (!std::is_same<VT, double>::value) {
    return false;  // VP methods run their outer loop in FP64
  } else {
  if (!E.true_check) return false;
  E.halo(*E.A, x);
  launch_spmv<double, double>(E.ctx, *E.A, x, TrueChkEpi<double>{b, r, E.st}, Stop{nullptr, nullptr});
  int done = 0;
  if (cudaMemcpyAsync(&done, &E.st->k.done, sizeof(int), cudaMemcpyDeviceToHost, E.ctx->stream) != cudaSuccess ||
      cudaStreamSynchronize(E.ctx->stream) != cudaSuccess)
    return false;
  return done == kRunning;
  }
}

// No iteration left after a failed check: the method ends as out of loops.
template <class VT>
inline void true_check_exhausted(const Env<VT> &E) {
  launch_scalar(E.ctx, SetDoneOp{E.st, kMaxLoop}, Stop{nullptr, nullptr});
}

// ------------------------------------------------------------------ iteration issue
// Systems small enough that an iteration's kernels take a few microseconds
// are bound by launching: the host spends about as long on the three to five
// launches of an iteration as the GPU spends running them. When every
// iteration issues the same kernels with the same arguments (all device
// state lives in KState), the iterations after the first chunk are replayed
// from a CUDA graph holding kGraphChunk iterations, one host launch per chunk.
// Kernels past the method's stop return at once, as they do without graphs.
constexpr int kGraphChunk = 16;
constexpr long long kGraphMaxN = 1 << 20;  // rows; larger systems are HBM-bound

struct ChunkGraph {
  ks_ctx *ctx;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;  // kernels per replay, for the launch count
  ~ChunkGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  template <class F>
  bool capture(F &&issue) {
    const long long l0 = ctx->launches;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      (void)cudaGetLastError();
      return false;
    }
    issue();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    kernels = ctx->launches - l0;
    ctx->launches = l0;  // counted again at every replay
    if (e != cudaSuccess || !g) {
      (void)cudaGetLastError();
      return false;
    }
    const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      exec = nullptr;
      (void)cudaGetLastError();
      return false;
    }
    return true;
  }
  void launch() {
    cudaGraphLaunch(exec, ctx->stream);
    ctx->launches += kernels;
  }
};

// Issues iterations 1..maxloop: body(L) queues iteration L. `fixed`: every
// iteration after the first queues the same kernels, with arguments that
// repeat with a period dividing kGraphChunk (CG alternates two direction
// slots), so a chunk captured at iteration L replays as iterations
// L + kGraphChunk, L + 2 kGraphChunk, ...
template <class VT, class F>
inline void run_iterations(const Env<VT> &E, bool fixed, F &&body) {
  Poller P{E.ctx, E.hflag, E.lookahead};
  long long L = 1;
  if (fixed && E.outer && !E.comm && E.n <= kGraphMaxN && E.sp.maxloop > 2 * kGraphChunk) {
    // the first chunk is launched directly (it also sets up every kernel)
    for (; L <= kGraphChunk; L++) {
      body(L);
      if (P.step()) return;
    }
    ChunkGraph G{E.ctx};
    if (G.capture([&] {
          for (int j = 0; j < kGraphChunk; j++) body(L + j);
        })) {
      Poller PC{E.ctx, E.hflag, 2};  // lookahead in chunks
      for (; L <= E.sp.maxloop; L += kGraphChunk) {
        G.launch();
        if (PC.step()) return;
      }
      return;
    }
  }
  for (; L <= E.sp.maxloop; L++) {
    body(L);
    if (E.outer && P.step()) return;
  }
}

// SpMV input formed on the fly: the CG direction p_L[c] = beta p_{L-1}[c] +
// r_L[c], with the direction update's operations (XpbyToOp), so every value
// read equals the one the update would have stored, bit for bit.
template <class VT>
struct GDir {
  static constexpr bool kPlain = false;
  const VT *__restrict__ pold;
  const VT *__restrict__ r;
  const double *beta;
  VT b;
  __device__ __forceinline__ GDir prep() const {
    GDir g = *this;
    g.b = (VT)rd(beta);
    return g;
  }
  template <class AT>
  __device__ __forceinline__ AT get(int c) const {
    return (AT)add_rn(mul_rn(b, __ldg(pold + c)), __ldg(r + c));
  }
};

// q = A p with p formed in the SpMV's reads (GDir): the row's own p_L is
// stored for the x update and the next iteration; (p,q) -> alpha (CgMvEpi).
template <class VT>
struct CgMvDirEpi {
  using acc_t = VT;
  const VT *pold;
  const VT *r;
  VT *p;
  VT *q;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    const VT b = (VT)rd(&st->k.s[S_BETA]);
    const VT pi = add_rn(mul_rn(b, pold[i]), r[i]);
    p[i] = pi;
    q[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(pi), widen(v)));
  }
  __device__ void finish(const double (&s)[1]) const {
    st->k.s[S_ALPHA] = rdiv(st, st->k.s[S_RR], s[0]);
  }
};

// SpMV with its input read through a gather GX (mv: a plain vector).
template <class VT, class GX, class Epi>
inline void mv_g(const Env<VT> &E, const CsrDev &M, const GX &gx, const Epi &epi) {
  if constexpr (std::is_same<VT, double>::value) {
    launch_spmv_g<1, double, GX, Epi>(E.ctx, M, gx, gx, epi, E.stop());
  } else {
    if (E.mvals == KS_BF16)
      launch_spmv_g<1, __nv_bfloat16, GX, Epi>(E.ctx, M, gx, gx, epi, E.stop());
    else
      launch_spmv_g<1, float, GX, Epi>(E.ctx, M, gx, gx, epi, E.stop());
  }
}

// cg::solve, with the x update deferred to the direction ring where the
// vectors do not fit in L2. On systems of up to kGraphMaxN rows whose SpMV
// reads a diagonal copy, the SpMV forms the direction p = beta p + r itself
// from the previous direction and r (GDir) and stores its own rows of p: two
// kernels per iteration instead of three, which pays where the iteration is
// bound by its kernel boundaries (512^2 adjoint CG workload on B200: 0.198 ->
// 0.168 s). On larger systems reading two vectors per diagonal costs more
// than the update kernel it removes (160^3 FP32 inner CG: 3.4 us more per
// iteration), and with CSR the gather of two vectors per nonzero does too
// (128^3: 15 us more per SpMV against 8 us saved), so they keep the separate
// direction update.
// Small systems (up to kResMaxRows rows, one GPU, FP64; ks_params.cluster_solve
// 0): the whole solve as one launch of one thread-block cluster
// (ks_resident.cuh). Returns false,
// having launched nothing, when the system does not qualify or no cluster of
// the needed shape fits on the device.
inline bool run_cg_resident(const Env<double> &E, const double *b, double *x, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A->val) return false;
  const ResShape sh = resident_shape(E.n);
  if (!sh.C) return false;
  const CsrDev &A = *E.A;
  const ResCgArgs a{A.ptr, A.col, A.col16, A.val, b, x, E.st, E.ctx->d_err, (int)E.n, sh.shift};
  bool fits = false;
  if (res_cg(sh, A.col16 != nullptr, E.ctx->stream, a, true, &fits) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  launch_scalar(E.ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  E.ctx->launches++;
  ProfLaunch pl(E.ctx, kOther);  // a whole solve in one cluster launch
  const cudaError_t e = res_cg(sh, A.col16 != nullptr, E.ctx->stream, a, false, nullptr);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(E.ctx, e, "cluster-resident CG launch");
  return true;
}

// Larger systems whose vectors fit on chip across the GPU (up to about 14,400
// rows per SM in FP64, one GPU, a diagonal copy; ks_params.cluster_solve 0):
// the whole solve as one cooperative kernel of one CTA per SM, r and q in
// TMEM, p and x in shared memory (k_cg_onchip, ks_inner_resident.cuh): no
// kernel boundary and no vector pass through HBM per iteration, only the
// matrix and the neighbouring CTAs' p. Returns false, having launched
// nothing, when the system does not qualify.
inline bool run_cg_onchip(const Env<double> &E, const double *b, double *x, double *P, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A->dia_nd || !E.A->dia_val) return false;
  ks_ctx *ctx = E.ctx;
  IrShape sh;
  if (!ir_shape<double>(ctx, E.n, &sh, true)) return false;
  bool fits = false;
  const IrArgs probe{};
  if (ir_launch<double, double>(ctx, *E.A, probe, sh, true, &fits, 0) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  // P takes the first two workspace slots: with the stencil path it sits
  // between two zero pads wider than the largest offset
  const long long pad = ir_p_pad(*E.A);
  const bool stencil = ir_stencil_ok(*E.A, E.n) && 2 * E.ld >= E.n + 2 * pad;
  double *const Pp = P + (stencil ? pad : 0);
  if (reinterpret_cast<uintptr_t>(Pp) % 32) return false;  // 32-byte vector loads of P
  launch_scalar(ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  const IrArgs a{b, x, Pp, E.st, nullptr, ctx->partials, (IrSync *)ctx->ir_sync, ctx->d_err, ctx->wait_ns,
                 (int)E.n, sh.rpc, sh.K, 1, stencil ? 1 : 0};
  cudaError_t e = cudaMemsetAsync(ctx->ir_sync, 0, ir_sync_bytes(sh.G), ctx->stream);
  if (e == cudaSuccess && stencil) e = cudaMemsetAsync(P, 0, sizeof(double) * pad, ctx->stream);
  if (e == cudaSuccess && stencil) e = cudaMemsetAsync(Pp + E.n, 0, sizeof(double) * pad, ctx->stream);
  // a profiled solve counts the whole solve as one SpMV-class launch
  if (e == cudaSuccess) e = ir_launch<double, double>(ctx, *E.A, a, sh, false, &fits, kMv);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "on-chip CG launch");
  return true;
}

template <class VT>
ks_status run_cg(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws) {
  if constexpr (std::is_same<VT, double>::value) {
    ks_status s = KS_OK;
    if (run_cg_resident(E, b, x, &s)) return s;
    if (run_cg_onchip(E, b, x, ws, &s)) return s;
  }
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *q = W.take();
  const bool defer = defer_x(E, KS_CG);
  const bool fused = E.A->dia_nd > 0 && !E.comm && E.n <= kGraphMaxN && (!defer || dir_ring(E.sp) >= 2);
  // without the ring: p in place, or two alternating slots when the SpMV forms
  // p (a second slot would crowd the vectors of a large system out of L2)
  const int D = defer ? dir_ring(E.sp) : (fused ? 2 : 1);
  DirRing<VT> R{W.take(D), E.ld, D, dws};
  init_state(E, b);
  if (!defer) vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, R.slot(1), nullptr, nullptr, E.st, START_CG});
  run_iterations(E, !defer, [&](long long L) {
    VT *p = R.slot(L);
    if (fused) {
      // iteration 1: beta = 0 and p_0 := r, so p_1 = 0 r + r = r (r finite)
      const VT *pold = L == 1 ? r : R.slot(L + D - 1);
      mv_g(E, *E.A, GDir<VT>{pold, r, &E.st->k.s[S_BETA], (VT)0}, CgMvDirEpi<VT>{pold, r, p, q, E.st});
    } else {
      mv(E, *E.A, (const VT *)p, CgMvEpi<VT>{p, q, E.st});
    }
    if (defer) {
      vec(E, RUpdOp<VT>{r, q, E.st, 0, R.aslot(L)});
      ring_step(E, R, x, L);
    } else {
      vec(E, XrUpdOp<VT>{x, r, p, q, E.st, 0});
    }
    if (!fused) vec(E, XpbyToOp<VT>{p, r, R.slot(L + 1), &E.st->k.s[S_BETA]});
  });
  if (defer) ring_final(E, R, x);
  return KS_OK;
}

// ------------------------------------------------------------------ CR
// cr::solve (cr.cpp:152-263): x/r update with check; s = A r, (r,s) -> beta;
// p = beta p + r, q = beta q + s with (q,q) -> next alpha.
template <class VT>
struct CrStartMvEpi {  // q = A p; s = q; rs = (r,s); alpha = rs/(q,q)
  using acc_t = VT;
  const VT *r;
  VT *q;
  VT *s;
  DevState *st;
  static constexpr int ND = 2;
  __device__ void row(int i, VT v, double (&acc)[2]) const {
    q[i] = v;
    s[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(r[i]), widen(v)));
    acc[1] = add_rn(acc[1], mul_rn(widen(v), widen(v)));
  }
  __device__ void finish(const double (&sm)[2]) const {
    st->k.s[S_RR] = sm[0];
    st->k.s[S_ALPHA] = rdiv(st, sm[0], sm[1]);
  }
};

template <class VT>
struct CrMvEpi {  // s = A r; rs2 = (r,s); beta = rs2/rs; rs = rs2
  using acc_t = VT;
  const VT *r;
  VT *s;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    s[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(r[i]), widen(v)));
  }
  __device__ void finish(const double (&sm)[1]) const {
    st->k.s[S_BETA] = rdiv(st, sm[0], st->k.s[S_RR]);
    st->k.s[S_RR] = sm[0];
  }
};

// p = beta p + r into the next ring slot; q = beta q + s in place; (q,q) ->
// alpha = s[RR] / (q,q) (Xpby2Op with the direction ring).
template <class VT>
struct Xpby2ToOp {
  const VT *p;
  const VT *r;
  VT *pn;
  VT *q;
  const VT *s;
  DevState *st;
  static constexpr int ND = 1;
  struct Regs {
    VT p, r, q, s;
  };
  __device__ Regs load(long long i) const { return {p[i], r[i], q[i], s[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT b = (VT)rd(&st->k.s[S_BETA]);
    pn[i] = add_rn(mul_rn(b, g.p), g.r);
    const VT qi = add_rn(mul_rn(b, g.q), g.s);
    q[i] = qi;
    acc[0] = add_rn(acc[0], mul_rn(widen(qi), widen(qi)));
  }
  __device__ void finish(const double (&sm)[1]) const { st->k.s[S_ALPHA] = rdiv(st, st->k.s[S_RR], sm[0]); }
};

// CR on small systems as one thread-block-cluster launch (as run_cg_resident).
inline bool run_cr_resident(const Env<double> &E, const double *b, double *x, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A->val) return false;
  const ResShape sh = resident_shape(E.n);
  if (!sh.C) return false;
  const CsrDev &A = *E.A;
  const ResCgArgs a{A.ptr, A.col, A.col16, A.val, b, x, E.st, E.ctx->d_err, (int)E.n, sh.shift};
  bool fits = false;
  if (res_cr(sh, A.col16 != nullptr, E.ctx->stream, a, true, &fits) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  launch_scalar(E.ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  E.ctx->launches++;
  ProfLaunch pl(E.ctx, kOther);  // a whole solve in one cluster launch
  const cudaError_t e = res_cr(sh, A.col16 != nullptr, E.ctx->stream, a, false, nullptr);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(E.ctx, e, "cluster-resident CR launch");
  return true;
}

// CR above the thread-block-cluster limit with r and p in shared memory, q
// and s in TMEM and x in place in global memory (k_cr_onchip,
// ks_inner_resident.cuh: one GPU, FP64, a diagonal copy, up to ~2.1M rows;
// ks_params.cluster_solve 0): the whole solve as one cooperative launch. R,
// the published r, takes workspace slots 0-1, between two zero pads for the
// stencil path. Returns false, having launched nothing, when the system does
// not qualify.
inline bool run_cr_onchip(const Env<double> &E, const double *b, double *x, double *ws, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A->dia_nd || !E.A->dia_val) return false;
  if (reinterpret_cast<uintptr_t>(x) % 16) return false;  // 16-byte vector accesses of x
  ks_ctx *ctx = E.ctx;
  const CsrDev &A = *E.A;
  IrShape sh;
  if (!ir_shape<double>(ctx, E.n, &sh)) return false;
  bool fits = false;
  const IrArgs probe{};
  auto launch = [&](const IrArgs &a, bool pr) {
    return A.dia_nd == 7 ? icr_launch_n<7>(ctx, A, a, sh, pr, &fits)
                         : A.dia_nd == 5 ? icr_launch_n<5>(ctx, A, a, sh, pr, &fits)
                                         : icr_launch_n<0>(ctx, A, a, sh, pr, &fits);
  };
  if (launch(probe, true) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  const long long pad = ir_p_pad(A);
  const bool stencil = ir_stencil_ok(A, E.n) && 2 * E.ld >= E.n + 2 * pad;
  double *const R = ws + (stencil ? pad : 0);
  if (reinterpret_cast<uintptr_t>(R) % 32) return false;  // 32-byte vector loads of R
  launch_scalar(ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  const IrArgs a{b, x, R, E.st, nullptr, ctx->partials, (IrSync *)ctx->ir_sync, ctx->d_err, ctx->wait_ns,
                 (int)E.n, sh.rpc, sh.K, 1, stencil ? 1 : 0};
  cudaError_t e = cudaMemsetAsync(ctx->ir_sync, 0, ir_sync_bytes(sh.G), ctx->stream);
  if (e == cudaSuccess && stencil) e = cudaMemsetAsync(ws, 0, sizeof(double) * pad, ctx->stream);
  if (e == cudaSuccess && stencil) e = cudaMemsetAsync(R + E.n, 0, sizeof(double) * pad, ctx->stream);
  if (e == cudaSuccess) e = launch(a, false);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "on-chip CR launch");
  return true;
}

template <class VT>
ks_status run_cr(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws) {
  if constexpr (std::is_same<VT, double>::value) {
    ks_status s = KS_OK;
    if (run_cr_resident(E, b, x, &s)) return s;
    if (run_cr_onchip(E, b, x, ws, &s)) return s;
  }
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *q = W.take(), *s = W.take();
  const bool defer = defer_x(E, KS_CR);
  const int D = defer ? dir_ring(E.sp) : 1;
  DirRing<VT> R{W.take(D), E.ld, D, dws};
  init_state(E, b);
  if (!defer) vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, R.slot(1), nullptr, nullptr, E.st, START_CHECK});
  mv(E, *E.A, (const VT *)R.slot(1), CrStartMvEpi<VT>{r, q, s, E.st});
  run_iterations(E, !defer, [&](long long L) {
    if (defer) {
      vec(E, RUpdOp<VT>{r, q, E.st, 1, R.aslot(L)});
      ring_step(E, R, x, L);
    } else {
      vec(E, XrUpdOp<VT>{x, r, R.slot(L), q, E.st, 1});
    }
    mv(E, *E.A, (const VT *)r, CrMvEpi<VT>{r, s, E.st});
    vec(E, Xpby2ToOp<VT>{R.slot(L), r, R.slot(L + 1), q, s, E.st});
  });
  if (defer) ring_final(E, R, x);
  return KS_OK;
}

// ------------------------------------------------------------------ BiCG
// bicg::solve (bicg.cpp:162-277).
template <class VT>
struct BicgMvTEpi {  // r* = -alpha (A^T p*) + r*; rr2 = (r*, r) -> beta
  using acc_t = VT;
  VT *rs;
  const VT *r;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    const VT a = (VT)rd(&st->k.s[S_ALPHA]);
    const VT ri = add_rn(mul_rn((VT)(-a), v), rs[i]);
    rs[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(r[i])));
  }
  __device__ void finish(const double (&sm)[1]) const {
    st->k.s[S_BETA] = rdiv(st, sm[0], st->k.s[S_RR]);
    st->k.s[S_RR] = sm[0];
  }
};

// q = A p with (p*, q) -> alpha (CgMvEpi), and t = A^T p* stored for the
// A^T epilogue that runs after the r update (spmv_dia_pair_kernel).
template <class VT>
struct BicgPairEpi {
  using acc_t = VT;
  CgMvEpi<VT> e;
  VT *t;
  static constexpr int ND = 1;
  __device__ void row(int i, VT q, VT tv, double (&acc)[1]) const {
    t[i] = tv;
    e.row(i, q, acc);
  }
  __device__ void finish(const double (&s)[1]) const { e.finish(s); }
};

// BiCG after the pair SpMV, in one pass: x += alpha p (unless deferred),
// r -= alpha q and r* -= alpha t (t = A^T p*), (r,r) for the stopping test and
// (r*,r) for beta (bicg.cpp:242-262) with the engine's decisions in order: the
// test (RUpdOp / XrUpdOp mode 1), then beta (BicgMvTEpi) if it did not stop
// the method. The per-element operations are those two kernels'; (r*,r) adds
// its terms in this pass's order instead of the A^T SpMV's.
template <class VT, bool kDefer>
struct BicgUpd2Op {
  VT *x;
  const VT *p;
  VT *r;
  const VT *q;
  VT *rs;
  const VT *t;
  DevState *st;
  double *aslot;  // the ring's alpha slot (deferred x)
  static constexpr int ND = 2;
  struct Regs {
    VT x, p, q, r, t, rs;
  };
  __device__ Regs load(long long i) const {
    if constexpr (kDefer)
      return {(VT)0, (VT)0, q[i], r[i], t[i], rs[i]};
    else
      return {x[i], p[i], q[i], r[i], t[i], rs[i]};
  }
  __device__ void store(long long i, const Regs &g, double (&acc)[2]) const {
    const VT a = (VT)rd(&st->k.s[S_ALPHA]);
    if constexpr (!kDefer) x[i] = add_rn(mul_rn(a, g.p), g.x);
    const VT ri = add_rn(mul_rn((VT)(-a), g.q), g.r);
    r[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
    const VT si = add_rn(mul_rn((VT)(-a), g.t), g.rs);
    rs[i] = si;
    acc[1] = add_rn(acc[1], mul_rn(widen(si), widen(ri)));
  }
  __device__ void finish(const double (&s)[2]) const {
    if constexpr (kDefer) {
      *aslot = st->k.s[S_ALPHA];
      st->k.aux[A_PENDING]++;
    }
    check_top(st, st->k.loop + 1, sqrt(s[0]) / st->k.s[S_BNORM]);
    if (st->k.done == kRunning) {
      st->k.s[S_BETA] = rdiv(st, s[1], st->k.s[S_RR]);
      st->k.s[S_RR] = s[1];
    }
  }
};

// Whether BiCG's two SpMVs can run as one pass over A's diagonal copy: one
// GPU, 5 or 7 diagonals in the full layout (nd arrays of n values), and A^T's
// copy the mirror of A's (its diagonal k at minus A's offset nd-1-k).
inline bool dia_pair_ok(const CsrDev &A, const CsrDev &T, long long n) {
  const int nd = A.dia_nd;
  if ((nd != 5 && nd != 7) || T.dia_nd != nd || A.dia_sym || T.dia_sym || !A.dia_val || !A.dia_mask ||
      !T.dia_mask)
    return false;
  if (A.n != n || T.n != n || A.dia_ds != n || A.dia_cmin != 0 || A.dia_cmax != n || T.dia_cmin != 0 ||
      T.dia_cmax != n)
    return false;
  for (int k = 0; k < nd; k++)
    if (T.dia_off[k] != -A.dia_off[nd - 1 - k]) return false;
  return true;
}

// A^T's diagonals as a view of A's copy: diagonal k (offset o) is A's
// diagonal nd-1-k (offset -o) read o rows further on; masks are A^T's.
inline DiaT<double> dview_mirror(const CsrDev &A, const CsrDev &T) {
  DiaT<double> d = dview<double>(T);
  const int nd = A.dia_nd;
  for (int k = 0; k < nd; k++) {
    d.vb[k] = A.dia_val + (long long)(nd - 1 - k) * A.dia_ds;
    d.vs[k] = T.dia_off[k];
  }
  return d;
}

// The pair SpMV on the grid of the A SpMV (epilogue EpiA) it replaces, so
// that a sum in its epilogue adds its terms in the same order.
template <int NDG, class EpiA, class Epi>
inline void launch_pair_n(ks_ctx *ctx, const CsrDev &A, const CsrDev &T, const double *p, const double *ps,
                          const Epi &epi, Stop stop) {
  const long long need = ((long long)A.n + kThreads - 1) / kThreads;
  const long long wave = (long long)ctx->num_sms * spmv_dia_ctas_per_sm<1, NDG, double, GPtr<double>, EpiA>(ctx->device);
  ctx->next_class = kMv;
  launch_k(ctx, spmv_dia_pair_kernel<NDG, GPtr<double>, Epi>,
           dim3((unsigned)std::max<long long>(1, std::min(need, wave))), dim3(kThreads), 0, dview<double>(A),
           dview_mirror(A, T), GPtr<double>{p}, GPtr<double>{ps}, epi, stop, red_of(ctx, 0));
}

template <class EpiA, class Epi>
inline void launch_pair(ks_ctx *ctx, const CsrDev &A, const CsrDev &T, const double *p, const double *ps,
                        const Epi &epi, Stop stop) {
  if (A.dia_nd == 7)
    launch_pair_n<7, EpiA, Epi>(ctx, A, T, p, ps, epi, stop);
  else
    launch_pair_n<5, EpiA, Epi>(ctx, A, T, p, ps, epi, stop);
}

// Whether BiCG-type methods take the pair SpMV: one GPU, FP64, the mirrored
// diagonal copies, and a copy that does not fit in L2 (within 60 %, the
// deferred-x rule): a copy that fits is read from L2 by the second SpMV, and
// the separate SpMVs are as fast (convdiff 104^3, 63 MB: 23.8 against
// 24.5 ms for BiCG; 128^3, 117 MB: 47.1 against 43.9 ms).
template <class VT>
inline bool use_pair(const Env<VT> &E) {
  if constexpr (!std::is_same<VT, double>::value) {
    return false;
  } else {
    return !E.comm && E.mvals == KS_FP64 && E.AT && dia_pair_ok(*E.A, *E.AT, E.n) &&
           (double)E.A->dia_nd * (double)E.n * sizeof(double) > 0.6 * (double)E.ctx->l2_bytes;
  }
}

// p_next = beta p + r (pn: the next ring slot, or p itself); ps = beta ps + rs.
template <class VT>
struct Xpby2PlainOp {
  const VT *p;
  const VT *r;
  VT *pn;
  VT *ps;
  const VT *rs;
  const double *beta;
  static constexpr int ND = 0;
  struct Regs {
    VT p, r, ps, rs;
  };
  __device__ Regs load(long long i) const { return {p[i], r[i], ps[i], rs[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const VT b = (VT)rd(beta);
    pn[i] = add_rn(mul_rn(b, g.p), g.r);
    ps[i] = add_rn(mul_rn(b, g.ps), g.rs);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// Ap with p formed in the SpMV's reads (GDir, as in CG): the row's own p_L
// is stored, and p*_L = beta p*_{L-1} + r*_L formed and stored in place (only
// row i reads entry i here); (p*, Ap) -> alpha (CgMvEpi on p*).
template <class VT>
struct BicgMvDirEpi {
  using acc_t = VT;
  const VT *pold;
  const VT *r;
  VT *p;
  VT *ps;
  const VT *rs;
  VT *ap;
  DevState *st;
  static constexpr int ND = 1;
  __device__ void row(int i, VT v, double (&acc)[1]) const {
    const VT b = (VT)rd(&st->k.s[S_BETA]);
    p[i] = add_rn(mul_rn(b, pold[i]), r[i]);
    const VT psi = add_rn(mul_rn(b, ps[i]), rs[i]);
    ps[i] = psi;
    ap[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(psi), widen(v)));
  }
  __device__ void finish(const double (&s)[1]) const {
    st->k.s[S_ALPHA] = rdiv(st, st->k.s[S_RR], s[0]);
  }
};

// BiCG on small systems as one thread-block-cluster launch (as
// run_cg_resident).
inline bool run_bicg_resident(const Env<double> &E, const double *b, double *x, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A->val || !E.AT || !E.AT->val)
    return false;
  const ResShape sh = resident_shape(E.n);
  if (!sh.C) return false;
  const CsrDev &A = *E.A, &T = *E.AT;
  const ResBicgArgs a{A.ptr, A.col,  A.col16, A.val, T.ptr,         T.col,      T.col16,
                      T.val, b,      x,       E.st,  E.ctx->d_err, (int)E.n, sh.shift};
  bool fits = false;
  const bool ia16 = A.col16 != nullptr, it16 = T.col16 != nullptr;
  if (res_bicg(sh, ia16, it16, E.ctx->stream, a, true, &fits) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  launch_scalar(E.ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  E.ctx->launches++;
  ProfLaunch pl(E.ctx, kOther);  // a whole solve in one cluster launch
  const cudaError_t e = res_bicg(sh, ia16, it16, E.ctx->stream, a, false, nullptr);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(E.ctx, e, "cluster-resident BiCG launch");
  return true;
}

// bicg::solve. On systems of up to kGraphMaxN rows with a diagonal copy the
// A-SpMV forms both directions (as run_cg does for p), and the separate
// direction update is gone: three kernels per iteration instead of four.
// BiCG above the thread-block-cluster limit with its six vectors in shared
// memory (k_bicg_onchip, ks_inner_resident.cuh: one GPU, FP64, A and A^T
// with a diagonal copy, up to kIrTile rows per SM; ks_params.
// cluster_solve 0): the whole solve as one cooperative launch. P and P*, the
// published directions, take workspace slots 0-1 and from 2 on, each between
// two zero pads wider than the largest offset. Returns false, having launched
// nothing, when the system does not qualify.
inline bool run_bicg_onchip(const Env<double> &E, const double *b, double *x, double *ws, ks_status *s) {
  if (E.sp.cluster_solve || !E.outer || E.comm || E.mvals != KS_FP64 || !E.A || !E.AT) return false;
  const CsrDev &A = *E.A, &T = *E.AT;
  if (!A.dia_nd || !A.dia_val || A.dia_nd != T.dia_nd || !T.dia_val) return false;
  if (A.dia_cmin != 0 || A.dia_cmax != E.n || T.dia_cmin != 0 || T.dia_cmax != E.n) return false;
  ks_ctx *ctx = E.ctx;
  const long long G = ctx->num_sms;
  const long long rpc = ((E.n + G - 1) / G + 31) / 32 * 32;
  if (G > kIrMaxGrid || rpc > kIrTile) return false;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  const size_t smem = sizeof(double) * kIbVecs * (size_t)rpc;
  if (smem + 2048 > (size_t)optin) return false;
  // the stencil quad path where both qualify (P and P* zero-padded), else
  // the generic quad path (clamped columns)
  const bool stencil = ir_stencil_ok(A, E.n) && ir_stencil_ok(T, E.n);
  const long long pad = stencil ? std::max(ir_p_pad(A), ir_p_pad(T)) : 0;
  if (2 * E.ld < E.n + 2 * pad) return false;
  bool fits = false;
  auto launch = [&](const IrArgs &a, bool pr) {
    return A.dia_nd == 7 ? ib_launch_n<7>(ctx, A, T, a, smem, (int)G, pr, &fits)
                         : A.dia_nd == 5 ? ib_launch_n<5>(ctx, A, T, a, smem, (int)G, pr, &fits)
                                         : ib_launch_n<0>(ctx, A, T, a, smem, (int)G, pr, &fits);
  };
  const IrArgs probe{};
  if (launch(probe, true) != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return false;
  }
  // P in slots 0-1, P* from the next 4-element boundary (32-byte vector
  // loads of both), within BiCG's six or more slots
  const long long ps0 = (2 * E.ld + 3) / 4 * 4;
  if (ps0 + E.n + 2 * pad > 6 * E.ld) return false;
  double *const P = ws + pad, *const Ps = ws + ps0 + pad;
  if (reinterpret_cast<uintptr_t>(P) % 32 || reinterpret_cast<uintptr_t>(Ps) % 32) return false;
  launch_scalar(ctx, InitOp{E.st, E.sp.eps, E.sp.maxloop, E.record ? 1 : 0}, Stop{nullptr, E.outer_done});
  IrArgs a{b, x, P, E.st, nullptr, ctx->partials, (IrSync *)ctx->ir_sync, ctx->d_err, ctx->wait_ns,
           (int)E.n, (int)rpc, 1, 1, stencil ? 1 : 0};
  a.P2 = Ps;
  cudaError_t e = cudaMemsetAsync(ctx->ir_sync, 0, ir_sync_bytes((int)G), ctx->stream);
  if (stencil)
    for (double *z : {ws, P + E.n, ws + ps0, Ps + E.n})
      if (e == cudaSuccess) e = cudaMemsetAsync(z, 0, sizeof(double) * pad, ctx->stream);
  if (e == cudaSuccess) e = launch(a, false);
  *s = e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "on-chip BiCG launch");
  return true;
}

template <class VT>
ks_status run_bicg(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws) {
  if constexpr (std::is_same<VT, double>::value) {
    ks_status s = KS_OK;
    if (run_bicg_resident(E, b, x, &s)) return s;
    if (run_bicg_onchip(E, b, x, ws, &s)) return s;
  }
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *rs = W.take(), *ps = W.take(), *mvv = W.take();
  const bool defer = defer_x(E, KS_BICG);
  const bool fused = E.A->dia_nd > 0 && !E.comm && E.n <= kGraphMaxN && (!defer || dir_ring(E.sp) >= 2);
  const int D = defer ? dir_ring(E.sp) : (fused ? 2 : 1);  // as in run_cg
  DirRing<VT> R{W.take(D), E.ld, D, dws};
  // q = A p and t = A^T p* in one pass over A's diagonal copy (use_pair)
  VT *tv = W.take();
  const bool pair = !fused && use_pair(E);
  init_state(E, b);
  if (!defer) vec(E, ZeroOp<VT>{x});
  // (r*, r) = (r, r) at the start
  start_from_zero(E, StartEpi<VT>{b, r, rs, R.slot(1), ps, E.st, START_CG});
  run_iterations(E, !defer, [&](long long L) {
    VT *p = R.slot(L);
    if (fused) {
      // iteration 1: beta = 0, p_0 := r and p*_0 = r: p_1 = r, p*_1 = r* (r finite)
      const VT *pold = L == 1 ? r : R.slot(L + D - 1);
      mv_g(E, *E.A, GDir<VT>{pold, r, &E.st->k.s[S_BETA], (VT)0},
           BicgMvDirEpi<VT>{pold, r, p, ps, rs, mvv, E.st});
    } else if (pair) {
      if constexpr (std::is_same<VT, double>::value) {
        const BicgPairEpi<double> pe{CgMvEpi<double>{ps, mvv, E.st}, tv};  // alpha = rr/(p*, Ap)
        launch_pair<CgMvEpi<double>>(E.ctx, *E.A, *E.AT, p, ps, pe, E.stop());
      }
    } else {
      mv(E, *E.A, (const VT *)p, CgMvEpi<VT>{ps, mvv, E.st});  // alpha = rr/(p*, Ap)
    }
    if (pair) {
      if (defer) {
        vec(E, BicgUpd2Op<VT, true>{nullptr, nullptr, r, mvv, rs, tv, E.st, R.aslot(L)});
        ring_step(E, R, x, L);
      } else {
        vec(E, BicgUpd2Op<VT, false>{x, p, r, mvv, rs, tv, E.st, nullptr});
      }
    } else {
      if (defer) {
        vec(E, RUpdOp<VT>{r, mvv, E.st, 1, R.aslot(L)});
        ring_step(E, R, x, L);
      } else {
        vec(E, XrUpdOp<VT>{x, r, p, mvv, E.st, 1});
      }
      mv(E, *E.AT, (const VT *)ps, BicgMvTEpi<VT>{rs, r, E.st});
    }
    if (!fused) vec(E, Xpby2PlainOp<VT>{p, r, R.slot(L + 1), ps, rs, &E.st->k.s[S_BETA]});
  });
  if (defer) ring_final(E, R, x);
  return KS_OK;
}

// ------------------------------------------------------------------ GCR
// gcr::solve (gcr.cpp:178-317). Device arrays: qq[m], beta[m].
template <class VT>
struct GcrQ0Epi {  // Q0 = A P0; qq[0] = (Q0,Q0); rq = (r,Q0) -> alpha
  using acc_t = VT;
  const VT *r;
  VT *q0;
  double *qq;
  DevState *st;
  static constexpr int ND = 2;
  __device__ void row(int i, VT v, double (&acc)[2]) const {
    q0[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(v), widen(v)));
    acc[1] = add_rn(acc[1], mul_rn(widen(r[i]), widen(v)));
  }
  __device__ void finish(const double (&s)[2]) const {
    qq[0] = s[0];
    st->k.s[S_ALPHA] = rdiv(st, s[1], s[0]);
  }
};

// x += alpha P_k; if (!last) { r -= alpha Q_k; (r,r) -> check }.
template <class VT>
struct GcrXrOp {
  VT *x;
  VT *r;
  const VT *pk;
  const VT *qk;
  DevState *st;
  int last;
  static constexpr int ND = 1;
  struct Regs {
    VT x, p, q, r;
  };
  __device__ Regs load(long long i) const {
    if (last) return {x[i], pk[i], (VT)0, (VT)0};
    return {x[i], pk[i], qk[i], r[i]};
  }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT a = (VT)rd(&st->k.s[S_ALPHA]);
    x[i] = add_rn(mul_rn(a, g.p), g.x);
    if (!last) {
      const VT ri = add_rn(mul_rn((VT)(-a), g.q), g.r);
      r[i] = ri;
      acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
    }
  }
  __device__ void finish(const double (&s)[1]) const {
    if (!last) check_gcr(st, sqrt(s[0]) / st->k.s[S_BNORM]);
  }
};

struct GcrBetaPut {  // beta[i] = -(Av, Q_i) / qq[i]   (blas::Gcr_sp_1)
  double *beta;
  const double *qq;
  DevState *st;
  __device__ void put(int, int i, double v) const { beta[i] = rdiv(st, -v, qq[i]); }
};

// P_{k+1} = z + sum_i beta_i P_i, Q_{k+1} = Av + sum_i beta_i Q_i, the sums
// accumulated from zero in index order (gcr.cpp:277-308); then
// qq[k+1] = (Q_{k+1},Q_{k+1}) and alpha = (r, Q_{k+1}) / qq[k+1]. Runs in
// basis_kernel over the two bases P and Q.
template <class VT>
struct GcrPQOp {
  using vt = VT;
  static constexpr int NB = 2, ND = 2;
  const VT *P;
  const VT *Q;
  long long ld;
  int k1;  // number of terms (k+1)
  const double *beta;
  const VT *z;
  const VT *Av;
  const VT *r;
  VT *pn;
  VT *qn;
  double *qq_next;
  DevState *st;
  struct St {
    VT pa, qa;
  };
  __device__ bool active() const { return true; }
  __device__ int count() const { return k1; }
  __device__ const VT *base(int b) const { return b == 0 ? P : Q; }
  __device__ St init(long long) const { return {(VT)0, (VT)0}; }
  __device__ void step(St &s, int i, const VT (&v)[2]) const {
    const VT bi = (VT)rd(beta + i);
    s.pa = add_rn(mul_rn(bi, v[0]), s.pa);
    s.qa = add_rn(mul_rn(bi, v[1]), s.qa);
  }
  __device__ void done(long long j, const St &s, double (&acc)[2]) const {
    pn[j] = add_rn(z[j], s.pa);
    const VT qv = add_rn(Av[j], s.qa);
    qn[j] = qv;
    acc[0] = add_rn(acc[0], mul_rn(widen(qv), widen(qv)));
    acc[1] = add_rn(acc[1], mul_rn(widen(r[j]), widen(qv)));
  }
  __device__ void finish(const double (&sm)[2]) const {
    *qq_next = sm[0];
    st->k.s[S_ALPHA] = rdiv(st, sm[1], sm[0]);
  }
};

template <class VT>
struct InnerRunner;  // VP inner solves (defined below)

struct SetLoopOp {
  DevState *st;
  long long v;
  __device__ void run() const { st->k.loop = v; }
};

// Shared GCR / VPGCR body. With `inner` set, each new direction is the inner
// solver's approximation of A^{-1} r (vpgcr.cpp:693-846).
template <class VT>
ks_status run_gcr_core(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws,
                       InnerRunner<VT> *inner) {
  const long long n = E.n, ld = E.ld;
  const int m = (int)E.sp.restart;
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *Av = W.take(), *z = W.take();
  VT *P = W.take(m), *Q = W.take(m);
  double *qq = dws, *beta = dws + m;
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  launch_scalar(E.ctx, SetLoopOp{E.st, 1}, E.stop());  // loop = 1 (gcr.cpp:41)
  Poller P_{E.ctx, E.hflag, E.lookahead};
  long long issued_steps = 0;
  bool stop_host = false;
  bool x_zero = true;  // the first cycle starts from x = 0
  while (!stop_host) {
    // cycle start: r = b - A x, then the first direction
    const StartEpi<VT> se{b, r, inner ? nullptr : P, nullptr, nullptr, E.st, START_GCR};
    if (x_zero)
      start_from_zero(E, se);
    else
      mv(E, *E.A, (const VT *)x, se);
    x_zero = false;
    if (inner) inner->solve(r, P);  // P_0 = M(r)
    mv(E, *E.A, (const VT *)P, GcrQ0Epi<VT>{r, Q, qq, E.st});
    for (int k = 0; k < m; k++) {
      const bool last = (k == m - 1);
      vec(E, GcrXrOp<VT>{x, r, P + (long long)k * ld, Q + (long long)k * ld, E.st, last ? 1 : 0});
      issued_steps++;
      if (last) break;
      const VT *znew = r;
      if (inner) {
        inner->solve(r, z);
        znew = z;
      }
      mv(E, *E.A, znew, StoreEpi<VT, VT>{Av});
      KS_TRY(launch_block_dot<1, VT>(E.ctx, Q, ld, k + 1, Av, nullptr, n, GcrBetaPut{beta, qq, E.st},
                                     E.stop()));
      launch_basis(E.ctx, n, k + 1,
                   GcrPQOp<VT>{P, Q, ld, k + 1, beta, znew, Av, r, P + (long long)(k + 1) * ld,
                               Q + (long long)(k + 1) * ld, qq + k + 1, E.st},
                   E.stop());
      // Each step is one check of the loop counter, so the method has
      // stopped on the device after at most maxloop steps.
      if ((E.outer && P_.step()) || issued_steps >= E.sp.maxloop) {
        stop_host = true;
        break;
      }
    }
    if (stop_host || (E.outer && P_.step()) || issued_steps >= E.sp.maxloop) {
      // VPGCR: x is current after every step; a failed true-residual check
      // restarts the cycles from it
      if (!inner || !true_check_continue(E, b, (const VT *)x, r)) break;
      if (issued_steps >= E.sp.maxloop) {
        true_check_exhausted(E);
        break;
      }
      stop_host = false;
    }
  }
  return KS_OK;
}

// ------------------------------------------------------------------ GMRES
// gmres::solve (gmres.cpp:232-422) / vpgmres::solve (vpgmres.cpp:746-944).
// Device arrays: H (m+1) x m row-major, cs[m], sn[m], e[m+1], y[m].
struct GmArrays {
  double *H, *cs, *sn, *e, *y;
  int m;
};

template <class VT>
struct ScaleOp {  // out = a / t, t from slot (Scalar_x_div_a)
  const VT *a;
  VT *out;
  const double *t;
  static constexpr int ND = 0;
  struct Regs {
    VT a;
  };
  __device__ Regs load(long long i) const { return {a[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const { out[i] = div_rn(g.a, (VT)rd(t)); }
  __device__ void finish(const double (&)[1]) const {}
};

// Stopping test of step k (gmres.cpp:270-324): record (count+1, |e_k|/|b|);
// maxloop first, then eps. The device remembers k for the final assembly.
__device__ __forceinline__ void gm_check(const GmArrays &g, DevState *st, int k) {
  const long long count = st->k.loop;
  const double err = fabs(g.e[k]) / st->k.s[S_BNORM];
  record(st, count + 1, err);
  st->k.aux[A_CONVK] = k;
  if (count + 1 >= st->k.aux[A_MAXLOOP])
    set_done(st, kMaxLoop);
  else if (err <= st->k.s[S_EPS])
    set_done(st, kConverged);
  else if (err != err)
    set_done(st, kNaN);
}

// Cycle start scalars: e = 0, e[0] = t; then the stopping test of step 0.
struct GmCycleOp {
  GmArrays g;
  DevState *st;
  __device__ void run() const {
    for (int i = 0; i < g.m; i++) g.e[i] = 0.0;
    g.e[0] = st->k.s[S_T];
    st->k.aux[A_KIDX] = 0;
    gm_check(g, st, 0);
  }
};

struct GmPutH {  // H[i][k] = (w, V_i)
  double *H;
  int m, k;
  __device__ void put(int, int i, double v) const { H[(long long)i * m + k] = v; }
};

// H[k+1][k] = |w| arrives in s[T] from the block AXPY; then the Givens
// rotations of column k (gmres.cpp:384-399), count++ and, unless step k ends
// the cycle, the stopping test at the top of step k+1.
struct GmGivensOp {  // arguments of gm_givens_kernel
  GmArrays g;
  DevState *st;
  int k;
  int check_next;
};

// The Givens step of column k (gmres.cpp:384-399): H[k+1][k] = |w|, the k
// earlier rotations applied in order, the new rotation, e updated, count++
// and, unless step k ends the cycle, the stopping test of step k+1. The
// column and the rotations are staged in shared memory by the whole CTA, so
// the chain of k dependent rotations reads shared memory, not global memory.
__global__ void __launch_bounds__(kThreads) gm_givens_kernel(GmGivensOp op, Stop stop) {
  extern __shared__ double gsm[];  // column k (k + 2), cs (k), sn (k)
  pdl_wait();
  if (stop()) return;
  const int k = op.k, m = op.g.m;
  double *H = op.g.H;
  double *col = gsm, *cs = gsm + (k + 2), *sn = cs + k;
  for (int i = threadIdx.x; i <= k + 1; i += blockDim.x) col[i] = H[(long long)i * m + k];
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    cs[i] = op.g.cs[i];
    sn[i] = op.g.sn[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    DevState *st = op.st;
    col[k + 1] = st->k.s[S_T];
    for (int i = 0; i <= k - 1; i++) {
      const double t1 = col[i], t2 = col[i + 1];
      col[i] = cs[i] * t1 - sn[i] * t2;
      col[i + 1] = sn[i] * t1 + cs[i] * t2;
    }
    const double hkk = col[k], hk1 = col[k + 1];
    const double a = sqrt(hkk * hkk + hk1 * hk1);
    const double ck = hkk / a, sk = -hk1 / a;
    op.g.cs[k] = ck;
    op.g.sn[k] = sk;
    op.g.e[k + 1] = sk * op.g.e[k];
    op.g.e[k] = ck * op.g.e[k];
    col[k] = ck * col[k] - sk * col[k + 1];
    col[k + 1] = 0.0;
    st->k.loop += 1;
    if (op.check_next) gm_check(op.g, st, k + 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i <= k + 1; i += blockDim.x) H[(long long)i * m + k] = col[i];
  pdl_trigger();
}

// Back substitution y = H^{-1} e on the leading size x size block
// (blas::Hye, blas.cpp:303-314). size < 0: take size from the stop step.
struct GmHyeOp {
  GmArrays g;
  DevState *st;
  int size;
  int final_mode;  // 1: run only when the method has stopped and not yet assembled
  __device__ void run() const {
    if (final_mode) {
      const int d = st->k.done;
      if (!(d == kConverged || d == kMaxLoop) || st->k.aux[A_FINAL]) return;
    }
    const int sz = size >= 0 ? size : (int)st->k.aux[A_CONVK];
    for (int i = 0; i < g.m; i++) g.y[i] = 0.0;
    for (int i = sz - 1; i >= 0; i--) {
      double t = 0.0;
      for (int j = i + 1; j < sz; j++) t += g.y[j] * g.H[(long long)i * g.m + j];
      g.y[i] = (g.e[i] - t) / g.H[(long long)i * g.m + i];
    }
  }
};

// x = x + sum_i y_i B_i, the sum accumulated from zero in index order
// (gmres.cpp:409-419), in basis_kernel. With `final_mode` the count comes
// from the stop step, and the update runs only once the method has stopped
// by convergence or maxloop and has not been assembled yet; `overwrite`
// reproduces the reference's Scalar_ax assembly (gmres.cpp:290-297): only
// the last term survives.
template <class VT>
struct GmUpdateOp {
  using vt = VT;
  static constexpr int NB = 1, ND = 0;
  const VT *B;
  long long ld;
  int cnt;
  const double *y;
  VT *x;
  const DevState *st;
  int final_mode;
  int overwrite;
  struct St {
    VT t;
  };
  __device__ int terms() const { return final_mode ? (int)st->k.aux[A_CONVK] : cnt; }
  __device__ bool active() const {
    if (!final_mode) return true;
    const int d = st->k.done;
    return (d == kConverged || d == kMaxLoop) && !st->k.aux[A_FINAL];
  }
  __device__ int count() const { return overwrite ? 0 : terms(); }
  __device__ const VT *base(int) const { return B; }
  __device__ St init(long long j) const {
    const int c = terms();
    if (overwrite && c > 0) return {mul_rn((VT)rd(y + c - 1), B[(long long)(c - 1) * ld + j])};
    return {(VT)0};
  }
  __device__ void step(St &s, int i, const VT (&v)[1]) const { s.t = add_rn(s.t, mul_rn((VT)rd(y + i), v[0])); }
  __device__ void done(long long j, const St &s, double (&)[1]) const { x[j] = add_rn(x[j], s.t); }
  __device__ void finish(const double (&)[1]) const {}
};

struct GmMarkFinal {
  DevState *st;
  __device__ void run() const {
    const int d = st->k.done;
    if ((d == kConverged || d == kMaxLoop) && !st->k.aux[A_FINAL]) st->k.aux[A_FINAL] = 1;
  }
};

template <class VT>
ks_status run_gmres_core(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws,
                         InnerRunner<VT> *inner) {
  const long long n = E.n, ld = E.ld;
  const int m = (int)E.sp.restart;
  if (m < 2) return set_error(E.ctx, KS_BAD_INPUT, "GMRES needs restart >= 2");
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *w = W.take(), *z = W.take();
  VT *V = W.take(m + 1);
  VT *Z = inner ? W.take(m) : nullptr;
  GmArrays g{dws, dws + (long long)(m + 1) * m, dws + (long long)(m + 1) * m + m,
             dws + (long long)(m + 1) * m + 2 * m, dws + (long long)(m + 1) * m + 3 * m + 1, m};
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  Poller P{E.ctx, E.hflag, E.lookahead};
  long long issued = 0;
  bool stop_host = false;
  const VT *B = inner ? Z : V;
  bool x_zero = true;  // the first cycle starts from x = 0
 restart:
  while (!stop_host) {
    const StartEpi<VT> se{b, r, nullptr, nullptr, nullptr, E.st, START_NORM};
    if (x_zero)
      start_from_zero(E, se);
    else
      mv(E, *E.A, (const VT *)x, se);
    x_zero = false;
    vec(E, ScaleOp<VT>{r, V, &E.st->k.s[S_T]});
    launch_scalar(E.ctx, GmCycleOp{g, E.st}, E.stop());
    for (int k = 0; k < m - 1; k++) {
      const VT *vk = V + (long long)k * ld;
      if (inner) {
        inner->solve(vk, Z + (long long)k * ld);
        mv(E, *E.A, (const VT *)(Z + (long long)k * ld), StoreEpi<VT, VT>{w});
      } else {
        mv(E, *E.A, vk, StoreEpi<VT, VT>{w});
      }
      KS_TRY(launch_block_dot<1, VT>(E.ctx, V, ld, k + 1, w, nullptr, n, GmPutH{g.H, m, k}, E.stop()));
      launch_basis(E.ctx, n, k + 1, BlockAxpyOp<VT>{V, ld, k + 1, g.H + k, m, w, &E.st->k.s[S_T], 1},
                   E.stop());  // s[T] = |w|
      vec(E, ScaleOp<VT>{w, V + (long long)(k + 1) * ld, &E.st->k.s[S_T]});
      launch_k(E.ctx, gm_givens_kernel, dim3(1), dim3(kThreads), sizeof(double) * (size_t)(3 * k + 2),
               GmGivensOp{g, E.st, k, k + 1 < m - 1 ? 1 : 0}, E.stop());
      issued++;
      if (E.outer && P.step()) {
        stop_host = true;
        break;
      }
      if (issued >= E.sp.maxloop) {
        stop_host = true;
        break;
      }
    }
    if (stop_host) break;
    // end of cycle (gmres.cpp:409-421)
    launch_scalar(E.ctx, GmHyeOp{g, E.st, m - 1, 0}, E.stop());
    launch_basis(E.ctx, n, m - 1, GmUpdateOp<VT>{B, ld, m - 1, g.y, x, E.st, 0, 0}, E.stop());
    if (E.outer && P.step()) break;
  }
  // The step that stopped the method (converged or maxloop) assembles x;
  // these kernels are gated by the stop reason, not by `done`.
  launch_scalar(E.ctx, GmHyeOp{g, E.st, -1, 1}, Stop{nullptr, E.outer_done});
  launch_basis(E.ctx, n, m - 1, GmUpdateOp<VT>{B, ld, 0, g.y, x, E.st, 1, E.faithful ? 1 : 0},
               Stop{nullptr, E.outer_done});
  launch_scalar(E.ctx, GmMarkFinal{E.st}, Stop{nullptr, E.outer_done});
  // VPGMRES: x is assembled; a failed true-residual check starts a new cycle
  // from it (the cycle start recomputes r = b - A x)
  if (inner && true_check_continue(E, b, (const VT *)x, r)) {
    if (issued >= E.sp.maxloop) {
      true_check_exhausted(E);
      return KS_OK;
    }
    stop_host = false;
    P = Poller{E.ctx, E.hflag, E.lookahead};
    goto restart;
  }
  return KS_OK;
}

// ------------------------------------------------------------------ k-skip CG
// kskipcg::solve (kskipcg.cpp:187-310). Per block of k+1 iterations: the
// matrix powers (4k+3 SpMVs in 2k+2 shared passes), one Gram pass, the scalar
// recurrence for all k+1 steps on the device, then k+1 x (SpMV + update).
// Device arrays: G = [delta(2k) | eta(2k+2) | zeta(2k+2)], coef = [alpha | beta](k+1).
struct KsCheckOp {  // gamma = (r,r) arrives in s[GAMMA]; check (nloop+1)
  DevState *st;
  long long nloop;
  __device__ void run() const {
    st->k.loop = nloop;
    const double g = st->k.s[S_GAMMA];
    const double err = sqrt(g) / st->k.s[S_BNORM];
    record(st, nloop + 1, err);
    if (err <= st->k.s[S_EPS])
      set_done(st, kConverged);
    else if (err != err)
      set_done(st, kNaN);
  }
};

struct KsCgRecOp {
  DevState *st;
  double *G;  // delta | eta | zeta
  double *coef;
  int k, fix, fixed;
  __device__ void run() const {
    double *delta = G, *eta = G + 2 * k, *zeta = G + 4 * k + 2;
    double gamma = st->k.s[S_GAMMA];
    for (int i = 0; i <= k; i++) {
      const double alpha = gamma / zeta[0];
      const double beta = alpha * zeta[1] / zeta[0] - 1.0;
      if (fix == 1) {
        gamma = beta * gamma;
      } else if (fix == 2) {
        const double t0 = gamma - alpha * eta[0];
        const double t1 = eta[0] - alpha * zeta[1];
        gamma = t0 - alpha * t1;
      }
      const int cnt = 2 * k - 2 * i;
      for (int j = 0; j < cnt; j++) {
        if (!fixed) {
          delta[j] = delta[j] - 2 * alpha * eta[j + 1] + alpha * alpha * eta[j + 2];
          const double eta_old = eta[j];
          eta[j] = delta[j] + beta * zeta[j + 1] - alpha * beta * zeta[j + 1];
          zeta[j] = eta[j + 1] + beta * eta_old + beta * beta * zeta[j] - alpha * beta * zeta[j + 1];
        } else {
          const double d = delta[j] - 2 * alpha * eta[j + 1] + alpha * alpha * zeta[j + 2];
          const double rp = eta[j] - alpha * zeta[j + 1];
          const double e = d + beta * rp;
          const double z = e + beta * rp + beta * beta * zeta[j];
          delta[j] = d;
          eta[j] = e;
          zeta[j] = z;
        }
      }
      coef[i] = alpha;
      coef[k + 1 + i] = beta;
    }
  }
};

// x += a p; r -= a Av; p = b p + r (kskipcg.cpp:292-305).
template <class VT>
struct KsUpdOp {
  VT *x;
  VT *r;
  VT *p;
  const VT *Av;
  const double *a;
  const double *bt;
  static constexpr int ND = 0;
  struct Regs {
    VT x, r, p, Av;
  };
  __device__ Regs load(long long i) const { return {x[i], r[i], p[i], Av[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const VT al = (VT)rd(a), be = (VT)rd(bt);
    x[i] = add_rn(mul_rn(al, g.p), g.x);
    const VT ri = add_rn(mul_rn((VT)(-al), g.Av), g.r);
    r[i] = ri;
    p[i] = add_rn(mul_rn(be, g.p), ri);
  }
  __device__ void finish(const double (&)[1]) const {}
};

template <class VT>
struct GammaOp {  // s[GAMMA] = (u, v)
  const VT *u;
  const VT *v;
  DevState *st;
  static constexpr int ND = 1;
  struct Regs {
    VT u, v;
  };
  __device__ Regs load(long long i) const { return {u[i], v[i]}; }
  __device__ void store(long long, const Regs &g, double (&acc)[1]) const {
    acc[0] = add_rn(acc[0], mul_rn(widen(g.u), widen(g.v)));
  }
  __device__ void finish(const double (&s)[1]) const { st->k.s[S_GAMMA] = s[0]; }
};

template <class VT>
struct Store2 {
  using acc_t = VT;
  VT *y0, *y1;
  static constexpr int ND = 0;
  __device__ void row(int r, VT a, VT b, double (&)[1]) const {
    y0[r] = a;
    y1[r] = b;
  }
  __device__ void finish(const double (&)[1]) const {}
};

template <class VT>
void matpow_t(const Env<VT> &E, const VT *r, const VT *p, int k, VT *Ar, VT *Ap) {
  const long long n = E.n, ld = E.ld;
  auto mv2 = [&](const VT *a, const VT *b2, VT *o0, VT *o1) {
    E.halo(*E.A, a);
    E.halo(*E.A, b2);
    if constexpr (std::is_same<VT, double>::value) {
      launch_spmv2<double, double>(E.ctx, *E.A, a, b2, Store2<VT>{o0, o1}, E.stop());
    } else {
      if (E.mvals == KS_BF16)
        launch_spmv2<__nv_bfloat16, float>(E.ctx, *E.A, a, b2, Store2<VT>{o0, o1}, E.stop());
      else
        launch_spmv2<float, float>(E.ctx, *E.A, a, b2, Store2<VT>{o0, o1}, E.stop());
    }
  };
  mv2(r, p, Ar, Ap);
  for (int i = 1; i < 2 * k + 1; i++)
    mv2(Ar + (long long)(i - 1) * ld, Ap + (long long)(i - 1) * ld, Ar + (long long)i * ld,
        Ap + (long long)i * ld);
  mv(E, *E.A, (const VT *)(Ap + (long long)(2 * k) * ld), StoreEpi<VT, VT>{Ap + (long long)(2 * k + 1) * ld});
}

template <class VT>
ks_status run_kskipcg(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws) {
  const long long n = E.n, ld = E.ld;
  const int k = E.sp.kskip;
  if (k < 0) return set_error(E.ctx, KS_BAD_INPUT, "kskip must be >= 0");
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *p = W.take(), *Av = W.take();
  VT *Ar = W.take(2 * k + 1), *Ap = W.take(2 * k + 2);
  double *G = dws, *coef = dws + 6 * k + 4;
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, p, nullptr, nullptr, E.st, START_KSKIP});
  Poller P{E.ctx, E.hflag, E.lookahead};
  long long nloop = 0;
  for (nloop = 0; nloop < E.sp.maxloop; nloop += k + 1) {
    vec(E, GammaOp<VT>{r, r, E.st});
    launch_scalar(E.ctx, KsCheckOp{E.st, nloop}, E.stop());
    matpow_t(E, r, p, k, Ar, Ap);
    if (k > 0)
      KS_TRY(launch_block_dot<1, VT>(E.ctx, Ar, ld, 2 * k, r, nullptr, n, PutArray{G, 0, 1}, E.stop()));
    KS_TRY(launch_block_dot<2, VT>(E.ctx, Ap, ld, 2 * k + 2, r, p, n,
                                   PutArray{G + 2 * k, 2 * k + 2, 1}, E.stop()));
    launch_scalar(E.ctx, KsCgRecOp{E.st, G, coef, k, E.sp.fix, E.faithful ? 0 : 1}, E.stop());
    for (int i = 0; i <= k; i++) {
      mv(E, *E.A, (const VT *)p, StoreEpi<VT, VT>{Av});
      vec(E, KsUpdOp<VT>{x, r, p, Av, coef + i, coef + k + 1 + i});
    }
    if (E.outer && P.step()) break;
  }
  return KS_OK;
}

// ------------------------------------------------------------------ k-skip BiCG
// kskipBicg::solve (kskipbicg.cpp:207-352).
// G = [theta(2k+1) | rho(2k+1) | eta(2k+2) | phi(2k+2)].
struct KsBicgRecOp {
  DevState *st;
  double *G;
  double *coef;
  int k;
  __device__ void run() const {
    double *theta = G, *rho = G + 2 * k + 1, *eta = G + 4 * k + 2, *phi = G + 6 * k + 4;
    double gamma = st->k.s[S_GAMMA];
    for (int i = 0; i <= k; i++) {
      const double alpha = gamma / phi[0];
      const double beta = 1.0 - (eta[0] + rho[0] - alpha * phi[1]) / phi[0];
      gamma = gamma * beta;
      const int cnt = 2 * k - 2 * i;
      for (int j = 0; j < cnt; j++) {
        theta[j] = theta[j] - alpha * eta[j + 1] - alpha * rho[j + 1] + alpha * alpha * phi[j + 2];
        const double t = theta[j] - alpha * beta * phi[j + 1];
        eta[j] = t + beta * eta[j];
        rho[j] = t + beta * rho[j];
        phi[j] = eta[j] + rho[j] - theta[j] + beta * beta * phi[j];
      }
      coef[i] = alpha;
      coef[k + 1 + i] = beta;
    }
  }
};

template <class VT>
struct KsXrOp {  // x += a p; r -= a Av
  VT *x;
  VT *r;
  const VT *p;
  const VT *Av;
  const double *a;
  static constexpr int ND = 0;
  struct Regs {
    VT x, p, r, av;
  };
  __device__ Regs load(long long i) const { return {x[i], p[i], r[i], Av[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const VT al = (VT)rd(a);
    x[i] = add_rn(mul_rn(al, g.p), g.x);
    r[i] = add_rn(mul_rn((VT)(-al), g.av), g.r);
  }
  __device__ void finish(const double (&)[1]) const {}
};

template <class VT>
struct KsRsEpi {  // r* = -a (A^T p*) + r*
  using acc_t = VT;
  VT *rs;
  const double *a;
  static constexpr int ND = 0;
  __device__ void row(int i, VT v, double (&)[1]) const {
    rs[i] = add_rn(mul_rn((VT)(-rd(a)), v), rs[i]);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// Av = A p and r* = -a (A^T p*) + r* (KsRsEpi) in one pass (the pair SpMV;
// no sums, so the same bits as the two SpMVs).
template <class VT>
struct KsPairEpi {
  using acc_t = VT;
  VT *Av;
  VT *rs;
  const double *a;
  static constexpr int ND = 0;
  __device__ void row(int i, VT q, VT t, double (&)[1]) const {
    Av[i] = q;
    rs[i] = add_rn(mul_rn((VT)(-rd(a)), t), rs[i]);
  }
  __device__ void finish(const double (&)[1]) const {}
};

template <class VT>
ks_status run_kskipbicg(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws) {
  const long long n = E.n, ld = E.ld;
  const int k = E.sp.kskip;
  if (k < 0) return set_error(E.ctx, KS_BAD_INPUT, "kskip must be >= 0");
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *p = W.take(), *rs = W.take(), *ps = W.take(), *Av = W.take();
  VT *Ar = W.take(2 * k + 1), *Ap = W.take(2 * k + 2);
  double *G = dws, *coef = dws + 8 * k + 6;
  const bool pair = use_pair(E);  // A p and A^T p* in one pass
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, p, rs, ps, E.st, START_KSKIP});
  Poller P{E.ctx, E.hflag, E.lookahead};
  for (long long nloop = 0; nloop < E.sp.maxloop; nloop += k + 1) {
    // the check uses |r|; gamma = (r*, r) comes right after
    vec(E, GammaOp<VT>{r, r, E.st});
    launch_scalar(E.ctx, KsCheckOp{E.st, nloop}, E.stop());
    matpow_t(E, r, p, k, Ar, Ap);
    vec(E, GammaOp<VT>{rs, r, E.st});
    KS_TRY(launch_block_dot<2, VT>(E.ctx, Ar, ld, 2 * k + 1, rs, ps, n, PutArray{G, 2 * k + 1, 1},
                                   E.stop()));
    KS_TRY(launch_block_dot<2, VT>(E.ctx, Ap, ld, 2 * k + 2, rs, ps, n,
                                   PutArray{G + 4 * k + 2, 2 * k + 2, 1}, E.stop()));
    launch_scalar(E.ctx, KsBicgRecOp{E.st, G, coef, k}, E.stop());
    for (int i = 0; i <= k; i++) {
      if (pair) {
        if constexpr (std::is_same<VT, double>::value)
          launch_pair<StoreEpi<double, double>>(E.ctx, *E.A, *E.AT, p, ps, KsPairEpi<double>{Av, rs, coef + i},
                                                E.stop());
        vec(E, KsXrOp<VT>{x, r, p, Av, coef + i});
      } else {
        mv(E, *E.A, (const VT *)p, StoreEpi<VT, VT>{Av});
        vec(E, KsXrOp<VT>{x, r, p, Av, coef + i});
        mv(E, *E.AT, (const VT *)ps, KsRsEpi<VT>{rs, coef + i});
      }
      vec(E, Xpby2PlainOp<VT>{p, r, p, ps, rs, coef + k + 1 + i});
    }
    if (E.outer && P.step()) break;
  }
  return KS_OK;
}

// ------------------------------------------------------------------ sizes
inline long long vec_count(int method, const Params &sp, long long n, size_t elem, size_t l2) {
  const long long m = sp.restart, k = sp.kskip;
  switch (method) {
    case KS_CG: return 2 + dir_slots(method, sp, n, elem, l2);
    case KS_CR: return 3 + dir_slots(method, sp, n, elem, l2);
    case KS_BICG: return 5 + dir_slots(method, sp, n, elem, l2);  // + A^T p* of the pair SpMV
    case KS_GCR: case KS_VPGCR: return 3 + 2 * m;
    case KS_GMRES: return 3 + (m + 1);
    case KS_VPGMRES: return 3 + (m + 1) + m;
    case KS_KSKIPCG: return 3 + (2 * k + 1) + (2 * k + 2);
    case KS_KSKIPBICG: return 5 + (2 * k + 1) + (2 * k + 2);
    case KS_VPCG: return 3 + (defer_x(KS_CG, sp, n, elem, l2) ? dir_ring(sp) : 1);  // r, z, A p, directions
    case KS_VPCR: return 5;
  }
  return 0;
}

inline long long dws_count(int method, const Params &sp) {
  const long long m = sp.restart, k = sp.kskip;
  switch (method) {
    case KS_GCR: case KS_VPGCR: return 2 * m + 2;
    case KS_GMRES: case KS_VPGMRES: return (m + 1) * m + 4 * m + 4;
    case KS_KSKIPCG: return 6 * k + 4 + 2 * (k + 1) + 4;
    case KS_KSKIPBICG: return 8 * k + 6 + 2 * (k + 1) + 4;
    case KS_CG: case KS_CR: case KS_BICG: case KS_VPCG: return kDirRing + 4;  // alpha ring
  }
  return 4;
}

// ------------------------------------------------------------------ inner solves
// A VP method's inner solve z ~ A^{-1} r (innerMethods::innerSelect,
// innerMethods.cpp:71-118): a fresh run of the inner method with the inner
// parameters, zero start, no history. In FP32/BF16 mode the right-hand side
// is rounded to FP32 on entry and z widened back to FP64 on exit.
template <class IT>
ks_status run_method(int method, const Env<IT> &E, const IT *b, IT *x, IT *ws, double *dws,
                     InnerRunner<IT> *inner);

// ------------------------------------------------------------------ on-chip inner CG
// The FP32 (or BF16-valued) inner CG of a VP method on a one-GPU matrix with
// a diagonal copy runs as one cooperative kernel per inner solve, its vectors
// on chip (k_inner_cg_resident, ks_inner_resident.cuh). Around it: the start
// (r = (float) b, (r,r), the state reset) and the end (z = (double) x) are
// vector passes, fused into the outer method's own kernels where the outer
// method is VPCG (its x/r update and its (r, z)).

// The inner state's reset (InitOp without history) and the top of iteration 1
// (StartZeroOp with START_CG, x = 0): |b| and (r,r) are the same sum.
__device__ __forceinline__ void inner_cg_start(DevState *st, double eps, long long maxloop, double rr) {
  st->k.done = kRunning;
  st->k.loop = 0;
  st->k.hlen = 0;
  st->k.s[S_EPS] = eps;
  st->k.aux[A_MAXLOOP] = maxloop;
  st->k.aux[A_RECORD] = 0;
  st->k.aux[A_CONVK] = 0;
  st->k.aux[A_FINAL] = 0;
  st->k.aux[A_PENDING] = 0;
  st->k.aux[A_XZERO] = 1;
  st->k.s[S_BETA] = 0.0;
  st->k.s[S_BNORM] = sqrt(rr);
  st->k.s[S_RR] = rr;
  check_top(st, 1, sqrt(rr) / st->k.s[S_BNORM]);
}

// Inner start from an outer vector b: r = (VT) b (ConvertOp), (r,r).
template <class VT>
struct CgInStartOp {
  const double *b;
  VT *r;
  DevState *st;
  double eps;
  long long maxloop;
  static constexpr int ND = 1;
  struct Regs {
    double b;
  };
  __device__ Regs load(long long i) const { return {b[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const VT ri = (VT)g.b;
    r[i] = ri;
    acc[0] = add_rn(acc[0], mul_rn(widen(ri), widen(ri)));
  }
  __device__ void finish(const double (&s)[1]) const { inner_cg_start(st, eps, maxloop, s[0]); }
};

// Inner end: z = (double) x (ConvertOp of the kernel-per-step loop's x; x
// is 0 if the inner method stopped before its first update), not stored
// when z is null. mode 1 / 2 also fuse VPCG's RzOp (init / beta) over the
// outer r and z on the outer state.
template <class VT>
struct CgInFinalOp {
  const VT *x;
  const DevState *ist;
  double *z;
  const double *r;
  DevState *ost;
  int mode;
  static constexpr int ND = 1;
  struct Regs {
    VT x;
    double r;
  };
  __device__ Regs load(long long i) const { return {x[i], mode ? r[i] : 0.0}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[1]) const {
    const double zi = __ldg(&ist->k.aux[A_XZERO]) ? 0.0 : (double)g.x;
    if (z) z[i] = zi;
    acc[0] = add_rn(acc[0], mul_rn(g.r, zi));
  }
  __device__ void finish(const double (&s)[1]) const {
    if (mode == 2) ost->k.s[S_BETA] = rdiv(ost, s[0], ost->k.s[S_RR]);
    if (mode) ost->k.s[S_RR] = s[0];
  }
};

// VPCG's direction update p = beta p + z (XpbyOp) with z read as the fast
// inner CG's solution in its own precision, widened in the register (0 while
// the inner solve left it at zero, as CgInFinalOp): the same bits as XpbyOp
// over the FP64 copy of z, which is then neither written nor read (160^3:
// 32.8 MB less written and 16.4 MB less read per outer iteration).
template <class IT>
struct XpbyInOp {
  const double *p;
  const IT *x;
  const DevState *ist;
  const double *beta;
  double *out;  // p itself, or the next slot of the direction ring
  static constexpr int ND = 0;
  struct Regs {
    double p;
    IT x;
  };
  __device__ Regs load(long long i) const { return {p[i], x[i]}; }
  __device__ void store(long long i, const Regs &g, double (&)[1]) const {
    const double zi = __ldg(&ist->k.aux[A_XZERO]) ? 0.0 : (double)g.x;
    out[i] = add_rn(mul_rn(rd(beta), g.p), zi);
  }
  __device__ void finish(const double (&)[1]) const {}
};

// VPCG's outer x/r update (XrUpdOp mode 1) fused with the start of the next
// fast inner solve from the new r: (r,r) in FP64 for the outer stopping
// test, r rounded to the inner precision and its (r,r) for the inner start.
template <class IT>
struct VpXrStartOp {
  double *x;
  double *r;
  const double *p;
  const double *q;
  DevState *st;
  IT *ri;
  DevState *ist;
  double ieps;
  long long imaxloop;
  static constexpr int ND = 2;
  struct Regs {
    double x, p, q, r;
  };
  __device__ Regs load(long long i) const { return {x[i], p[i], q[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[2]) const {
    const double a = rd(&st->k.s[S_ALPHA]);
    x[i] = add_rn(mul_rn(a, g.p), g.x);
    const double rn = add_rn(mul_rn(-a, g.q), g.r);
    r[i] = rn;
    acc[0] = add_rn(acc[0], mul_rn(rn, rn));
    const IT r32 = (IT)rn;
    ri[i] = r32;
    acc[1] = add_rn(acc[1], mul_rn(widen(r32), widen(r32)));
  }
  __device__ void finish(const double (&s)[2]) const {
    check_top(st, st->k.loop + 1, sqrt(s[0]) / st->k.s[S_BNORM]);
    inner_cg_start(ist, ieps, imaxloop, s[1]);
  }
};

// VpXrStartOp with x deferred to the direction ring (as RUpdOp for CG):
// r -= alpha q, the same sums in the same order, alpha recorded beside the
// ring slot and the iteration counted as pending for x.
template <class IT>
struct VpRStartOp {
  double *r;
  const double *q;
  DevState *st;
  IT *ri;
  DevState *ist;
  double ieps;
  long long imaxloop;
  double *aslot;
  static constexpr int ND = 2;
  struct Regs {
    double q, r;
  };
  __device__ Regs load(long long i) const { return {q[i], r[i]}; }
  __device__ void store(long long i, const Regs &g, double (&acc)[2]) const {
    const double a = rd(&st->k.s[S_ALPHA]);
    const double rn = add_rn(mul_rn(-a, g.q), g.r);
    r[i] = rn;
    acc[0] = add_rn(acc[0], mul_rn(rn, rn));
    const IT r32 = (IT)rn;
    ri[i] = r32;
    acc[1] = add_rn(acc[1], mul_rn(widen(r32), widen(r32)));
  }
  __device__ void finish(const double (&s)[2]) const {
    *aslot = st->k.s[S_ALPHA];
    st->k.aux[A_PENDING]++;
    check_top(st, st->k.loop + 1, sqrt(s[0]) / st->k.s[S_BNORM]);
    inner_cg_start(ist, ieps, imaxloop, s[1]);
  }
};

// The on-chip inner CG's buffers: its right-hand side r (FP32), the
// published directions P and the solution x, in the inner workspace.
struct InnerResBufs {
  float *r, *P, *x;
  int stencil;  // P zero-padded for the stencil path (ir_stencil_ok)
};

// One inner solve with the on-chip kernel (its start already issued).
inline ks_status run_cg_inner_resident(const Env<float> &E, const InnerResBufs &B, const IrShape &sh) {
  ks_ctx *ctx = E.ctx;
  IrArgs a{B.r, B.x, B.P, E.st, E.outer_done, ctx->partials, (IrSync *)ctx->ir_sync, ctx->d_err, ctx->wait_ns,
           (int)E.n, sh.rpc, sh.K, 0, B.stencil};
  cudaError_t e = cudaMemsetAsync(ctx->ir_sync, 0, ir_sync_bytes(sh.G), ctx->stream);
  if (e == cudaSuccess) {
    bool fits = false;
    e = E.mvals == KS_BF16 ? ir_launch<float, __nv_bfloat16>(ctx, *E.A, a, sh, false, &fits, kMvLow)
                           : ir_launch<float, float>(ctx, *E.A, a, sh, false, &fits, kMvLow);
  }
  return e == cudaSuccess ? KS_OK : cuda_fail(ctx, e, "on-chip inner CG launch");
}

template <class VT>
struct InnerRunner {
  // Outer-precision view (VT) and the inner environment.
  ks_ctx *ctx = nullptr;
  int method = KS_NONE;
  ks_precision iprec = KS_FP64;
  long long n = 0;
  Env<double> E64;
  Env<float> E32;
  double *ws64 = nullptr;
  float *ws32 = nullptr;
  double *dws = nullptr;
  float *b32 = nullptr, *z32 = nullptr;
  long long calls = 0;
  ks_status status = KS_OK;
  // on-chip inner CG (see above): chosen at set-up
  bool res_cg = false;
  InnerResBufs fb{};
  IrShape sh{};
  void setup_resident();
  void solve(const VT *b, VT *z);
};

// The on-chip inner CG applies where the inner method is CG in FP32 or with
// BF16 values, on one GPU, the SpMV reads a diagonal copy of those values,
// and the system fits the kernel's shape (ir_shape) on this device.
template <class VT>
void InnerRunner<VT>::setup_resident() {
  res_cg = false;
  if (method != KS_CG || iprec == KS_FP64 || E32.comm || !E32.A || !E32.A->dia_nd) return;
  if (iprec == KS_FP32 ? !E32.A->dia_val32 : !E32.A->dia_val16) return;
  if (vec_count(KS_CG, E32.sp, E32.n, sizeof(float), ctx->l2_bytes) < 3) return;  // P (two slots) and r
  if (!ir_shape<float>(ctx, E32.n, &sh)) return;
  bool fits = false;
  const IrArgs none{};
  const cudaError_t e = iprec == KS_BF16 ? ir_launch<float, __nv_bfloat16>(ctx, *E32.A, none, sh, true, &fits, 0)
                                         : ir_launch<float, float>(ctx, *E32.A, none, sh, true, &fits, 0);
  if (e != cudaSuccess || !fits) {
    (void)cudaGetLastError();
    return;
  }
  // P in the first two slots (16-byte vector loads need their alignment),
  // between two zero pads wider than the largest offset for the stencil path
  Ws<float> W{ws32, E32.ld, E32.off};
  const long long pad = ir_p_pad(*E32.A);
  float *const preg = W.take(2);
  fb.stencil = ir_stencil_ok(*E32.A, E32.n) && 2 * E32.ld >= E32.n + 2 * pad ? 1 : 0;
  fb.P = preg + (fb.stencil ? pad : 0);
  fb.r = W.take();
  fb.x = z32;
  if (reinterpret_cast<uintptr_t>(fb.P) % 16) return;
  if (fb.stencil && (cudaMemsetAsync(preg, 0, sizeof(float) * pad, ctx->stream) != cudaSuccess ||
                     cudaMemsetAsync(fb.P + E32.n, 0, sizeof(float) * pad, ctx->stream) != cudaSuccess)) {
    (void)cudaGetLastError();
    return;
  }
  res_cg = true;
}

template <class VT>
void InnerRunner<VT>::solve(const VT *b, VT *z) {
  calls++;
  if (status != KS_OK) return;
  if constexpr (std::is_same<VT, double>::value) {
    if (iprec == KS_FP64) {
      status = run_method<double>(method, E64, b, z, ws64, dws, nullptr);
    } else if (res_cg) {
      const Stop os{nullptr, E32.outer_done};
      launch_vec(ctx, n, CgInStartOp<float>{b, fb.r, E32.st, E32.sp.eps, E32.sp.maxloop}, os);
      status = run_cg_inner_resident(E32, fb, sh);
      launch_vec(ctx, n, CgInFinalOp<float>{fb.x, E32.st, z, nullptr, nullptr, 0}, os);
    } else {
      launch_vec(ctx, n, ConvertOp<double, float>{b, b32}, Stop{nullptr, E32.outer_done});
      status = run_method<float>(method, E32, b32, z32, ws32, dws, nullptr);
      launch_vec(ctx, n, ConvertOp<float, double>{z32, z}, Stop{nullptr, E32.outer_done});
    }
  } else {
    status = KS_UNIMPLEMENTED;  // VP methods run their outer loop in FP64
  }
}

// ------------------------------------------------------------------ VPCG / VPCR
template <class VT>
struct RzOp {  // rr2 = (r, z); beta = rr2 / rr; rr = rr2   (vpcg.cpp:733-745)
  const VT *r;
  const VT *z;
  DevState *st;
  int init;  // 1: just rr = (r,z)
  static constexpr int ND = 1;
  struct Regs {
    VT r, z;
  };
  __device__ Regs load(long long i) const { return {r[i], z[i]}; }
  __device__ void store(long long, const Regs &g, double (&acc)[1]) const {
    acc[0] = add_rn(acc[0], mul_rn(widen(g.r), widen(g.z)));
  }
  __device__ void finish(const double (&s)[1]) const {
    if (!init) st->k.s[S_BETA] = rdiv(st, s[0], st->k.s[S_RR]);
    st->k.s[S_RR] = s[0];
  }
};

template <class VT>
ks_status run_vpcg(const Env<VT> &E, const VT *b, VT *x, VT *ws, double *dws, InnerRunner<VT> *inner) {
  // vpcg.cpp:659-750. With the on-chip inner CG its start is fused into the
  // outer x/r update and its end into (r, z); where the outer vectors do not
  // fit in L2 (defer_x, CG's rule) x += alpha p is deferred to a ring of
  // directions, as in run_cg: the x/r update then reads and writes neither x
  // nor p, and x gets the same bits.
  bool fast = false;
  if constexpr (std::is_same<VT, double>::value) fast = inner->res_cg;
  const bool defer = fast && defer_x(E, KS_CG);
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *z = W.take(), *mvv = W.take();
  const int D = defer ? dir_ring(E.sp) : 1;
  DirRing<VT> R{W.take(D), E.ld, D, dws};
  long long Lr = 1;  // ring position of the current direction (1 after each start)
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, nullptr, nullptr, nullptr, E.st, START_CHECK});
  // z = M r, rr = (r, z), p = z: the method's start, and its restart after a
  // failed true-residual check (r then holds b - A x)
  auto start = [&]() {
    if constexpr (std::is_same<VT, double>::value) {
      if (fast) {
        InnerRunner<double> &I = *inner;
        const Env<float> &F = I.E32;
        const Stop os{nullptr, F.outer_done};
        I.calls++;
        launch_vec(E.ctx, E.n, CgInStartOp<float>{r, I.fb.r, F.st, F.sp.eps, F.sp.maxloop}, os);
        if (I.status == KS_OK) I.status = run_cg_inner_resident(F, I.fb, I.sh);
        launch_vec(E.ctx, E.n, CgInFinalOp<float>{I.fb.x, F.st, z, r, E.st, 1}, os);
        Lr = 1;
        vec(E, CopyOp<VT>{z, R.slot(Lr)});
        return;
      }
    }
    inner->solve(r, z);
    Lr = 1;
    vec(E, CopyOp<VT>{z, R.slot(Lr)});
    vec(E, RzOp<VT>{r, z, E.st, 1});
  };
  auto iteration = [&]() {
    VT *p = R.slot(Lr);
    mv(E, *E.A, (const VT *)p, CgMvEpi<VT>{p, mvv, E.st});
    if constexpr (std::is_same<VT, double>::value) {
      if (fast) {
        InnerRunner<double> &I = *inner;
        const Env<float> &F = I.E32;
        I.calls++;
        if (defer) {
          vec(E, VpRStartOp<float>{r, mvv, E.st, I.fb.r, F.st, F.sp.eps, F.sp.maxloop, R.aslot(Lr)});
          ring_step(E, R, x, Lr);  // before the next direction overwrites the first slot
        } else {
          vec(E, VpXrStartOp<float>{x, r, p, mvv, E.st, I.fb.r, F.st, F.sp.eps, F.sp.maxloop});
        }
        if (I.status == KS_OK) I.status = run_cg_inner_resident(F, I.fb, I.sh);
        launch_vec(E.ctx, E.n, CgInFinalOp<float>{I.fb.x, F.st, nullptr, r, E.st, 2},
                   Stop{nullptr, F.outer_done});
        VT *pn = defer ? R.slot(Lr + 1) : p;
        vec(E, XpbyInOp<float>{p, I.fb.x, F.st, &E.st->k.s[S_BETA], pn});
        Lr++;
        return;
      }
    }
    vec(E, XrUpdOp<VT>{x, r, p, mvv, E.st, 1});
    inner->solve(r, z);
    vec(E, RzOp<VT>{r, z, E.st, 0});
    vec(E, XpbyOp<VT>{p, z, &E.st->k.s[S_BETA]});
  };
  start();
  long long issued = 0;
  for (;;) {
    Poller P{E.ctx, E.hflag, E.lookahead};
    while (issued < E.sp.maxloop) {
      iteration();
      issued++;
      if (P.step()) break;
    }
    if (defer) ring_final(E, R, x);  // the check reads x
    if (!true_check_continue(E, b, x, r)) break;
    if (issued >= E.sp.maxloop) {
      true_check_exhausted(E);
      break;
    }
    start();
  }
  return KS_OK;
}

template <class VT>
struct VpcrMvEpi {  // Av = A z; zaz(2) = (z, Av); init: Ap = Av, alpha from (Ap,Ap)
  using acc_t = VT;
  const VT *z;
  VT *Av;
  VT *Ap;  // set on init
  DevState *st;
  int init;
  static constexpr int ND = 2;
  __device__ void row(int i, VT v, double (&acc)[2]) const {
    Av[i] = v;
    if (init) Ap[i] = v;
    acc[0] = add_rn(acc[0], mul_rn(widen(z[i]), widen(v)));
    acc[1] = add_rn(acc[1], mul_rn(widen(v), widen(v)));
  }
  __device__ void finish(const double (&s)[2]) const {
    if (init) {
      st->k.s[S_RR] = s[0];
      st->k.s[S_ALPHA] = rdiv(st, s[0], s[1]);
    } else {
      st->k.s[S_BETA] = rdiv(st, s[0], st->k.s[S_RR]);
      st->k.s[S_RR] = s[0];
    }
  }
};

template <class VT>
ks_status run_vpcr(const Env<VT> &E, const VT *b, VT *x, VT *ws, InnerRunner<VT> *inner) {
  Ws<VT> W{ws, E.ld, E.off};
  VT *r = W.take(), *p = W.take(), *z = W.take(), *Av = W.take(), *Ap = W.take();
  init_state(E, b);
  vec(E, ZeroOp<VT>{x});
  start_from_zero(E, StartEpi<VT>{b, r, nullptr, nullptr, nullptr, E.st, START_CHECK});
  // vpcr.cpp:670-775; start() also restarts after a failed true-residual check
  auto start = [&]() {
    inner->solve(r, z);
    vec(E, CopyOp<VT>{z, p});
    mv(E, *E.A, (const VT *)z, VpcrMvEpi<VT>{z, Av, Ap, E.st, 1});
  };
  start();
  long long issued = 0;
  for (;;) {
    Poller P{E.ctx, E.hflag, E.lookahead};
    while (issued < E.sp.maxloop) {
      vec(E, XrUpdOp<VT>{x, r, p, Ap, E.st, 1});
      inner->solve(r, z);
      mv(E, *E.A, (const VT *)z, VpcrMvEpi<VT>{z, Av, nullptr, E.st, 0});
      vec(E, Xpby2Op<VT>{p, z, Ap, Av, E.st, 1});
      issued++;
      if (P.step()) break;
    }
    if (!true_check_continue(E, b, x, r)) break;
    if (issued >= E.sp.maxloop) {
      true_check_exhausted(E);
      break;
    }
    start();
  }
  return KS_OK;
}

template <class IT>
ks_status run_method(int method, const Env<IT> &E, const IT *b, IT *x, IT *ws, double *dws,
                     InnerRunner<IT> *inner) {
  switch (method) {
    case KS_CG: return run_cg(E, b, x, ws, dws);
    case KS_CR: return run_cr(E, b, x, ws, dws);
    case KS_BICG: return run_bicg(E, b, x, ws, dws);
    case KS_GCR: return run_gcr_core(E, b, x, ws, dws, (InnerRunner<IT> *)nullptr);
    case KS_GMRES: return run_gmres_core(E, b, x, ws, dws, (InnerRunner<IT> *)nullptr);
    case KS_KSKIPCG: return run_kskipcg(E, b, x, ws, dws);
    case KS_KSKIPBICG: return run_kskipbicg(E, b, x, ws, dws);
  }
  if constexpr (std::is_same<IT, double>::value) {
    switch (method) {
      case KS_VPCG: return run_vpcg(E, b, x, ws, dws, inner);
      case KS_VPCR: return run_vpcr(E, b, x, ws, inner);
      case KS_VPGCR: return run_gcr_core(E, b, x, ws, dws, inner);
      case KS_VPGMRES: return run_gmres_core(E, b, x, ws, dws, inner);
    }
  }
  return set_error(E.ctx, KS_UNIMPLEMENTED, "method not implemented");
}

static bool is_vp(int m) { return m == KS_VPCG || m == KS_VPCR || m == KS_VPGCR || m == KS_VPGMRES; }
static bool is_inner_ok(int m) {
  return m == KS_CG || m == KS_CR || m == KS_GCR || m == KS_BICG || m == KS_GMRES || m == KS_KSKIPCG ||
         m == KS_KSKIPBICG;
}
static bool needs_T(int m) { return m == KS_BICG || m == KS_KSKIPBICG; }

struct Alloc {  // RAII for pool buffers
  ks_ctx *ctx;
  std::vector<void *> bufs;
  ~Alloc() {
    for (void *p : bufs) pool_release(ctx, p);
  }
  template <class T>
  ks_status get(size_t count, T **out) {
    void *p = nullptr;
    KS_TRY(pool_get(ctx, sizeof(T) * std::max<size_t>(count, 1) + 256, &p));
    bufs.push_back(p);
    *out = (T *)p;
    return KS_OK;
  }
};

// out[0] = |x - y|^2, out[1] = |y|^2 (the report's x_rel_diff).
struct DiffNormOp {
  const double *x;
  const double *y;
  double *out;
  static constexpr int ND = 2;
  struct Regs {
    double x, y;
  };
  __device__ Regs load(long long i) const { return {x[i], y[i]}; }
  __device__ void store(long long, const Regs &g, double (&acc)[2]) const {
    const double d = sub_rn(g.x, g.y);
    acc[0] = add_rn(acc[0], mul_rn(d, d));
    acc[1] = add_rn(acc[1], mul_rn(g.y, g.y));
  }
  __device__ void finish(const double (&s)[2]) const {
    out[0] = s[0];
    out[1] = s[1];
  }
};

__global__ void k_copy_state(const DevState *st, long long *out) {
  out[0] = st->k.done;
  out[1] = st->k.loop;
  out[2] = st->k.hlen;
  out[3] = st->k.aux[A_CONVK];
  out[4] = (long long)st->k.s[S_TRUECNT];
}

}  // namespace ks

using namespace ks;

static ks_status solve_impl(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                            const ks_params *prm, const double *b, double *x, int64_t *hist_iter,
                            double *hist_err, int64_t hist_cap, ks_report *rep) {
  if (outer == KS_KSKIPCR || outer == KS_VPBICG)
    return set_error(ctx, KS_UNIMPLEMENTED, "Not implemented (as in the reference)");
  const bool vp = is_vp(outer);
  if (!vp && !is_inner_ok(outer)) return set_error(ctx, KS_BAD_INPUT, "unknown outer solver");
  if (vp && !is_inner_ok(inner))
    return set_error(ctx, KS_BAD_INPUT, "VP methods need an inner solver (cg cr gcr bicg gmres kskipcg kskipbicg)");
  const bool trans = prm->transpose != 0;
  const bool need_T = needs_T(outer) || (vp && needs_T(inner)) || trans;
  if (need_T && !mat->has_T)
    return set_error(ctx, KS_BAD_INPUT, "this method needs the transpose (upload with KS_MAT_TRANSPOSE)");
  const CsrDev *A = trans ? &mat->T : &mat->A;
  const CsrDev *AT = trans ? &mat->A : (mat->has_T ? &mat->T : &mat->A);
  const ks_precision ip = vp ? (ks_precision)prm->inner_precision : KS_FP64;
  if (ip == KS_FP32 && !A->val32) return set_error(ctx, KS_BAD_INPUT, "FP32 inner solve needs KS_MAT_FP32");
  if (ip == KS_BF16 && !A->val16) return set_error(ctx, KS_BAD_INPUT, "BF16 inner solve needs KS_MAT_BF16");
  if (ip != KS_FP64 && needs_T(inner) && !(ip == KS_FP32 ? (const void *)AT->val32 : (const void *)AT->val16))
    return set_error(ctx, KS_BAD_INPUT, "low-precision inner BiCG needs the transpose's value copy");

  Params outer_sp{prm->outer_maxloop, prm->outer_eps, prm->outer_restart, prm->outer_kskip, prm->outer_fix,
                  prm->x_update, prm->cluster_solve};
  Params inner_sp{prm->inner_maxloop, prm->inner_eps, prm->inner_restart, prm->inner_kskip, prm->inner_fix,
                  prm->x_update, prm->cluster_solve};
  if (prm->x_update < 0 || prm->x_update > 2) return set_error(ctx, KS_BAD_INPUT, "x_update must be 0, 1 or 2");
  if (prm->cluster_solve < 0 || prm->cluster_solve > 1)
    return set_error(ctx, KS_BAD_INPUT, "cluster_solve must be 0 or 1");
  if (prm->inner_fast < 0 || prm->inner_fast > 1) return set_error(ctx, KS_BAD_INPUT, "inner_fast must be 0 or 1");
  if (prm->true_residual < 0 || prm->true_residual > 2)
    return set_error(ctx, KS_BAD_INPUT, "true_residual must be 0, 1 or 2");
  if (prm->profile < 0 || prm->profile > 1) return set_error(ctx, KS_BAD_INPUT, "profile must be 0 or 1");
  if ((outer == KS_GCR || outer == KS_GMRES || outer == KS_VPGCR || outer == KS_VPGMRES) &&
      (outer_sp.restart < 1 || outer_sp.restart > 1024))
    return set_error(ctx, KS_BAD_INPUT, "restart must be in [1, 1024]");
  if (vp && (inner == KS_GCR || inner == KS_GMRES) && (inner_sp.restart < 1 || inner_sp.restart > 1024))
    return set_error(ctx, KS_BAD_INPUT, "inner restart must be in [1, 1024]");
  if (outer_sp.kskip < 0 || outer_sp.kskip > 100 || inner_sp.kskip < 0 || inner_sp.kskip > 100)
    return set_error(ctx, KS_BAD_INPUT, "kskip must be in [0, 100]");

  KS_CUDA(ctx, cudaSetDevice(ctx->device));
  const long long n = A->n;
  const DistInfo *dist = mat->dist;
  const long long ld = dist ? dist->ld() : n, off = dist ? dist->off() : 0;
  Alloc al{ctx, {}};
  // A row-split solve sums every reduction over the ranks while it runs.
  struct SplitScope {
    ks_ctx *c;
    SplitScope(ks_ctx *c_, ks_comm *comm) : c(c_) {
      c->red_comm = comm;
      c->dist_status = KS_OK;
    }
    ~SplitScope() {
      c->red_comm = nullptr;
      c->poll_done = nullptr;
    }
  } scope(ctx, dist ? dist->comm : nullptr);
  // device state (outer, inner) and history
  DevState *st = nullptr, *ist = nullptr;
  KS_TRY(al.get(2, &st));
  ist = st + 1;
  const long long hcap = std::max<long long>(1, std::min<long long>(outer_sp.maxloop + 2, 1LL << 26));
  double *d_hist = nullptr;
  long long *d_hit = nullptr;
  KS_TRY(al.get(hcap, &d_hist));
  KS_TRY(al.get(hcap, &d_hit));
  {
    DevState h[2];
    std::memset(h, 0, sizeof(h));
    h[0].k.hist_err = d_hist;
    h[0].k.hist_it = d_hit;
    h[0].k.hcap = hcap;
    h[0].host_done = nullptr;
    int *mapped = nullptr;
    if (cudaHostGetDevicePointer((void **)&mapped, ctx->h_flags, 0) == cudaSuccess) h[0].host_done = mapped;
    else (void)cudaGetLastError();
    KS_CUDA(ctx, cudaMemcpyAsync(st, h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->h_flags[0] = 0;

  // workspaces
  double *ws = nullptr, *dws = nullptr;
  KS_TRY(al.get((size_t)(vec_count(outer, outer_sp, n, sizeof(double), ctx->l2_bytes) * ld), &ws));
  double *xs = x;  // a split solve works on a windowed copy of x (restarts multiply x)
  if (dist) {
    KS_TRY(al.get((size_t)ld, &xs));
    xs += off;
  }
  ctx->poll_done = &st->k.done;
  KS_TRY(al.get((size_t)dws_count(outer, outer_sp), &dws));

  Env<double> E;
  E.ctx = ctx;
  E.A = A;
  E.AT = AT;
  E.mvals = KS_FP64;
  E.st = st;
  E.record = true;
  E.outer = true;
  E.sp = outer_sp;
  E.faithful = prm->reference_defects != 0;
  E.n = n;
  E.ld = ld;
  E.off = off;
  if (dist) {
    E.comm = dist->comm;
    E.planA = trans ? &dist->planT : &dist->planA;
    E.planT = trans ? &dist->planA : &dist->planT;
  }
  E.hflag = (volatile int *)ctx->h_flags;
  E.true_check = vp && (prm->true_residual == 1 || (prm->true_residual == 0 && ip != KS_FP64));
  E.lookahead = prm->poll_interval > 0 ? prm->poll_interval : (vp ? 2 : 8);
  E.lookahead = std::min(E.lookahead, ctx->nflags - 1);  // event ring size
  if (!ctx->h_flags || !st) return KS_CUDA_ERROR;

  InnerRunner<double> IR;
  if (vp) {
    IR.ctx = ctx;
    IR.method = inner;
    IR.iprec = ip;
    IR.n = n;
    KS_TRY(al.get((size_t)dws_count(inner, inner_sp), &IR.dws));
    if (ip == KS_FP64) {
      Env<double> &I = IR.E64;
      I = E;
      I.st = ist;
      I.outer_done = &st->k.done;
      I.record = false;
      I.outer = false;
      I.sp = inner_sp;
      I.hflag = nullptr;
      KS_TRY(al.get((size_t)(vec_count(inner, inner_sp, n, sizeof(double), ctx->l2_bytes) * ld), &IR.ws64));
    } else {
      Env<float> &I = IR.E32;
      I.ctx = ctx;
      I.A = A;
      I.AT = AT;
      I.mvals = ip;
      I.st = ist;
      I.outer_done = &st->k.done;
      I.record = false;
      I.outer = false;
      I.sp = inner_sp;
      I.faithful = E.faithful;
      I.n = n;
      I.ld = ld;
      I.off = off;
      I.comm = E.comm;
      I.planA = E.planA;
      I.planT = E.planT;
      I.hflag = nullptr;
      KS_TRY(al.get((size_t)(vec_count(inner, inner_sp, n, sizeof(float), ctx->l2_bytes) * ld), &IR.ws32));
      KS_TRY(al.get((size_t)ld, &IR.b32));
      KS_TRY(al.get((size_t)ld, &IR.z32));
      IR.b32 += off;
      IR.z32 += off;
      if (prm->inner_fast == 0) IR.setup_resident();
    }
  }

  // per-class device times (ks_params.profile)
  struct ProfScope {
    ks_ctx *c;
    ProfScope(ks_ctx *c_, bool on) : c(c_) {
      c->prof_on = on ? 1 : 0;
      c->prof_class.clear();
    }
    ~ProfScope() { c->prof_on = 0; }
  } prof(ctx, prm->profile == 1);
  KS_CUDA(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
  ctx->ir_used = false;
  ks_status s = run_method<double>(outer, E, b, xs, ws, dws, vp ? &IR : nullptr);
  if (s == KS_OK && vp) s = IR.status;
  if (ctx->ir_used) {
    ir_l2_release(ctx, mat->A);
    if (mat->has_T) ir_l2_release(ctx, mat->T);
    ctx->ir_used = false;
  }
  KS_CUDA(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
  if (s == KS_OK && dist) {
    // true residual |b - A x| / |b| over all ranks (not gated by `done`: the
    // method has stopped by now), then x out of the window
    E.halo(*A, xs);
    launch_spmv<double, double>(ctx, *A, (const double *)xs, ResidEpi<double>{b, nullptr, ctx->d_result},
                                Stop{nullptr, nullptr});
    KS_CUDA(ctx, cudaMemcpyAsync(x, xs, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  if (s == KS_OK && ctx->dist_status != KS_OK) s = ctx->dist_status;
  if (s != KS_OK) {
    cudaStreamSynchronize(ctx->stream);
    return s;
  }
  KS_CUDA(ctx, cudaGetLastError());
  long long *d_out = nullptr;
  KS_TRY(al.get(5, &d_out));
  k_copy_state<<<1, 1, 0, ctx->stream>>>(st, d_out);
  long long hs[5];
  KS_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, d_out, sizeof(hs), cudaMemcpyDeviceToHost, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memcpy(hs, ctx->h_pinned, sizeof(hs));
  KS_TRY(check_device_error(ctx));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  const int done = (int)hs[0];
  ks_status st_code = KS_NOT_CONVERGED;
  if (done == kConverged) st_code = KS_OK;
  else if (done == kBreakdown) st_code = KS_BREAKDOWN;
  else if (done == kNaN) st_code = KS_NAN_DETECTED;
  long long loop = hs[1];
  // reported "loop =" values (cg.cpp:246, gmres.cpp:427, kskipcg.cpp:314, kskipbicg.cpp:356)
  const int kk = outer_sp.kskip;
  if (outer == KS_GMRES || outer == KS_VPGMRES) {
    loop = loop + 1;
  } else if (outer == KS_KSKIPCG || outer == KS_KSKIPBICG) {
    long long nl = loop;
    if (done != kConverged) {  // ran out: nloop is the first multiple of k+1 >= maxloop
      nl = ((outer_sp.maxloop + kk) / (kk + 1)) * (kk + 1);
      if (outer_sp.maxloop <= 0) nl = 0;
    }
    loop = (outer == KS_KSKIPCG) ? nl - kk + 1 : nl + 1;
  } else if (outer == KS_GCR || outer == KS_VPGCR) {
    // loop as the device left it
  } else if (done == kMaxLoop || done == kRunning) {
    loop = outer_sp.maxloop + 1;
  }
  const long long hlen = hs[2];
  if (hist_err && hist_cap > 0) {
    const long long cnt = std::min<long long>(std::min<long long>(hlen, hcap), hist_cap);
    if (cnt > 0) {
      KS_CUDA(ctx, cudaMemcpy(hist_err, d_hist, sizeof(double) * cnt, cudaMemcpyDeviceToHost));
      if (hist_iter) KS_CUDA(ctx, cudaMemcpy(hist_iter, d_hit, sizeof(long long) * cnt, cudaMemcpyDeviceToHost));
    }
  }
  if (rep) {
    rep->status = st_code;
    rep->loop = loop;
    rep->hist_len = hlen;
    rep->final_rel_res = 0.0;
    if (hlen > 0 && hlen <= hcap) {
      double last = 0.0;
      KS_CUDA(ctx, cudaMemcpy(&last, d_hist + hlen - 1, sizeof(double), cudaMemcpyDeviceToHost));
      rep->final_rel_res = last;
    }
    rep->solve_seconds = ms * 1e-3;
    rep->inner_iterations = vp ? IR.calls : 0;
    rep->spmv_count = 0;
    rep->true_res_log10 = 0.0;
    rep->true_rel_res = 0.0;
    rep->x_rel_diff = -1.0;
    rep->true_residual_checks = hs[4];
    rep->t_mv = rep->t_dot = rep->t_other = rep->t_memset = rep->t_h2d = rep->t_d2h = rep->t_mv_low = 0.0;
    rep->n_mv = rep->n_dot = rep->n_other = rep->n_memset = rep->n_mv_low = 0;
    if (prm->profile == 1) {  // the stream is synchronised: every event has completed
      double t[kNumClasses] = {0, 0, 0, 0, 0};
      long long c[kNumClasses] = {0, 0, 0, 0, 0};
      for (size_t i = 0; i < ctx->prof_class.size(); i++) {
        float ms = 0.f;
        const int k = ctx->prof_class[i];
        c[k]++;
        if (cudaEventElapsedTime(&ms, ctx->prof_events[2 * i], ctx->prof_events[2 * i + 1]) == cudaSuccess)
          t[k] += ms * 1e-3;
        else
          (void)cudaGetLastError();
      }
      rep->t_mv = t[kMv] + t[kMvLow];
      rep->t_dot = t[kDot];
      rep->t_other = t[kOther];
      rep->t_memset = t[kMemset];
      rep->n_mv = c[kMv] + c[kMvLow];
      rep->n_dot = c[kDot];
      rep->n_other = c[kOther];
      rep->n_memset = c[kMemset];
      rep->t_mv_low = t[kMvLow];
      rep->n_mv_low = c[kMvLow];
    }
    if (prm->x_ref && !dist) {  // |x - x_ref| / |x_ref| over the solution
      launch_vec(ctx, n, DiffNormOp{x, prm->x_ref, ctx->d_result}, Stop{nullptr, nullptr});
      KS_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_result, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                   ctx->stream));
      KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      const double s2[2] = {ctx->h_pinned[0], ctx->h_pinned[1]};
      rep->x_rel_diff = s2[1] > 0.0 ? std::sqrt(s2[0]) / std::sqrt(s2[1]) : (s2[0] > 0.0 ? INFINITY : 0.0);
    }
    if (dist) {  // summed over the ranks after the solve
      double s2[2];
      KS_CUDA(ctx, cudaMemcpy(s2, ctx->d_result, sizeof(s2), cudaMemcpyDeviceToHost));
      rep->true_rel_res = std::sqrt(s2[0]) / std::sqrt(s2[1]);
      rep->true_res_log10 = std::log10(rep->true_rel_res);
    }
  }
  return st_code;
}

// Host containers (the workspace list, the buffer pool) can throw; no
// exception leaves a C entry point.
template <class F>
static ks_status solve_no_throw(ks_ctx *ctx, F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return set_error(ctx, KS_OUT_OF_MEMORY, "host allocation failed");
  } catch (...) {
    return set_error(ctx, KS_BAD_INPUT, "host container size out of range");
  }
}

static ks_status solve_entry(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                             const ks_params *params, const ks_vec *b, ks_vec *x, int64_t *hist_iter,
                             double *hist_err, int64_t hist_cap, ks_report *report);
static ks_status solve_host_entry(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                                  const ks_params *params, const double *b, double *x, int64_t *hist_iter,
                                  double *hist_err, int64_t hist_cap, ks_report *report);

extern "C" {

void ks_params_default(ks_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->outer_maxloop = 10000;
  p->outer_eps = 1e-8;
  p->outer_restart = 1000;
  p->outer_kskip = 2;
  p->outer_fix = 2;
  p->inner_maxloop = 50;
  p->inner_eps = 1e-1;
  p->inner_restart = 1000;
  p->inner_kskip = 2;
  p->inner_fix = 2;
  p->inner_precision = KS_FP64;
  p->reference_defects = 0;
  p->transpose = 0;
  p->poll_interval = 0;
}

ks_status ks_solve(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                   const ks_params *params, const ks_vec *b, ks_vec *x, int64_t *hist_iter,
                   double *hist_err, int64_t hist_cap, ks_report *report) {
  if (!ctx) return KS_BAD_INPUT;
  return solve_no_throw(
      ctx, [&] { return solve_entry(ctx, mat, outer, inner, params, b, x, hist_iter, hist_err, hist_cap, report); });
}

ks_status ks_solve_host(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                        const ks_params *params, const double *b, double *x, int64_t *hist_iter,
                        double *hist_err, int64_t hist_cap, ks_report *report) {
  if (!ctx) return KS_BAD_INPUT;
  return solve_no_throw(ctx, [&] {
    return solve_host_entry(ctx, mat, outer, inner, params, b, x, hist_iter, hist_err, hist_cap, report);
  });
}

}  // extern "C"

static ks_status solve_entry(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                             const ks_params *params, const ks_vec *b, ks_vec *x, int64_t *hist_iter,
                             double *hist_err, int64_t hist_cap, ks_report *report) {
  if (!ctx || !mat || !b || !x || mat->ctx != ctx || b->ctx != ctx || x->ctx != ctx) return KS_BAD_INPUT;
  if (b->type != KS_FP64 || x->type != KS_FP64 || b->n != mat->A.n || x->n != mat->A.n)
    return set_error(ctx, KS_BAD_INPUT, "ks_solve: b and x must be FP64 vectors of length n");
  ks_params def;
  if (!params) {
    ks_params_default(&def);
    params = &def;
  }
  ks_status s = solve_impl(ctx, mat, outer, inner, params, (const double *)b->d, (double *)x->d, hist_iter,
                           hist_err, hist_cap, report);
  if (report && !mat->dist && (s == KS_OK || s == KS_NOT_CONVERGED || s == KS_BREAKDOWN || s == KS_NAN_DETECTED)) {
    double lg = 0, rel = 0;
    const ks_mat *m = mat;
    if (params->transpose) {
      // residual of A^T x = b
      launch_spmv<double, double>(ctx, m->T, (const double *)x->d,
                                  ResidEpi<double>{(const double *)b->d, nullptr, ctx->d_result},
                                  Stop{nullptr, nullptr});
      double sc[2];
      KS_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_result, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
      KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      rel = std::sqrt(ctx->h_pinned[0]) / std::sqrt(ctx->h_pinned[1]);
      lg = std::log10(rel);
    } else {
      ks_status c = ks_check_error(m, b, x, &lg, &rel);
      if (c != KS_OK) return c;
    }
    report->true_res_log10 = lg;
    report->true_rel_res = rel;
  }
  return s;
}

static ks_status solve_host_entry(ks_ctx *ctx, const ks_mat *mat, ks_solver outer, ks_solver inner,
                                  const ks_params *params, const double *b, double *x, int64_t *hist_iter,
                                  double *hist_err, int64_t hist_cap, ks_report *report) {
  if (!ctx || !mat || !b || !x || mat->ctx != ctx) return KS_BAD_INPUT;
  // b and x live in the context's buffer pool between calls: no device
  // allocation (and no synchronising free) per solve
  const long long n = mat->A.n;
  void *buf = nullptr;
  KS_TRY(pool_get(ctx, sizeof(double) * (size_t)(2 * n) + 256, &buf));
  ks_vec vb, vx;
  vb.ctx = vx.ctx = ctx;
  vb.n = vx.n = n;
  vb.type = vx.type = KS_FP64;
  vb.d = buf;
  vx.d = (char *)buf + ((sizeof(double) * (size_t)n + 255) / 256) * 256;
  // with params->profile the copies are timed too (the times report's H2D / D2H)
  const bool prof = params && params->profile == 1 && report;
  float up_ms = 0.f, down_ms = 0.f;
  if (prof) cudaEventRecord(ctx->ev_start, ctx->stream);
  ks_status r = ks_vec_upload(&vb, b);
  if (prof) {
    cudaEventRecord(ctx->ev_stop, ctx->stream);
    cudaEventSynchronize(ctx->ev_stop);
    cudaEventElapsedTime(&up_ms, ctx->ev_start, ctx->ev_stop);
  }
  if (r == KS_OK) {
    r = ks_solve(ctx, mat, outer, inner, params, &vb, &vx, hist_iter, hist_err, hist_cap, report);
    if (r == KS_OK || r == KS_NOT_CONVERGED || r == KS_BREAKDOWN || r == KS_NAN_DETECTED) {
      if (prof) cudaEventRecord(ctx->ev_start, ctx->stream);
      const ks_status d = ks_vec_download(&vx, x);
      if (prof) {
        cudaEventRecord(ctx->ev_stop, ctx->stream);
        cudaEventSynchronize(ctx->ev_stop);
        cudaEventElapsedTime(&down_ms, ctx->ev_start, ctx->ev_stop);
        report->t_h2d = up_ms * 1e-3;
        report->t_d2h = down_ms * 1e-3;
      }
      if (d != KS_OK) r = d;
    }
  }
  pool_release(ctx, buf);
  return r;
}

extern "C" {

ks_status ks_adjoint_grad(ks_ctx *ctx, const ks_mat *mat, ks_solver solver, ks_solver inner,
                          const ks_params *params, const ks_vec *x, const ks_vec *g, ks_vec *grad_b,
                          ks_vec *grad_val, ks_report *report) {
  if (!ctx || !mat || !x || !g || x->type != KS_FP64 || g->type != KS_FP64) return KS_BAD_INPUT;
  ks_params p;
  if (params) p = *params;
  else ks_params_default(&p);
  p.transpose = 1;
  ks_vec *lam = grad_b;
  ks_vec *own = nullptr;
  if (!lam) {
    KS_TRY(ks_vec_create(ctx, mat->A.n, KS_FP64, &own));
    lam = own;
  }
  ks_status s = ks_solve(ctx, mat, solver, inner, &p, g, lam, nullptr, nullptr, 0, report);
  if ((s == KS_OK || s == KS_NOT_CONVERGED) && grad_val) {
    ks_status q = ks_pattern_grad(mat, lam, x, grad_val);
    if (q != KS_OK) s = q;
  }
  if (own) ks_vec_destroy(own);
  return s;
}

}  // extern "C"
