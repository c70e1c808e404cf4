// Internal definitions shared by the kernel and host translation units.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "krylov_sm100.h"

namespace ks {

// ---------------------------------------------------------------- launch shape
constexpr int kThreads = 256;       // threads per CTA for every kernel here
constexpr int kRowsPerBlock = 256;  // rows staged by one SpMV row block
constexpr int kNnzPerBlock = 2048;  // nonzeros staged by one SpMV row block
constexpr int kChunk = 4;           // nonzeros per vectorised load (int4 cols)
constexpr int kPad = 8;             // tail padding of col/val arrays (elements)
constexpr int kMaxDots = 8;         // simultaneous reductions in one kernel
constexpr int kBlockDotGroup = 8;   // tall-skinny dots per pass
constexpr int kMaxGroups = 128;     // block-dot groups in one launch (1024 dots)
constexpr int kMaxDiag = 8;         // diagonals of a matrix's diagonal copy (8-bit row masks)

// ---------------------------------------------------------------- state
// Device-resident scalar state of one running Krylov method. Every scalar of
// the recurrences lives here; the host only reads `done` and the history.
enum DoneCode : int {
  kRunning = 0,
  kConverged = 1,
  kMaxLoop = 2,
  kBreakdown = 3,
  kNaN = 4,
};

struct KState {
  double s[96];          // named scalar slots (per method)
  int done;              // DoneCode
  int pad0;
  long long loop;        // the method's iteration counter
  long long hlen;        // history entries written
  long long hcap;        // history capacity
  long long aux[8];      // method-specific integers (e.g. GMRES step index)
  double *hist_err;      // device history arrays (capacity hcap)
  long long *hist_it;
};

// Stop predicate: a kernel does nothing once either flag is set. Used so a
// whole queued iteration turns into no-ops after convergence, and so inner
// solves of a VP method stop when the outer method has finished.
struct Stop {
  const int *a;
  const int *b;
  __device__ __forceinline__ bool operator()() const {
    return (a && *(volatile const int *)a) || (b && *(volatile const int *)b);
  }
};

// Reduction scratch: per-CTA partials plus a last-CTA-done counter.
struct Red {
  double *partials;     // [kMaxDots * kMaxGroups? ] x grid
  unsigned *counter;
};

// ---------------------------------------------------------------- matrices
struct CsrDev {
  int n = 0;
  long long nnz = 0;
  int *ptr = nullptr;
  int *col = nullptr;
  // Column indices as 16-bit offsets from the row (col - row), kept when every
  // offset fits in [-32768, 32767]; the SpMV then reads 2 bytes per column
  // instead of 4. Null when an offset does not fit or KS_MAT_INDEX32 is set.
  short *col16 = nullptr;
  double *val = nullptr;
  float *val32 = nullptr;
  __nv_bfloat16 *val16 = nullptr;
  int *rb = nullptr;  // row-block boundaries, nrb + 1 entries
  int4 *rbi = nullptr;  // per row block: first row, end row, first nonzero, end nonzero
  int nrb = 0;
  // Diagonal copy of a stencil-like matrix, read by the SpMV instead of the
  // CSR arrays: every row holds its columns at offsets (col - row) from a set
  // of dia_nd <= kMaxDiag offsets, dia_off ascending. Values are stored
  // diagonal-major, dia_val[d * dia_ds + i] (0 where row i has no entry on
  // diagonal d), and bit d of dia_mask[i] is set where it has one. Kept only
  // when every row lists its columns in increasing order (so a row summed
  // diagonal by diagonal is summed in its CSR order) and the diagonals are at
  // least 3/4 full; dia_nd = 0 otherwise or with KS_MAT_NO_DIAG.
  int dia_nd = 0;
  int dia_off[kMaxDiag] = {};
  int dia_cmin = 0, dia_cmax = 0;  // columns of x the diagonals may reach
  double *dia_val = nullptr;
  float *dia_val32 = nullptr;
  __nv_bfloat16 *dia_val16 = nullptr;
  unsigned char *dia_mask = nullptr;
  // Symmetric half storage (dia_sym = 1): when A equals its transpose bit for
  // bit (pattern and values; offsets symmetric about a main diagonal), only
  // the main diagonal and the upper diagonals are kept, dia_nd / 2 + 1 of
  // them, each of dia_ds = dia_pad + n elements: dia_pad leading zeros, then
  // row 0 .. n-1. Row i's entry on lower diagonal d (offset -o) is
  // A[i][i-o] = A[i-o][i], the upper mirror's element at row i - o, which
  // for i < o lands in the zero pad. dia_sym = 0: all dia_nd diagonals, each
  // of n elements (dia_ds = n, dia_pad = 0).
  int dia_sym = 0;
  int dia_pad = 0;
  long long dia_ds = 0;
};

template <class MT>
struct CsrK {
  const int *__restrict__ ptr;
  const int *__restrict__ col;
  const MT *__restrict__ val;
  const int *__restrict__ rb;
  int nrb;
  int n;
};

template <class MT>
inline CsrK<MT> view(const CsrDev &A);
template <>
inline CsrK<double> view<double>(const CsrDev &A) {
  return {A.ptr, A.col, A.val, A.rb, A.nrb, A.n};
}
template <>
inline CsrK<float> view<float>(const CsrDev &A) {
  return {A.ptr, A.col, A.val32, A.rb, A.nrb, A.n};
}
template <>
inline CsrK<__nv_bfloat16> view<__nv_bfloat16>(const CsrDev &A) {
  return {A.ptr, A.col, A.val16, A.rb, A.nrb, A.n};
}

// ---------------------------------------------------------------- arithmetic
// Round-to-nearest operations that the compiler may not contract into FMA:
// the reference's host loops (blas.cpp) round the product and the sum
// separately, and so do these.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

template <class T>
__device__ __forceinline__ T to(double v);
template <>
__device__ __forceinline__ double to<double>(double v) { return v; }
template <>
__device__ __forceinline__ float to<float>(double v) { return (float)v; }

__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ double widen(float v) { return (double)v; }
__device__ __forceinline__ float val_as_float(__nv_bfloat16 v) { return __bfloat162float(v); }

// Matrix value -> accumulation type.
template <class AT, class MT>
__device__ __forceinline__ AT mval(MT v) { return (AT)v; }
template <>
__device__ __forceinline__ float mval<float, __nv_bfloat16>(__nv_bfloat16 v) {
  return __bfloat162float(v);
}

// Hint: bring the line holding p into L2 (no register, no fault on use).
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// ---------------------------------------------------------------- PDL
// Programmatic dependent launch: every kernel lets the next one in the stream
// be scheduled at once (trigger) and waits for the previous one's results
// only where it needs them (wait). Both are no-ops for a kernel launched
// without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums of ND values; result valid in every thread. Fixed order, so
// deterministic for a fixed launch shape.
template <int ND>
__device__ __forceinline__ void block_sum(double (&v)[ND]) {
  __shared__ double sh[ND][kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; d++) v[d] = warp_sum(v[d]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < ND; d++) sh[d][wid] = v[d];
  }
  __syncthreads();
#pragma unroll
  for (int d = 0; d < ND; d++) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; w++) s += sh[d][w];
    v[d] = s;
  }
}

// Single-pass deterministic grid reduction (last CTA done) over G CTAs, this
// CTA being number `bid`. Every one of the G CTAs must call it exactly once.
// Returns true in all threads of the last CTA to arrive, which then holds the
// grand totals in `v`. No CTA waits on another: the last arriving CTA does the
// final sum in a fixed order, so there is no spin and the result does not
// depend on arrival order.
template <int ND>
__device__ __forceinline__ bool grid_sum_n(double (&v)[ND], double *partials,
                                           unsigned *counter, unsigned G,
                                           unsigned bid) {
  __shared__ bool is_last;
  block_sum<ND>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < ND; d++) partials[(size_t)d * G + bid] = v[d];
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    is_last = (prev == G - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  // Several loads in flight per thread; the order is still fixed. Few
  // values: four running sums per value. Many values (block dots): one
  // running sum per value, all values' loads of one round issued together.
  const unsigned B = blockDim.x;
  if constexpr (ND >= 4) {
#pragma unroll
    for (int d = 0; d < ND; d++) v[d] = 0.0;
    for (unsigned i = threadIdx.x; i < G; i += B) {
#pragma unroll
      for (int d = 0; d < ND; d++) v[d] += __ldcg(partials + (size_t)d * G + i);
    }
  } else {
#pragma unroll
    for (int d = 0; d < ND; d++) {
      const double *p = partials + (size_t)d * G;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      unsigned i = threadIdx.x;
      for (; i + 3 * B < G; i += 4 * B) {
        s0 += __ldcg(p + i);
        s1 += __ldcg(p + i + B);
        s2 += __ldcg(p + i + 2 * B);
        s3 += __ldcg(p + i + 3 * B);
      }
      for (; i < G; i += B) s0 += __ldcg(p + i);
      v[d] = (s0 + s1) + (s2 + s3);
    }
  }
  block_sum<ND>(v);
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// Last-CTA detection without sums (a kernel that only needs one thread to run
// a scalar step after every CTA has finished its stores).
__device__ __forceinline__ bool grid_last(unsigned *counter) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned G = gridDim.x * gridDim.y;
    is_last = atomicAdd(counter, 1u) == G - 1;
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

template <int ND>
__device__ __forceinline__ bool grid_sum(double (&v)[ND], double *partials,
                                         unsigned *counter) {
  return grid_sum_n<ND>(v, partials, counter, gridDim.x * gridDim.y,
                        blockIdx.y * gridDim.x + blockIdx.x);
}


}  // namespace ks

// ---------------------------------------------------------------- handles
struct ks_ctx {
  int device = 0;
  int num_sms = 148;
  size_t l2_bytes = 0;  // L2 cache size of the device
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool ir_used = false;         // an on-chip CG kernel ran in this solve (ir_l2_release)
  double *partials = nullptr;   // reduction scratch
  size_t partials_len = 0;
  unsigned *counters = nullptr; // last-CTA-done counters
  int ncounters = 0;
  int *d_err = nullptr;         // set by a kernel whose bounded wait ran out
  unsigned long long wait_ns = 2000000000ull;  // limit of those waits (ks_ctx_set_wait_limit)
  double *d_result = nullptr;   // device staging for scalar results
  size_t d_result_len = 0;
  double *h_pinned = nullptr;   // pinned host staging (scalars)
  size_t h_pinned_len = 0;
  int *h_flags = nullptr;       // pinned ring of polled `done` flags
  int nflags = 0;
  cudaEvent_t *flag_events = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::vector<std::pair<void *, size_t>> pool;  // reusable device buffers
  std::vector<bool> pool_busy;
  std::string last_error;
  long long launches = 0;       // kernels launched (diagnostics)
  // Row-split solve in progress: its communicator (reductions are summed over
  // the ranks), the first transport error, the stage of the summed values,
  // and the outer method's `done` with a mapped snapshot ring for polling.
  struct ks_comm *red_comm = nullptr;
  ks_status dist_status = KS_OK;
  double *d_stage = nullptr;    // kStageLen doubles
  const int *poll_done = nullptr;
  int *h_snap = nullptr;        // mapped host ring (nflags entries)
  int *d_snap = nullptr;        // its device view
  // Per-class device time of a solve (ks_params.profile): every launch_k
  // records an event before and after its kernel and the class the launcher
  // set in next_class (ks::KernelClass; reset to kOther after each launch).
  void *ir_sync = nullptr;      // barrier state of the on-chip inner CG (ks_inner_resident.cuh)
  int prof_on = 0;
  int next_class = 0;
  std::vector<cudaEvent_t> prof_events;  // pool, reused across solves
  std::vector<unsigned char> prof_class;  // class of recorded launch i
};

namespace ks {
constexpr int kStageLen = 4096;  // >= 2 x 1024 block-dot results, >= kMaxDots
// Kernel classes of the times report (times.cpp:60-76).
// kMvLow: an SpMV reading FP32 / BF16 values (reported within kMv too).
enum KernelClass : int { kOther = 0, kMv = 1, kDot = 2, kMemset = 3, kMvLow = 4, kNumClasses = 5 };
}

namespace ks {
struct DistInfo;  // ks_dist.cuh
}

struct ks_mat {
  ks_ctx *ctx = nullptr;
  ks::CsrDev A;
  ks::CsrDev T;
  bool has_T = false;
  unsigned flags = 0;
  ks::DistInfo *dist = nullptr;  // rows of a split solve; null on one GPU
};

struct ks_vec {
  ks_ctx *ctx = nullptr;
  long long n = 0;
  ks_precision type = KS_FP64;
  void *d = nullptr;
  bool owned = false;
};

namespace ks {

inline size_t elem_size(ks_precision t) {
  return t == KS_FP64 ? 8 : (t == KS_FP32 ? 4 : 2);
}

// Error plumbing for host code.
ks_status set_error(ks_ctx *ctx, ks_status s, const std::string &msg);
ks_status cuda_fail(ks_ctx *ctx, cudaError_t e, const char *what);

#define KS_CUDA(ctx, call)                                   \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return ::ks::cuda_fail((ctx), _e, #call); \
  } while (0)

#define KS_TRY(...)                    \
  do {                                 \
    ks_status _s = (__VA_ARGS__);      \
    if (_s != KS_OK) return _s;        \
  } while (0)

// Scratch sizing.
int red_grid(const ks_ctx *ctx);  // CTAs of the vector kernels
// Reads and clears the context's timeout flag (synchronises the stream).
ks_status check_device_error(ks_ctx *ctx);

// Workspace pool (device buffers reused across solves).
ks_status pool_get(ks_ctx *ctx, size_t bytes, void **out);
void pool_release(ks_ctx *ctx, void *p);

}  // namespace ks
