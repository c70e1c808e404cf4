// Context, matrices, vectors and the primitive operations of the C ABI.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "ks_dist.cuh"
#include "ks_kernels.cuh"
#include "ks_ops.cuh"

namespace ks {

ks_status set_error(ks_ctx *ctx, ks_status s, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

ks_status cuda_fail(ks_ctx *ctx, cudaError_t e, const char *what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  (void)cudaGetLastError();  // clear a sticky launch error where possible
  ks_status s = (e == cudaErrorMemoryAllocation) ? KS_OUT_OF_MEMORY : KS_CUDA_ERROR;
  return set_error(ctx, s, msg);
}

int red_grid(const ks_ctx *ctx) { return ctx->num_sms * 4; }

ks_status check_device_error(ks_ctx *ctx) {
  int flag = 0;
  KS_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (flag) {
    KS_CUDA(ctx, cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
    return set_error(ctx, KS_TIMEOUT, "a bounded wait on a shared-memory staging barrier ran out");
  }
  return KS_OK;
}

ks_status pool_get(ks_ctx *ctx, size_t bytes, void **out) {
  bytes = std::max<size_t>(bytes, 256);
  int best = -1;
  for (size_t i = 0; i < ctx->pool.size(); i++) {
    if (ctx->pool_busy[i] || ctx->pool[i].second < bytes) continue;
    if (best < 0 || ctx->pool[i].second < ctx->pool[best].second) best = (int)i;
  }
  if (best >= 0) {
    ctx->pool_busy[best] = true;
    *out = ctx->pool[best].first;
    return KS_OK;
  }
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    // Free idle buffers and retry once.
    for (size_t i = 0; i < ctx->pool.size();) {
      if (!ctx->pool_busy[i]) {
        cudaFree(ctx->pool[i].first);
        ctx->pool.erase(ctx->pool.begin() + i);
        ctx->pool_busy.erase(ctx->pool_busy.begin() + i);
      } else {
        i++;
      }
    }
    (void)cudaGetLastError();
    e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(workspace)");
  }
  ctx->pool.push_back({p, bytes});
  ctx->pool_busy.push_back(true);
  *out = p;
  return KS_OK;
}

void pool_release(ks_ctx *ctx, void *p) {
  for (size_t i = 0; i < ctx->pool.size(); i++)
    if (ctx->pool[i].first == p) ctx->pool_busy[i] = false;
}

// ------------------------------------------------------------- row blocks
// Greedy CSR-Adaptive partition: a block takes consecutive rows while it has
// at most kRowsPerBlock rows and kNnzPerBlock nonzeros; a row longer than
// kNnzPerBlock forms a block of its own.
static std::vector<int> row_blocks(const int32_t *ptr, int n) {
  std::vector<int> rb;
  rb.reserve(n / 64 + 2);
  rb.push_back(0);
  int r = 0;
  while (r < n) {
    const int r0 = r;
    const long long j0 = ptr[r0];
    r = r0 + 1;
    if ((long long)ptr[r0 + 1] - j0 <= kNnzPerBlock) {
      while (r < n && r - r0 < kRowsPerBlock && (long long)ptr[r + 1] - j0 <= kNnzPerBlock) r++;
    }
    rb.push_back(r);
  }
  return rb;
}

// ------------------------------------------------------------- transpose
__global__ void k_col_count(const int *__restrict__ col, long long nnz, int *__restrict__ cnt) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nnz;
       j += (long long)gridDim.x * blockDim.x)
    atomicAdd(cnt + col[j], 1);
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive scan of `in` (n entries) into `out` (n+1 entries, out[n] = total),
// tile by tile; tile totals go to `sums`.
__global__ void k_scan_tiles(const int *__restrict__ in, int n, int *__restrict__ out,
                             long long *__restrict__ sums) {
  __shared__ long long sh[kScanThreads];
  const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  long long v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; q++) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    s += v[q];
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < kScanThreads; o <<= 1) {
    long long t = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  long long run = sh[threadIdx.x] - s;  // exclusive prefix of this thread
#pragma unroll
  for (int q = 0; q < kScanItems; q++) {
    if (base + q < n) out[base + q] = (int)run;
    run += v[q];
  }
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = sh[threadIdx.x];
}

__global__ void k_scan_sums(long long *sums, int ntiles) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    long long run = 0;
    for (int i = 0; i < ntiles; i++) {
      long long t = sums[i];
      sums[i] = run;
      run += t;
    }
    sums[ntiles] = run;
  }
}

__global__ void k_scan_add(int *out, int n, const long long *__restrict__ sums, int ntiles) {
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  for (int q = 0; q < kScanItems; q++) {
    const int idx = blockIdx.x * kScanTile + q * kScanThreads + threadIdx.x;
    if (idx < n) out[idx] += (int)sums[blockIdx.x];
  }
  if (i == 0) out[n] = (int)sums[ntiles];
}

__global__ void k_scatter_t(const int *__restrict__ ptr, const int *__restrict__ col,
                            const double *__restrict__ val, int n, int *__restrict__ cursor,
                            int *__restrict__ trow, double *__restrict__ tval) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (int j = ptr[r]; j < ptr[r + 1]; j++) {
      const int d = atomicAdd(cursor + col[j], 1);
      trow[d] = r;
      tval[d] = val[j];
    }
  }
}

// Within each column, order the entries by row (the scatter's atomics leave
// them in arrival order). Insertion sort per column: columns of sparse PDE
// matrices are short.
__global__ void k_sort_cols(const int *__restrict__ tptr, int n, int *__restrict__ trow,
                            double *__restrict__ tval) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const int a = tptr[c], b = tptr[c + 1];
    for (int i = a + 1; i < b; i++) {
      const int kr = trow[i];
      const double kv = tval[i];
      int j = i - 1;
      while (j >= a && trow[j] > kr) {
        trow[j + 1] = trow[j];
        tval[j + 1] = tval[j];
        j--;
      }
      trow[j + 1] = kr;
      tval[j + 1] = kv;
    }
  }
}

__global__ void k_to_f32(const double *__restrict__ a, float *__restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

__global__ void k_to_bf16(const double *__restrict__ a, __nv_bfloat16 *__restrict__ b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16_rn((float)a[i]);
}

// Checks every column index (cmin <= col < cmax) and stores col - row as
// int16 where it fits: flags |= 1 for a column out of range, |= 2 for an
// offset outside [-32768, 32767] (col16 is then discarded by the caller).
// Rows of a split solve store col - r0, so col - row is the global offset.
__global__ void k_col16(const int *__restrict__ ptr, const int *__restrict__ col, int n, long long cmin,
                        long long cmax, short *__restrict__ col16, int *flags) {
  int bad = 0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const int j1 = ptr[r + 1];
    for (int j = ptr[r]; j < j1; j++) {
      const int c = col[j];
      if (c < cmin || c >= cmax) {
        bad |= 1;
        continue;
      }
      const int d = c - (int)r;
      if (d < -32768 || d > 32767)
        bad |= 2;
      else if (col16)
        col16[j] = (short)d;
    }
  }
  if (bad) atomicOr(flags, bad);
}

// Diagonal copy (CsrDev::dia_*), pass 1: the distinct offsets col - row of
// the matrix, collected in a per-CTA set in shared memory and merged into the
// global set `offs` (kMaxDiag slots, kDiagEmpty where free). flags |= 1 for a
// row whose columns are not strictly increasing, |= 2 for more than kMaxDiag
// distinct offsets.
constexpr int kDiagEmpty = INT_MIN;

__device__ __forceinline__ bool diag_insert(int *set, int d) {
  for (int s = 0; s < kMaxDiag; s++) {
    int v = *(volatile int *)&set[s];
    if (v == kDiagEmpty) {
      v = atomicCAS(&set[s], kDiagEmpty, d);
      if (v == kDiagEmpty) return true;
    }
    if (v == d) return true;
  }
  return false;
}

__global__ void k_dia_scan(const int *__restrict__ ptr, const int *__restrict__ col, int n, int *offs, int *flags) {
  __shared__ int s_off[kMaxDiag];
  __shared__ int s_flags;
  if (threadIdx.x < kMaxDiag) s_off[threadIdx.x] = kDiagEmpty;
  if (threadIdx.x == 0) s_flags = 0;
  __syncthreads();
  int bad = 0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const int j0 = ptr[r], j1 = ptr[r + 1];
    int last = kDiagEmpty;
    for (int j = j0; j < j1; j++) {
      const int c = col[j];
      if (j > j0 && c <= col[j - 1]) bad |= 1;
      const int d = c - (int)r;
      if (d == last) continue;
      if (diag_insert(s_off, d))
        last = d;
      else
        bad |= 2;
    }
  }
  if (bad) atomicOr(&s_flags, bad);
  __syncthreads();
  if (threadIdx.x < kMaxDiag) {
    const int d = s_off[threadIdx.x];
    if (d != kDiagEmpty && !diag_insert(offs, d)) atomicOr(flags, 2);
  }
  if (threadIdx.x == 0 && s_flags) atomicOr(flags, s_flags);
}

struct DiagOffsets {
  int nd;
  int off[kMaxDiag];
};

// Pass 2: values diagonal-major (dval zeroed beforehand) and the row masks.
__global__ void k_dia_fill(const int *__restrict__ ptr, const int *__restrict__ col,
                           const double *__restrict__ val, int n, DiagOffsets o, double *__restrict__ dval,
                           unsigned char *__restrict__ mask) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    unsigned m = 0;
    for (int j = ptr[r]; j < ptr[r + 1]; j++) {
      const int d = col[j] - (int)r;
      for (int k = 0; k < o.nd; k++) {
        if (o.off[k] == d) {
          dval[(long long)k * n + r] = val[j];
          m |= 1u << k;
          break;
        }
      }
    }
    mask[r] = (unsigned char)m;
  }
}

// Pass 3: is the copy symmetric? For every lower diagonal d (offset -o) and
// its mirror u = nd - 1 - d (offset +o), row i's entry on d must equal row
// i - o's entry on u in presence and value, bit for bit (the zeros of absent
// entries compare equal); a row i < o has no entry on d. flag = 1 otherwise.
__global__ void k_dia_symcheck(const double *__restrict__ dval, const unsigned char *__restrict__ mask, int n,
                               DiagOffsets o, int *flag) {
  const int h = o.nd / 2;
  int bad = 0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    const unsigned m = mask[r];
    for (int d = 0; d < h; d++) {
      const int u = o.nd - 1 - d;
      const long long q = r + o.off[d];
      const unsigned has = (m >> d) & 1u;
      if (q < 0) {
        bad |= (int)has;
        continue;
      }
      const unsigned hu = (mask[q] >> u) & 1u;
      const long long a = __double_as_longlong(dval[(long long)d * n + r]);
      const long long b = __double_as_longlong(dval[(long long)u * n + q]);
      if (has != hu || a != b) bad = 1;
    }
  }
  if (bad) atomicOr(flag, 1);
}

static void free_dia(CsrDev &A) {
  cudaFree(A.dia_val);
  cudaFree(A.dia_val32);
  cudaFree(A.dia_val16);
  cudaFree(A.dia_mask);
  A.dia_val = nullptr;
  A.dia_val32 = nullptr;
  A.dia_val16 = nullptr;
  A.dia_mask = nullptr;
  A.dia_nd = 0;
  A.dia_sym = 0;
  A.dia_pad = 0;
  A.dia_ds = 0;
}

// Builds the diagonal copy when the matrix qualifies (CsrDev::dia_*); leaves
// dia_nd = 0 otherwise. Value copies follow the CSR ones (FP32, BF16). A
// matrix equal to its transpose (on one GPU: the copy must hold every row a
// lower diagonal reaches) keeps the symmetric half only.
static ks_status build_diagonals(ks_ctx *ctx, CsrDev &A, unsigned flags, long long cmin, long long cmax) {
  if (A.n < 1 || A.nnz < 1) return KS_OK;
  const int g = ctx->num_sms * 8;
  int *d_buf = nullptr;  // kMaxDiag offsets, then the flags
  KS_CUDA(ctx, cudaMalloc(&d_buf, sizeof(int) * (kMaxDiag + 1)));
  int h_buf[kMaxDiag + 1];
  for (int k = 0; k < kMaxDiag; k++) h_buf[k] = kDiagEmpty;
  h_buf[kMaxDiag] = 0;
  cudaError_t e = cudaMemcpyAsync(d_buf, h_buf, sizeof(h_buf), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    k_dia_scan<<<g, 256, 0, ctx->stream>>>(A.ptr, A.col, A.n, d_buf, d_buf + kMaxDiag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h_buf, d_buf, sizeof(h_buf), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(d_buf);
    return cuda_fail(ctx, e, "diagonal scan");
  }
  DiagOffsets o{};
  for (int k = 0; k < kMaxDiag; k++)
    if (h_buf[k] != kDiagEmpty) o.off[o.nd++] = h_buf[k];
  std::sort(o.off, o.off + o.nd);
  // unordered rows, too many diagonals, or diagonals less than 3/4 full: CSR only
  if (h_buf[kMaxDiag] || o.nd < 1 || 4 * A.nnz < 3LL * o.nd * A.n) {
    cudaFree(d_buf);
    return KS_OK;
  }
  const long long len = (long long)o.nd * A.n;
  // The copy is an optimisation: if the device cannot hold it, CSR serves.
  auto got = [&](cudaError_t a) {
    if (a == cudaSuccess) return true;
    (void)cudaGetLastError();
    free_dia(A);
    return false;
  };
  // + 8 elements of tail: 4-row vector loads of the last diagonal's last rows
  if (!got(cudaMalloc(&A.dia_val, sizeof(double) * (size_t)(len + 8))) ||
      !got(cudaMalloc(&A.dia_mask, (size_t)A.n + 8))) {
    cudaFree(d_buf);
    return KS_OK;
  }
  KS_CUDA(ctx, cudaMemsetAsync(A.dia_val, 0, sizeof(double) * (size_t)(len + 8), ctx->stream));
  KS_CUDA(ctx, cudaMemsetAsync(A.dia_mask, 0, (size_t)A.n + 8, ctx->stream));
  k_dia_fill<<<g, 256, 0, ctx->stream>>>(A.ptr, A.col, A.val, A.n, o, A.dia_val, A.dia_mask);
  KS_CUDA(ctx, cudaGetLastError());
  // symmetric half storage
  const int h = o.nd / 2;
  bool sym = (o.nd & 1) && o.off[h] == 0 && cmin == 0 && cmax == A.n && h > 0;
  for (int k = 0; sym && k < h; k++) sym = o.off[k] == -o.off[o.nd - 1 - k];
  if (sym) {
    int flag = 0;
    e = cudaMemsetAsync(d_buf, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) {
      k_dia_symcheck<<<g, 256, 0, ctx->stream>>>(A.dia_val, A.dia_mask, A.n, o, d_buf);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, d_buf, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      cudaFree(d_buf);
      return cuda_fail(ctx, e, "diagonal symmetry check");
    }
    sym = flag == 0;
  }
  cudaFree(d_buf);
  long long ds = A.n, stored = len + 8;
  int pad = 0;
  if (sym) {
    // the lower diagonals' reads start up to -off[0] rows before row 0; the
    // pad and the stride are whole multiples of 4 elements with 4 to spare
    // either side, so 4-row vector loads of any diagonal stay inside the copy
    // and aligned
    pad = ((-o.off[0] + 3) / 4) * 4 + 4;
    ds = ((long long)pad + A.n + 3) / 4 * 4 + 8;
    stored = (long long)(h + 1) * ds;
    double *sv = nullptr;
    if (cudaMalloc(&sv, sizeof(double) * (size_t)stored) == cudaSuccess) {
      KS_CUDA(ctx, cudaMemsetAsync(sv, 0, sizeof(double) * (size_t)stored, ctx->stream));
      for (int j = 0; j <= h; j++)
        KS_CUDA(ctx, cudaMemcpyAsync(sv + (long long)j * ds + pad, A.dia_val + (long long)(h + j) * A.n,
                                     sizeof(double) * (size_t)A.n, cudaMemcpyDeviceToDevice, ctx->stream));
      KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      cudaFree(A.dia_val);
      A.dia_val = sv;
    } else {  // no room for the half copy next to the full one: keep the full one
      (void)cudaGetLastError();
      sym = false;
      ds = A.n;
      stored = len + 8;
      pad = 0;
    }
  }
  if ((flags & KS_MAT_FP32) && !got(cudaMalloc(&A.dia_val32, sizeof(float) * (size_t)stored))) return KS_OK;
  if ((flags & KS_MAT_BF16) && !got(cudaMalloc(&A.dia_val16, sizeof(__nv_bfloat16) * (size_t)stored))) return KS_OK;
  if (A.dia_val32) k_to_f32<<<g, 256, 0, ctx->stream>>>(A.dia_val, A.dia_val32, stored);
  if (A.dia_val16) k_to_bf16<<<g, 256, 0, ctx->stream>>>(A.dia_val, A.dia_val16, stored);
  KS_CUDA(ctx, cudaGetLastError());
  A.dia_nd = o.nd;
  for (int k = 0; k < kMaxDiag; k++) A.dia_off[k] = k < o.nd ? o.off[k] : 0;
  A.dia_cmin = (int)cmin;
  A.dia_cmax = (int)cmax;
  A.dia_sym = sym ? 1 : 0;
  A.dia_pad = pad;
  A.dia_ds = ds;
  return KS_OK;
}

static void free_csr(CsrDev &A) {
  free_dia(A);
  cudaFree(A.ptr);
  cudaFree(A.col);
  cudaFree(A.col16);
  cudaFree(A.val);
  cudaFree(A.val32);
  cudaFree(A.val16);
  cudaFree(A.rb);
  cudaFree(A.rbi);
  A = CsrDev();
}

// col/val carry kPad tail elements and ptr kPad tail entries (zeroed) so the
// 16-byte-granular bulk copies of a row block's arrays stay inside them.
static ks_status alloc_csr(ks_ctx *ctx, CsrDev &A, int n, long long nnz) {
  A.n = n;
  A.nnz = nnz;
  KS_CUDA(ctx, cudaMalloc(&A.ptr, sizeof(int) * (size_t)(n + 1 + kPad)));
  KS_CUDA(ctx, cudaMemsetAsync(A.ptr + n + 1, 0, sizeof(int) * kPad, ctx->stream));
  KS_CUDA(ctx, cudaMalloc(&A.col, sizeof(int) * (size_t)(nnz + kPad)));
  KS_CUDA(ctx, cudaMalloc(&A.val, sizeof(double) * (size_t)(nnz + kPad)));
  KS_CUDA(ctx, cudaMemsetAsync(A.col + nnz, 0, sizeof(int) * kPad, ctx->stream));
  KS_CUDA(ctx, cudaMemsetAsync(A.val + nnz, 0, sizeof(double) * kPad, ctx->stream));
  return KS_OK;
}

static ks_status finish_csr(ks_ctx *ctx, CsrDev &A, const int32_t *host_ptr, unsigned flags, long long cmin = 0,
                            long long cmax = -1) {
  if (cmax < 0) cmax = A.n;
  std::vector<int> rb = row_blocks(host_ptr, A.n);
  A.nrb = (int)rb.size() - 1;
  KS_CUDA(ctx, cudaMalloc(&A.rb, sizeof(int) * rb.size()));
  KS_CUDA(ctx, cudaMemcpyAsync(A.rb, rb.data(), sizeof(int) * rb.size(), cudaMemcpyHostToDevice,
                               ctx->stream));
  std::vector<int4> rbi((size_t)A.nrb);
  for (int b = 0; b < A.nrb; b++) rbi[b] = make_int4(rb[b], rb[b + 1], host_ptr[rb[b]], host_ptr[rb[b + 1]]);
  KS_CUDA(ctx, cudaMalloc(&A.rbi, sizeof(int4) * std::max<size_t>(rbi.size(), 1)));
  KS_CUDA(ctx, cudaMemcpyAsync(A.rbi, rbi.data(), sizeof(int4) * rbi.size(), cudaMemcpyHostToDevice,
                               ctx->stream));
  const long long tot = A.nnz + kPad;
  const int g = ctx->num_sms * 8;
  {
    if (!(flags & KS_MAT_INDEX32)) {
      KS_CUDA(ctx, cudaMalloc(&A.col16, sizeof(short) * (size_t)tot));
      KS_CUDA(ctx, cudaMemsetAsync(A.col16 + A.nnz, 0, sizeof(short) * kPad, ctx->stream));
    }
    int *d_flags = nullptr, h_flags = 0;
    KS_CUDA(ctx, cudaMalloc(&d_flags, sizeof(int)));
    cudaError_t e = cudaMemsetAsync(d_flags, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) {
      k_col16<<<g, 256, 0, ctx->stream>>>(A.ptr, A.col, A.n, cmin, cmax, A.col16, d_flags);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_flags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_flags);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "column index check");
    if (h_flags & 1) return set_error(ctx, KS_BAD_INPUT, "column index out of range");
    if (h_flags & 2) {
      cudaFree(A.col16);
      A.col16 = nullptr;
    }
  }
  if (flags & KS_MAT_FP32) {
    KS_CUDA(ctx, cudaMalloc(&A.val32, sizeof(float) * (size_t)tot));
    k_to_f32<<<g, 256, 0, ctx->stream>>>(A.val, A.val32, tot);
  }
  if (flags & KS_MAT_BF16) {
    KS_CUDA(ctx, cudaMalloc(&A.val16, sizeof(__nv_bfloat16) * (size_t)tot));
    k_to_bf16<<<g, 256, 0, ctx->stream>>>(A.val, A.val16, tot);
  }
  KS_CUDA(ctx, cudaGetLastError());
  if (!(flags & KS_MAT_NO_DIAG)) KS_TRY(build_diagonals(ctx, A, flags, cmin, cmax));
  // rb and rbi are host vectors going out of scope: the copies must complete first.
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return KS_OK;
}

static ks_status build_transpose(ks_ctx *ctx, ks_mat *m) {
  CsrDev &A = m->A;
  CsrDev &T = m->T;
  const int n = A.n;
  KS_TRY(alloc_csr(ctx, T, n, A.nnz));
  int *cnt = nullptr, *cursor = nullptr;
  long long *sums = nullptr;
  const int ntiles = (n + kScanTile - 1) / kScanTile;
  KS_CUDA(ctx, cudaMalloc(&cnt, sizeof(int) * (size_t)(n + 1)));
  KS_CUDA(ctx, cudaMalloc(&cursor, sizeof(int) * (size_t)(n + 1)));
  KS_CUDA(ctx, cudaMalloc(&sums, sizeof(long long) * (size_t)(ntiles + 1)));
  KS_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(n + 1), ctx->stream));
  const int g = ctx->num_sms * 8;
  k_col_count<<<g, 256, 0, ctx->stream>>>(A.col, A.nnz, cnt);
  k_scan_tiles<<<std::max(ntiles, 1), kScanThreads, 0, ctx->stream>>>(cnt, n, T.ptr, sums);
  k_scan_sums<<<1, 32, 0, ctx->stream>>>(sums, ntiles);
  k_scan_add<<<std::max(ntiles, 1), kScanThreads, 0, ctx->stream>>>(T.ptr, n, sums, ntiles);
  KS_CUDA(ctx, cudaMemcpyAsync(cursor, T.ptr, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToDevice,
                               ctx->stream));
  k_scatter_t<<<g, 256, 0, ctx->stream>>>(A.ptr, A.col, A.val, n, cursor, T.col, T.val);
  k_sort_cols<<<g, 256, 0, ctx->stream>>>(T.ptr, n, T.col, T.val);
  KS_CUDA(ctx, cudaGetLastError());
  std::vector<int32_t> tptr((size_t)n + 1);
  KS_CUDA(ctx, cudaMemcpyAsync(tptr.data(), T.ptr, sizeof(int) * (size_t)(n + 1),
                               cudaMemcpyDeviceToHost, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(cnt);
  cudaFree(cursor);
  cudaFree(sums);
  KS_TRY(finish_csr(ctx, T, tptr.data(), m->flags));
  m->has_T = true;
  return KS_OK;
}

static ks_status check_csr(ks_ctx *ctx, int64_t n, int64_t nnz, const int32_t *ptr,
                           const int32_t *col) {
  if (n < 1 || n >= (1LL << 31) - 1 || nnz < 0 || nnz >= (1LL << 31) - 1)
    return set_error(ctx, KS_BAD_INPUT, "n and nnz must fit the int32 CSR format (n >= 1)");
  if (ptr) {
    if (ptr[0] != 0 || ptr[n] != nnz)
      return set_error(ctx, KS_BAD_INPUT, "ptr[0] must be 0 and ptr[n] must equal nnz");
    for (int64_t i = 0; i < n; i++)
      if (ptr[i + 1] < ptr[i]) return set_error(ctx, KS_BAD_INPUT, "ptr must be non-decreasing");
  }
  if (col) {
    for (int64_t j = 0; j < nnz; j++)
      if (col[j] < 0 || col[j] >= n) return set_error(ctx, KS_BAD_INPUT, "column index out of range");
  }
  return KS_OK;
}

// ------------------------------------------------------------- primitive kernels
__global__ void k_copy_bytes_done(const int *src, int *dst) { *dst = *src; }

}  // namespace ks

using namespace ks;

// ============================================================= C ABI: context
// Host containers (std::vector, new) can throw; no exception leaves a C
// entry point: running out of host memory is KS_OUT_OF_MEMORY, any other
// exception (a size no container can hold) KS_BAD_INPUT.
template <class F>
static ks_status no_throw(F &&f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return KS_OUT_OF_MEMORY;
  } catch (...) {
    return KS_BAD_INPUT;
  }
}

extern "C" {

int ks_abi_version(void) { return KS_ABI_VERSION; }

int ks_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return n;
}

const char *ks_status_string(ks_status s) {
  switch (s) {
    case KS_OK: return "converged / ok";
    case KS_NOT_CONVERGED: return "not converged (maxloop reached)";
    case KS_BREAKDOWN: return "breakdown (zero Krylov denominator)";
    case KS_NAN_DETECTED: return "non-finite scalar in the recurrence";
    case KS_BAD_INPUT: return "bad input";
    case KS_CUDA_ERROR: return "CUDA error";
    case KS_TIMEOUT: return "bounded device wait timed out";
    case KS_OUT_OF_MEMORY: return "out of device memory";
    case KS_NO_DEVICE: return "no CUDA device";
    case KS_IO_ERROR: return "CRS file error";
    case KS_UNIMPLEMENTED: return "not implemented";
  }
  return "unknown status";
}

const char *ks_last_error(const ks_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int64_t ks_ctx_launches(const ks_ctx *ctx) { return ctx ? ctx->launches : 0; }

ks_status ks_ctx_create(int device, ks_ctx **out) {
  if (!out) return KS_BAD_INPUT;
  *out = nullptr;
  int ndev = ks_device_count();
  if (ndev <= 0) return KS_NO_DEVICE;
  if (device < 0 || device >= ndev) return KS_BAD_INPUT;
  ks_ctx *ctx = new (std::nothrow) ks_ctx();
  if (!ctx) return KS_OUT_OF_MEMORY;
  ctx->device = device;
  auto fail = [&](ks_status s) {
    ks_ctx_destroy(ctx);
    return s;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(KS_CUDA_ERROR);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(KS_CUDA_ERROR);
  ctx->num_sms = prop.multiProcessorCount;
  ctx->l2_bytes = (size_t)prop.l2CacheSize;
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(KS_CUDA_ERROR);
  ctx->stream = ctx->own_stream;
  ctx->partials_len = (size_t)kMaxGroups * kBlockDotGroup * (size_t)std::max(red_grid(ctx), ctx->num_sms * 8);
  if (cudaMalloc(&ctx->partials, sizeof(double) * ctx->partials_len) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  ctx->ncounters = kMaxGroups + 64;
  if (cudaMalloc(&ctx->counters, sizeof(unsigned) * ctx->ncounters) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  if (cudaMemset(ctx->counters, 0, sizeof(unsigned) * ctx->ncounters) != cudaSuccess)
    return fail(KS_CUDA_ERROR);
  if (cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess) return fail(KS_OUT_OF_MEMORY);
  if (cudaMemset(ctx->d_err, 0, sizeof(int)) != cudaSuccess) return fail(KS_CUDA_ERROR);
  ctx->d_result_len = 4096;
  if (cudaMalloc(&ctx->d_result, sizeof(double) * ctx->d_result_len) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  ctx->h_pinned_len = 4096;
  if (cudaMallocHost(&ctx->h_pinned, sizeof(double) * ctx->h_pinned_len) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  ctx->nflags = 64;
  if (cudaHostAlloc(&ctx->h_flags, sizeof(int) * ctx->nflags,
                    cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  std::memset(ctx->h_flags, 0, sizeof(int) * ctx->nflags);
  if (cudaHostAlloc(&ctx->h_snap, sizeof(int) * ctx->nflags, cudaHostAllocMapped | cudaHostAllocPortable) !=
          cudaSuccess ||
      cudaHostGetDevicePointer((void **)&ctx->d_snap, ctx->h_snap, 0) != cudaSuccess)
    return fail(KS_OUT_OF_MEMORY);
  std::memset(ctx->h_snap, 0, sizeof(int) * ctx->nflags);
  if (cudaMalloc(&ctx->d_stage, sizeof(double) * kStageLen) != cudaSuccess) return fail(KS_OUT_OF_MEMORY);
  // barrier state of the on-chip inner CG: 32 bytes + one flag per SM
  if (cudaMalloc(&ctx->ir_sync, 64 + 8 * (size_t)ctx->num_sms) != cudaSuccess) return fail(KS_OUT_OF_MEMORY);
  ctx->flag_events = new cudaEvent_t[ctx->nflags];
  for (int i = 0; i < ctx->nflags; i++) {
    if (cudaEventCreateWithFlags(&ctx->flag_events[i], cudaEventDisableTiming) != cudaSuccess)
      return fail(KS_CUDA_ERROR);
  }
  if (cudaEventCreate(&ctx->ev_start) != cudaSuccess || cudaEventCreate(&ctx->ev_stop) != cudaSuccess)
    return fail(KS_CUDA_ERROR);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(KS_CUDA_ERROR);
  *out = ctx;
  return KS_OK;
}

ks_status ks_ctx_destroy(ks_ctx *ctx) {
  if (!ctx) return KS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &b : ctx->pool) cudaFree(b.first);
  ctx->pool.clear();
  cudaFree(ctx->partials);
  cudaFree(ctx->counters);
  cudaFree(ctx->d_result);
  cudaFree(ctx->d_err);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  if (ctx->h_flags) cudaFreeHost(ctx->h_flags);
  if (ctx->h_snap) cudaFreeHost(ctx->h_snap);
  cudaFree(ctx->d_stage);
  if (ctx->flag_events) {
    for (int i = 0; i < ctx->nflags; i++)
      if (ctx->flag_events[i]) cudaEventDestroy(ctx->flag_events[i]);
    delete[] ctx->flag_events;
  }
  for (cudaEvent_t e : ctx->prof_events) cudaEventDestroy(e);
  cudaFree(ctx->ir_sync);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return KS_OK;
}

ks_status ks_ctx_set_wait_limit(ks_ctx *ctx, int64_t ns) {
  if (!ctx) return KS_BAD_INPUT;
  const int64_t cap = 10000000000LL;  // 10 s
  ctx->wait_ns = ns <= 0 ? kWaitLimitNs : (unsigned long long)std::min<int64_t>(ns, cap);
  return KS_OK;
}

ks_status ks_mat_dia_symmetric(const ks_mat *m, int *a_sym, int *t_sym) {
  if (!m) return KS_BAD_INPUT;
  if (a_sym) *a_sym = m->A.dia_sym;
  if (t_sym) *t_sym = m->has_T ? m->T.dia_sym : 0;
  return KS_OK;
}

ks_status ks_ctx_set_stream(ks_ctx *ctx, void *stream) {
  if (!ctx) return KS_BAD_INPUT;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return KS_OK;
}

ks_status ks_ctx_synchronize(ks_ctx *ctx) {
  if (!ctx) return KS_BAD_INPUT;
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);  // a bounded wait of a queued kernel that ran out
}

// ============================================================= C ABI: matrices
static ks_status upload_common(ks_ctx *ctx, int64_t n, int64_t nnz, const int32_t *ptr,
                               const int32_t *col, const double *val, unsigned flags, ks_mat **out,
                               cudaMemcpyKind kind) {
  if (!ctx || !out || !ptr || (nnz > 0 && (!col || !val))) return KS_BAD_INPUT;
  *out = nullptr;
  KS_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<int32_t> hptr;
  const int32_t *host_ptr = ptr;
  if (kind == cudaMemcpyHostToDevice) {
    KS_TRY(check_csr(ctx, n, nnz, ptr, col));
  } else {
    KS_TRY(check_csr(ctx, n, nnz, nullptr, nullptr));
    hptr.resize((size_t)n + 1);
    KS_CUDA(ctx, cudaMemcpy(hptr.data(), ptr, sizeof(int32_t) * (size_t)(n + 1), cudaMemcpyDeviceToHost));
    KS_TRY(check_csr(ctx, n, nnz, hptr.data(), nullptr));
    host_ptr = hptr.data();
  }
  ks_mat *m = new ks_mat();
  m->ctx = ctx;
  m->flags = flags;
  ks_status s = alloc_csr(ctx, m->A, (int)n, nnz);
  if (s == KS_OK) {
    cudaError_t e = cudaMemcpyAsync(m->A.ptr, ptr, sizeof(int) * (size_t)(n + 1), kind, ctx->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->A.col, col, sizeof(int) * (size_t)nnz, kind, ctx->stream);
    if (e == cudaSuccess && nnz > 0)
      e = cudaMemcpyAsync(m->A.val, val, sizeof(double) * (size_t)nnz, kind, ctx->stream);
    if (e != cudaSuccess) s = cuda_fail(ctx, e, "csr upload");
  }
  if (s == KS_OK) s = finish_csr(ctx, m->A, host_ptr, flags);
  if (s == KS_OK && (flags & KS_MAT_TRANSPOSE)) s = build_transpose(ctx, m);
  if (s != KS_OK) {
    ks_mat_destroy(m);
    return s;
  }
  *out = m;
  return KS_OK;
}

ks_status ks_csr_upload(ks_ctx *ctx, int64_t n, int64_t nnz, const int32_t *ptr, const int32_t *col,
                        const double *val, unsigned flags, ks_mat **out) {
  return no_throw([&] { return upload_common(ctx, n, nnz, ptr, col, val, flags, out, cudaMemcpyHostToDevice); });
}

ks_status ks_csr_upload_device(ks_ctx *ctx, int64_t n, int64_t nnz, const int32_t *d_ptr,
                               const int32_t *d_col, const double *d_val, unsigned flags,
                               ks_mat **out) {
  return no_throw(
      [&] { return upload_common(ctx, n, nnz, d_ptr, d_col, d_val, flags, out, cudaMemcpyDeviceToDevice); });
}

ks_status ks_mat_destroy(ks_mat *m) {
  if (!m) return KS_OK;
  if (m->ctx) {
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
  }
  free_csr(m->A);
  free_csr(m->T);
  delete m->dist;
  delete m;
  return KS_OK;
}

ks_status ks_mat_info(const ks_mat *m, int64_t *n, int64_t *nnz, int64_t *row_blocks) {
  if (!m) return KS_BAD_INPUT;
  if (n) *n = m->A.n;
  if (nnz) *nnz = m->A.nnz;
  if (row_blocks) *row_blocks = m->A.nrb;
  return KS_OK;
}

// ============================================================= C ABI: split rows
// Uploads one rank's rows of a row-split matrix (global column indices) and,
// for BiCG-type methods, the same rows of A^T; exchanges every rank's rows
// and windows once to build the halo plans.
static ks_status upload_rows(ks_ctx *ctx, CsrDev &A, long long nloc, const int32_t *ptr, const int32_t *col,
                             const double *val, long long r0, long long lo, long long hi, unsigned flags) {
  const long long j0 = ptr[0], nnz = ptr[nloc] - j0;
  std::vector<int32_t> lp((size_t)nloc + 1), lc((size_t)nnz);
  for (long long i = 0; i <= nloc; i++) lp[(size_t)i] = (int32_t)(ptr[i] - j0);
  for (long long j = 0; j < nnz; j++) lc[(size_t)j] = (int32_t)(col[j] - r0);
  KS_TRY(alloc_csr(ctx, A, (int)nloc, nnz));
  KS_CUDA(ctx, cudaMemcpyAsync(A.ptr, lp.data(), sizeof(int) * (size_t)(nloc + 1), cudaMemcpyHostToDevice, ctx->stream));
  if (nnz > 0) {
    KS_CUDA(ctx, cudaMemcpyAsync(A.col, lc.data(), sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, ctx->stream));
    KS_CUDA(ctx, cudaMemcpyAsync(A.val, val, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, ctx->stream));
  }
  return finish_csr(ctx, A, lp.data(), flags, lo - r0, hi - r0);  // synchronises: lp, lc may go
}

static ks_status plan_of(ks_ctx *ctx, const std::vector<long long> &all, int P, int rank, int lo_i, HaloPlan &plan) {
  std::vector<int64_t> rs((size_t)P + 1), lo((size_t)P), hi((size_t)P), sl(P), sh(P), rl(P), rh(P);
  for (int q = 0; q < P; q++) {
    rs[(size_t)q] = all[(size_t)q * 6 + 0];
    lo[(size_t)q] = all[(size_t)q * 6 + lo_i];
    hi[(size_t)q] = all[(size_t)q * 6 + lo_i + 1];
  }
  rs[(size_t)P] = all[(size_t)(P - 1) * 6 + 1];
  const ks_status s = ks_halo_plan(P, rank, rs.data(), lo.data(), hi.data(), sl.data(), sh.data(), rl.data(), rh.data());
  if (s != KS_OK) return set_error(ctx, s, "halo plan: windows do not cover the rows");
  plan.row_start.assign(rs.begin(), rs.end());
  plan.peer.resize((size_t)P);
  for (int q = 0; q < P; q++) plan.peer[(size_t)q] = HaloRange{sl[q], sh[q], rl[q], rh[q]};
  return KS_OK;
}

static ks_status dist_upload(ks_ctx *ctx, ks_comm *comm, int64_t n_global, int64_t r0, int64_t r1,
                             const int32_t *ptr, const int32_t *col, const double *val, const int32_t *tptr,
                             const int32_t *tcol, const double *tval, unsigned flags, ks_mat **out);

ks_status ks_dist_upload(ks_ctx *ctx, ks_comm *comm, int64_t n_global, int64_t r0, int64_t r1, const int32_t *ptr,
                         const int32_t *col, const double *val, const int32_t *tptr, const int32_t *tcol,
                         const double *tval, unsigned flags, ks_mat **out) {
  return no_throw([&] { return dist_upload(ctx, comm, n_global, r0, r1, ptr, col, val, tptr, tcol, tval, flags, out); });
}

static ks_status dist_upload(ks_ctx *ctx, ks_comm *comm, int64_t n_global, int64_t r0, int64_t r1,
                             const int32_t *ptr, const int32_t *col, const double *val, const int32_t *tptr,
                             const int32_t *tcol, const double *tval, unsigned flags, ks_mat **out) {
  if (!ctx || !comm || !out || !ptr || comm->ctx != ctx) return KS_BAD_INPUT;
  *out = nullptr;
  const bool want_t = (flags & KS_MAT_TRANSPOSE) != 0;
  if (want_t && !tptr) return set_error(ctx, KS_BAD_INPUT, "split rows with KS_MAT_TRANSPOSE need the rows of A^T");
  if (n_global < 1 || n_global >= (1LL << 31) - 1 || r0 < 0 || r1 < r0 || r1 > n_global)
    return set_error(ctx, KS_BAD_INPUT, "split rows: need 0 <= r0 <= r1 <= n_global < 2^31 - 1");
  const long long nloc = r1 - r0;
  auto check_rows = [&](const int32_t *p, const int32_t *c, const double *v) -> ks_status {
    for (long long i = 0; i < nloc; i++)
      if (p[i + 1] < p[i]) return set_error(ctx, KS_BAD_INPUT, "split rows: ptr must be non-decreasing");
    if (p[nloc] > p[0] && (!c || !v)) return KS_BAD_INPUT;
    for (long long j = 0; j < (long long)p[nloc] - p[0]; j++)
      if (c[j] < 0 || c[j] >= n_global) return set_error(ctx, KS_BAD_INPUT, "column index out of range");
    return KS_OK;
  };
  KS_CUDA(ctx, cudaSetDevice(ctx->device));
  KS_TRY(check_rows(ptr, col, val));
  if (want_t) KS_TRY(check_rows(tptr, tcol, tval));
  // every rank's rows and windows: r0 r1 lo hi tlo thi
  int64_t lo = r0, hi = r1, tlo = r0, thi = r1;
  KS_TRY(ks_halo_window(r0, r1, ptr, col, &lo, &hi));
  if (want_t) KS_TRY(ks_halo_window(r0, r1, tptr, tcol, &tlo, &thi));
  const long long mine[6] = {r0, r1, lo, hi, tlo, thi};
  std::vector<long long> all((size_t)comm->nranks * 6);
  KS_TRY(comm->allgather_host(mine, 6, all.data()));
  const int P = comm->nranks;
  if (all[0] != 0 || all[(size_t)(P - 1) * 6 + 1] != n_global)
    return set_error(ctx, KS_BAD_INPUT, "split rows: the ranks' rows must cover 0..n_global in rank order");
  for (int q = 1; q < P; q++)
    if (all[(size_t)q * 6] != all[(size_t)(q - 1) * 6 + 1])
      return set_error(ctx, KS_BAD_INPUT, "split rows: the ranks' rows must be contiguous in rank order");
  auto *d = new DistInfo();
  d->comm = comm;
  d->n_global = n_global;
  d->r0 = r0;
  d->r1 = r1;
  d->lo = lo;
  d->hi = hi;
  d->tlo = tlo;
  d->thi = thi;
  d->ext_lo = std::min(lo, tlo);
  d->ext_hi = std::max(hi, thi);
  ks_mat *m = new ks_mat();
  m->ctx = ctx;
  m->flags = flags;
  m->dist = d;
  ks_status s = plan_of(ctx, all, P, comm->rank, 2, d->planA);
  if (s == KS_OK && want_t) s = plan_of(ctx, all, P, comm->rank, 4, d->planT);
  if (s == KS_OK) s = upload_rows(ctx, m->A, nloc, ptr, col, val, r0, lo, hi, flags);
  if (s == KS_OK && want_t) {
    s = upload_rows(ctx, m->T, nloc, tptr, tcol, tval, r0, tlo, thi, flags);
    m->has_T = s == KS_OK;
  }
  if (s != KS_OK) {
    ks_mat_destroy(m);
    return s;
  }
  *out = m;
  return KS_OK;
}

ks_status ks_mat_dist_info(const ks_mat *m, int64_t *n_global, int64_t *r0, int64_t *r1, int64_t *ext_lo,
                           int64_t *ext_hi) {
  if (!m) return KS_BAD_INPUT;
  const DistInfo *d = m->dist;
  if (n_global) *n_global = d ? d->n_global : m->A.n;
  if (r0) *r0 = d ? d->r0 : 0;
  if (r1) *r1 = d ? d->r1 : m->A.n;
  if (ext_lo) *ext_lo = d ? d->ext_lo : 0;
  if (ext_hi) *ext_hi = d ? d->ext_hi : m->A.n;
  return KS_OK;
}

ks_status ks_mat_index_bytes(const ks_mat *m, int *a_bytes, int *t_bytes) {
  if (!m) return KS_BAD_INPUT;
  if (a_bytes) *a_bytes = m->A.col16 ? 2 : 4;
  if (t_bytes) *t_bytes = m->has_T ? (m->T.col16 ? 2 : 4) : 0;
  return KS_OK;
}

ks_status ks_mat_diagonals(const ks_mat *m, int *a_diagonals, int *t_diagonals) {
  if (!m) return KS_BAD_INPUT;
  if (a_diagonals) *a_diagonals = m->A.dia_nd;
  if (t_diagonals) *t_diagonals = m->has_T ? m->T.dia_nd : 0;
  return KS_OK;
}

ks_status ks_mat_transpose_download(const ks_mat *m, int32_t *tptr, int32_t *trow, double *tval) {
  if (!m || !m->has_T) return m ? set_error(m->ctx, KS_BAD_INPUT, "matrix has no transpose") : KS_BAD_INPUT;
  if (m->dist) return set_error(m->ctx, KS_UNIMPLEMENTED, "not available for split-row matrices");
  ks_ctx *ctx = m->ctx;
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (tptr) KS_CUDA(ctx, cudaMemcpy(tptr, m->T.ptr, sizeof(int) * (size_t)(m->T.n + 1), cudaMemcpyDeviceToHost));
  if (trow) KS_CUDA(ctx, cudaMemcpy(trow, m->T.col, sizeof(int) * (size_t)m->T.nnz, cudaMemcpyDeviceToHost));
  if (tval) KS_CUDA(ctx, cudaMemcpy(tval, m->T.val, sizeof(double) * (size_t)m->T.nnz, cudaMemcpyDeviceToHost));
  return KS_OK;
}

// ============================================================= C ABI: vectors
ks_status ks_vec_create(ks_ctx *ctx, int64_t n, ks_precision type, ks_vec **out) {
  if (!ctx || !out || n < 1 || type < KS_FP64 || type > KS_BF16) return KS_BAD_INPUT;
  *out = nullptr;
  KS_CUDA(ctx, cudaSetDevice(ctx->device));
  ks_vec *v = new (std::nothrow) ks_vec();
  if (!v) return KS_OUT_OF_MEMORY;
  v->ctx = ctx;
  v->n = n;
  v->type = type;
  v->owned = true;
  cudaError_t e = cudaMalloc(&v->d, elem_size(type) * (size_t)n + 64);
  if (e != cudaSuccess) {
    delete v;
    return cuda_fail(ctx, e, "cudaMalloc(vector)");
  }
  e = cudaMemsetAsync(v->d, 0, elem_size(type) * (size_t)n, ctx->stream);
  if (e != cudaSuccess) {
    cudaFree(v->d);
    delete v;
    return cuda_fail(ctx, e, "cudaMemset(vector)");
  }
  *out = v;
  return KS_OK;
}

ks_status ks_vec_wrap(ks_ctx *ctx, int64_t n, ks_precision type, void *device_ptr, ks_vec **out) {
  if (!ctx || !out || !device_ptr || n < 1 || type < KS_FP64 || type > KS_BF16) return KS_BAD_INPUT;
  if (((uintptr_t)device_ptr) % 16 != 0)
    return set_error(ctx, KS_BAD_INPUT, "wrapped device pointer must be 16-byte aligned");
  ks_vec *v = new (std::nothrow) ks_vec();
  if (!v) return KS_OUT_OF_MEMORY;
  v->ctx = ctx;
  v->n = n;
  v->type = type;
  v->d = device_ptr;
  v->owned = false;
  *out = v;
  return KS_OK;
}

ks_status ks_vec_destroy(ks_vec *v) {
  if (!v) return KS_OK;
  if (v->owned && v->d) {
    cudaSetDevice(v->ctx->device);
    cudaStreamSynchronize(v->ctx->stream);
    cudaFree(v->d);
  }
  delete v;
  return KS_OK;
}

ks_status ks_vec_upload_range(ks_vec *v, int64_t offset, int64_t count, const void *host) {
  if (!v || !host || offset < 0 || count < 0 || offset + count > v->n) return KS_BAD_INPUT;
  ks_ctx *ctx = v->ctx;
  const size_t es = elem_size(v->type);
  KS_CUDA(ctx, cudaMemcpyAsync((char *)v->d + es * offset, host, es * (size_t)count,
                               cudaMemcpyHostToDevice, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return KS_OK;
}

ks_status ks_vec_download_range(const ks_vec *v, int64_t offset, int64_t count, void *host) {
  if (!v || !host || offset < 0 || count < 0 || offset + count > v->n) return KS_BAD_INPUT;
  ks_ctx *ctx = v->ctx;
  const size_t es = elem_size(v->type);
  KS_CUDA(ctx, cudaMemcpyAsync(host, (const char *)v->d + es * offset, es * (size_t)count,
                               cudaMemcpyDeviceToHost, ctx->stream));
  KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return KS_OK;
}

ks_status ks_vec_upload(ks_vec *v, const void *host) {
  return v ? ks_vec_upload_range(v, 0, v->n, host) : KS_BAD_INPUT;
}

ks_status ks_vec_download(const ks_vec *v, void *host) {
  return v ? ks_vec_download_range(v, 0, v->n, host) : KS_BAD_INPUT;
}

ks_status ks_vec_fill(ks_vec *v, double value) {
  if (!v) return KS_BAD_INPUT;
  ks_ctx *ctx = v->ctx;
  if (v->type == KS_FP64)
    launch_vec(ctx, v->n, FillOp<double>{(double *)v->d, value}, Stop{nullptr, nullptr});
  else if (v->type == KS_FP32)
    launch_vec(ctx, v->n, FillOp<float>{(float *)v->d, (float)value}, Stop{nullptr, nullptr});
  else
    return set_error(ctx, KS_BAD_INPUT, "fill supports FP64 and FP32 vectors");
  KS_CUDA(ctx, cudaGetLastError());
  return KS_OK;
}

void *ks_vec_device_ptr(ks_vec *v) { return v ? v->d : nullptr; }
int64_t ks_vec_length(const ks_vec *v) { return v ? v->n : 0; }

}  // extern "C"
