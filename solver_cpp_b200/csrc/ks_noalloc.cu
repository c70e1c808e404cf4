// Allocation-free variant of the tall-skinny block dot.
//
// Some callers cannot allocate device memory at the moment they need this
// operation: code running while a CUDA stream is being captured into a graph
// (cudaMalloc is not a stream operation and is not allowed there), host
// applications that hand all device memory to their own pool allocator at
// start-up and forbid further cudaMalloc, and latency-critical loops that must
// not hit the driver allocator (cudaMalloc/cudaFree can synchronise the
// device). ks_block_dot_noalloc serves them: the caller passes the inputs and
// the output, and the only scratch it needs -- the per-CTA partial sums and the
// last-CTA-done counters of the grid reduction -- lives in one file-scope
// device array of fixed size, resident on every GPU that loads the library
// until the process exits. Nothing here calls cudaMalloc, cudaFree or any
// allocating routine.
#include <cstdio>
#include <mutex>

#include "ks_ops.cuh"

namespace ks {

constexpr int kNoAllocMaxK = KS_NOALLOC_MAX_K;                   // basis vectors per call
constexpr int kNoAllocGroups = kNoAllocMaxK / kBlockDotGroup;   // 8 groups of 8 dots
constexpr int kNoAllocGrid = 296;                               // CTAs per group (2 per SM)
constexpr size_t kNoAllocPartials = (size_t)kNoAllocGroups * kBlockDotGroup * kNoAllocGrid;
constexpr size_t kNoAllocCounterOffset = kNoAllocPartials * sizeof(double);  // multiple of 256
constexpr size_t kNoAllocBytes = kNoAllocCounterOffset + 256;   // 151,808 bytes

static_assert(kNoAllocMaxK % kBlockDotGroup == 0, "whole groups");
static_assert(kNoAllocCounterOffset % 256 == 0, "counters stay aligned");

// The scratch: partial sums (doubles) followed by one counter per group.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device. The array's name in host
// code is only a handle; the address a kernel may use comes from
// cudaGetSymbolAddress, taken once per device with that device current.
static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[64] = {nullptr};

static ks_status noalloc_scratch(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return KS_NO_DEVICE;
  }
  if (dev < 0 || dev >= 64) return KS_BAD_INPUT;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      std::fprintf(stderr, "ks_block_dot_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                   cudaGetErrorString(e));
      return KS_CUDA_ERROR;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return KS_OK;
}

}  // namespace ks

using namespace ks;

extern "C" ks_status ks_block_dot_noalloc(const double *V, int64_t ld, int k, const double *w, int64_t n,
                                          double *h, void *stream) {
  if (k < 0 || k > kNoAllocMaxK) {
    std::fprintf(stderr,
                 "ks_block_dot_noalloc: k = %d basis vectors is outside the allocation-free scratch "
                 "limit of 0..%d (use ks_block_dot for larger k)\n",
                 k, kNoAllocMaxK);
    return KS_BAD_INPUT;
  }
  if (k == 0) return KS_OK;
  if (!V || !w || !h || n < 1 || ld < n) {
    std::fprintf(stderr, "ks_block_dot_noalloc: null pointer, n < 1 or ld < n\n");
    return KS_BAD_INPUT;
  }
  void *scratch = nullptr;
  const ks_status s = noalloc_scratch(&scratch);
  if (s != KS_OK) return s;
  double *partials = (double *)scratch;
  unsigned *counters = (unsigned *)((unsigned char *)scratch + kNoAllocCounterOffset);
  cudaStream_t st = (cudaStream_t)stream;
  const int groups = (k + kBlockDotGroup - 1) / kBlockDotGroup;
  // Every call shares the scratch; the counters must start at zero.
  cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(unsigned) * groups, st);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return KS_CUDA_ERROR;
  }
  long long gx = (n + kThreads - 1) / kThreads;
  if (gx > kNoAllocGrid) gx = kNoAllocGrid;
  dim3 grid((unsigned)groups, (unsigned)gx);
  block_dot_kernel<1, double, PutArray><<<grid, kThreads, 0, st>>>(V, ld, k, w, nullptr, n, PutArray{h, 0, 1},
                                                                  Stop{nullptr, nullptr}, partials, counters);
  e = cudaGetLastError();
  return e == cudaSuccess ? KS_OK : KS_CUDA_ERROR;
}
