// Communicators of a row-split solve.
//
// * NCCL: libnccl.so.2 is opened at run time (the library itself does not
//   depend on it). The halo exchange is one group of point-to-point
//   sends/receives of contiguous byte ranges straight into the window, the
//   dots one in-place all-reduce; both are queued on the context stream.
// * Local: ranks emulated inside one process (several contexts, typically on
//   one GPU, each driven by its own host thread). The same queue of steps,
//   with the exchange done by device-to-device copies from the peer's vector
//   and the all-reduce by a kernel that sums every rank's values in rank
//   order; CUDA events order the streams and a host barrier (bounded wait)
//   hands the events and pointers over. No kernel waits on another.
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>

#include "ks_dist.cuh"

namespace ks {

// ------------------------------------------------------------------ NCCL
struct NcclApi {
  void *h = nullptr;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

static NcclApi *nccl_api() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return;
    NcclApi a;
    a.h = h;
    a.GetUniqueId = (decltype(a.GetUniqueId))dlsym(h, "ncclGetUniqueId");
    a.CommInitRank = (decltype(a.CommInitRank))dlsym(h, "ncclCommInitRank");
    a.CommDestroy = (decltype(a.CommDestroy))dlsym(h, "ncclCommDestroy");
    a.AllReduce = (decltype(a.AllReduce))dlsym(h, "ncclAllReduce");
    a.AllGather = (decltype(a.AllGather))dlsym(h, "ncclAllGather");
    a.Send = (decltype(a.Send))dlsym(h, "ncclSend");
    a.Recv = (decltype(a.Recv))dlsym(h, "ncclRecv");
    a.GroupStart = (decltype(a.GroupStart))dlsym(h, "ncclGroupStart");
    a.GroupEnd = (decltype(a.GroupEnd))dlsym(h, "ncclGroupEnd");
    a.GetErrorString = (decltype(a.GetErrorString))dlsym(h, "ncclGetErrorString");
    if (a.GetUniqueId && a.CommInitRank && a.CommDestroy && a.AllReduce && a.AllGather && a.Send && a.Recv &&
        a.GroupStart && a.GroupEnd && a.GetErrorString)
      api = a;
  });
  return api.h ? &api : nullptr;
}

struct NcclComm : ks_comm {
  NcclApi *api = nullptr;
  ncclComm_t comm = nullptr;
  long long *d_gather = nullptr;
  ~NcclComm() override {
    if (comm) api->CommDestroy(comm);
    cudaFree(d_gather);
  }
  ks_status fail(ncclResult_t r, const char *what) {
    return set_error(ctx, KS_CUDA_ERROR, std::string(what) + ": " + api->GetErrorString(r));
  }
  ks_status allreduce(double *buf, int count) override {
    const ncclResult_t r = api->AllReduce(buf, buf, (size_t)count, ncclDouble, ncclSum, comm, ctx->stream);
    return r == ncclSuccess ? KS_OK : fail(r, "ncclAllReduce");
  }
  ks_status exchange(const HaloPlan &plan, void *x, size_t elem) override {
    char *xl = (char *)x;
    const long long r0 = plan.row_start[rank];
    ncclResult_t r = api->GroupStart();
    for (int q = 0; q < nranks && r == ncclSuccess; q++) {
      if (q == rank) continue;
      const HaloRange &h = plan.peer[q];
      if (h.send_hi > h.send_lo)
        r = api->Send(xl + (h.send_lo - r0) * (long long)elem, (size_t)(h.send_hi - h.send_lo) * elem, ncclChar, q,
                      comm, ctx->stream);
      if (r == ncclSuccess && h.recv_hi > h.recv_lo)
        r = api->Recv(xl + (h.recv_lo - r0) * (long long)elem, (size_t)(h.recv_hi - h.recv_lo) * elem, ncclChar, q,
                      comm, ctx->stream);
    }
    const ncclResult_t e = api->GroupEnd();
    if (r != ncclSuccess) return fail(r, "ncclSend/ncclRecv");
    return e == ncclSuccess ? KS_OK : fail(e, "ncclGroupEnd");
  }
  ks_status allgather_host(const long long *mine, int count, long long *all) override {
    const size_t bytes = sizeof(long long) * (size_t)count;
    cudaFree(d_gather);
    d_gather = nullptr;
    KS_CUDA(ctx, cudaMalloc(&d_gather, bytes * (size_t)nranks));
    KS_CUDA(ctx, cudaMemcpyAsync(d_gather + (size_t)rank * count, mine, bytes, cudaMemcpyHostToDevice, ctx->stream));
    const ncclResult_t r =
        api->AllGather(d_gather + (size_t)rank * count, d_gather, bytes, ncclChar, comm, ctx->stream);
    if (r != ncclSuccess) return fail(r, "ncclAllGather");
    KS_CUDA(ctx, cudaMemcpyAsync(all, d_gather, bytes * (size_t)nranks, cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KS_OK;
  }
};

// ------------------------------------------------------------------ local
constexpr int kLocalMaxRanks = 16;

struct LocalGroup {
  int P = 0;
  std::mutex m;
  std::condition_variable cv;
  long long gen = 0;
  int arrived = 0;
  bool broken = false;
  std::vector<const void *> ptr;
  std::vector<cudaEvent_t> ev;
  std::vector<long long> host;
  // Wait until every rank has arrived; false (and the group broken for good)
  // if that takes longer than the limit, e.g. because a rank stopped early.
  bool barrier() {
    std::unique_lock<std::mutex> lk(m);
    if (broken) return false;
    const long long g = gen;
    if (++arrived == P) {
      arrived = 0;
      gen++;
      cv.notify_all();
      return true;
    }
    if (!cv.wait_for(lk, std::chrono::seconds(120), [&] { return gen != g || broken; }) || broken) {
      broken = true;
      cv.notify_all();
      return false;
    }
    return true;
  }
};

struct SumArgs {
  const double *src[kLocalMaxRanks];
};

__global__ void k_local_sum(SumArgs a, int P, int count, double *out) {
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    double s = a.src[0][i];
    for (int q = 1; q < P; q++) s += a.src[q][i];
    out[i] = s;
  }
}

struct LocalComm : ks_comm {
  std::shared_ptr<LocalGroup> g;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  double *d_tmp = nullptr;
  int tmp_len = 0;
  ~LocalComm() override {
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
    cudaFree(d_tmp);
  }
  ks_status timeout() { return set_error(ctx, KS_TIMEOUT, "local communicator: a rank did not arrive"); }
  // Publish (p, an event recorded now on this stream), meet the others and
  // read every rank's pointer and event; a second meeting keeps anyone from
  // publishing again before everyone has read this round.
  ks_status meet(const void *p, cudaEvent_t e, std::vector<const void *> &ptrs, std::vector<cudaEvent_t> &evs) {
    KS_CUDA(ctx, cudaEventRecord(e, ctx->stream));
    {
      std::lock_guard<std::mutex> lk(g->m);
      g->ptr[rank] = p;
      g->ev[rank] = e;
    }
    if (!g->barrier()) return timeout();
    {
      std::lock_guard<std::mutex> lk(g->m);
      ptrs = g->ptr;
      evs = g->ev;
    }
    if (!g->barrier()) return timeout();
    return KS_OK;
  }
  ks_status allreduce(double *buf, int count) override {
    if (count > tmp_len) {
      cudaFree(d_tmp);
      d_tmp = nullptr;
      tmp_len = 0;
      KS_CUDA(ctx, cudaMalloc(&d_tmp, sizeof(double) * (size_t)count));
      tmp_len = count;
    }
    std::vector<const void *> ptrs;
    std::vector<cudaEvent_t> evs;
    KS_TRY(meet(buf, ev_a, ptrs, evs));
    SumArgs a{};
    for (int q = 0; q < nranks; q++) {
      if (q != rank) KS_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, evs[q], 0));
      a.src[q] = (const double *)ptrs[q];
    }
    ctx->launches++;
    k_local_sum<<<1, 256, 0, ctx->stream>>>(a, nranks, count, d_tmp);
    KS_CUDA(ctx, cudaGetLastError());
    // every rank has read every buf before any rank overwrites its own
    KS_TRY(meet(nullptr, ev_b, ptrs, evs));
    for (int q = 0; q < nranks; q++)
      if (q != rank) KS_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, evs[q], 0));
    KS_CUDA(ctx, cudaMemcpyAsync(buf, d_tmp, sizeof(double) * (size_t)count, cudaMemcpyDeviceToDevice, ctx->stream));
    return KS_OK;
  }
  ks_status exchange(const HaloPlan &plan, void *x, size_t elem) override {
    std::vector<const void *> ptrs;
    std::vector<cudaEvent_t> evs;
    KS_TRY(meet(x, ev_a, ptrs, evs));
    char *xl = (char *)x;
    const long long r0 = plan.row_start[rank];
    for (int q = 0; q < nranks; q++) {
      const HaloRange &h = plan.peer[q];
      if (q == rank || h.recv_hi <= h.recv_lo) continue;
      KS_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, evs[q], 0));
      const char *src = (const char *)ptrs[q] + (h.recv_lo - plan.row_start[q]) * (long long)elem;
      KS_CUDA(ctx, cudaMemcpyAsync(xl + (h.recv_lo - r0) * (long long)elem, src,
                                   (size_t)(h.recv_hi - h.recv_lo) * elem, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    // the peers' copies out of this rank's x are done before x changes again
    KS_TRY(meet(nullptr, ev_b, ptrs, evs));
    for (int q = 0; q < nranks; q++)
      if (q != rank) KS_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, evs[q], 0));
    return KS_OK;
  }
  ks_status allgather_host(const long long *mine, int count, long long *all) override {
    {
      std::lock_guard<std::mutex> lk(g->m);
      if ((int)g->host.size() < nranks * count) g->host.resize((size_t)nranks * count);
      std::memcpy(g->host.data() + (size_t)rank * count, mine, sizeof(long long) * (size_t)count);
    }
    if (!g->barrier()) return timeout();
    {
      std::lock_guard<std::mutex> lk(g->m);
      std::memcpy(all, g->host.data(), sizeof(long long) * (size_t)nranks * count);
    }
    if (!g->barrier()) return timeout();
    return KS_OK;
  }
};

}  // namespace ks

using namespace ks;

extern "C" {

ks_status ks_comm_unique_id(void *id128) {
  if (!id128) return KS_BAD_INPUT;
  NcclApi *api = nccl_api();
  if (!api) return KS_UNIMPLEMENTED;
  ncclUniqueId id;
  if (api->GetUniqueId(&id) != ncclSuccess) return KS_CUDA_ERROR;
  std::memcpy(id128, &id, sizeof(id));
  return KS_OK;
}

ks_status ks_comm_create_nccl(ks_ctx *ctx, int nranks, int rank, const void *id128, ks_comm **out) {
  if (!ctx || !out || !id128 || nranks < 1 || rank < 0 || rank >= nranks) return KS_BAD_INPUT;
  *out = nullptr;
  NcclApi *api = nccl_api();
  if (!api) return set_error(ctx, KS_UNIMPLEMENTED, "libnccl.so.2 could not be loaded");
  KS_CUDA(ctx, cudaSetDevice(ctx->device));
  ncclUniqueId id;
  std::memcpy(&id, id128, sizeof(id));
  auto *c = new (std::nothrow) NcclComm();
  if (!c) return KS_OUT_OF_MEMORY;
  c->ctx = ctx;
  c->nranks = nranks;
  c->rank = rank;
  c->api = api;
  const ncclResult_t r = api->CommInitRank(&c->comm, nranks, id, rank);
  if (r != ncclSuccess) {
    c->comm = nullptr;
    const ks_status s = c->fail(r, "ncclCommInitRank");
    delete c;
    return s;
  }
  *out = c;
  return KS_OK;
}

ks_status ks_comm_create_local(ks_ctx *const *ctxs, int nranks, ks_comm **comms) {
  if (!ctxs || !comms || nranks < 1 || nranks > kLocalMaxRanks) return KS_BAD_INPUT;
  for (int q = 0; q < nranks; q++) {
    comms[q] = nullptr;
    if (!ctxs[q]) return KS_BAD_INPUT;
  }
  // host allocations can throw; no exception leaves this entry point
  std::shared_ptr<LocalGroup> g;
  try {
    g = std::make_shared<LocalGroup>();
    g->ptr.assign(nranks, nullptr);
    g->ev.assign(nranks, nullptr);
  } catch (...) {
    return KS_OUT_OF_MEMORY;
  }
  g->P = nranks;
  for (int q = 0; q < nranks; q++) {
    auto *c = new (std::nothrow) LocalComm();
    if (!c) {
      for (int p = 0; p < q; p++) {
        delete comms[p];
        comms[p] = nullptr;
      }
      return KS_OUT_OF_MEMORY;
    }
    c->ctx = ctxs[q];
    c->nranks = nranks;
    c->rank = q;
    c->g = g;
    cudaSetDevice(ctxs[q]->device);
    if (cudaEventCreateWithFlags(&c->ev_a, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_b, cudaEventDisableTiming) != cudaSuccess) {
      delete c;
      for (int p = 0; p < q; p++) {
        delete comms[p];
        comms[p] = nullptr;
      }
      return KS_CUDA_ERROR;
    }
    comms[q] = c;
  }
  return KS_OK;
}

ks_status ks_comm_destroy(ks_comm *comm) {
  if (!comm) return KS_OK;
  if (comm->ctx) {
    cudaSetDevice(comm->ctx->device);
    cudaStreamSynchronize(comm->ctx->stream);
  }
  delete comm;
  return KS_OK;
}

ks_status ks_comm_info(const ks_comm *comm, int *nranks, int *rank) {
  if (!comm) return KS_BAD_INPUT;
  if (nranks) *nranks = comm->nranks;
  if (rank) *rank = comm->rank;
  return KS_OK;
}

}  // extern "C"
