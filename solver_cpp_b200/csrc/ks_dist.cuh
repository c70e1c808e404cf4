// Row-split solves over several GPUs: the communicator interface, the halo
// plan of a rank and the distribution record of a matrix.
//
// A rank owns rows [r0, r1) of A and keeps every vector over a window
// [ext_lo, ext_hi) of global indices around them: the local part at offset
// r0 - ext_lo, the halo below and above it. Its local CSR stores columns as
// global column - r0 (negative for the halo below), so the SpMV gathers from
// the local part's pointer exactly as in a single-GPU solve, and the int16
// offsets col - row are the global ones.
#pragma once

#include <vector>

#include "ks_common.cuh"

namespace ks {

struct HaloRange {
  long long send_lo = 0, send_hi = 0;  // own rows the peer reads
  long long recv_lo = 0, recv_hi = 0;  // the peer's rows this rank reads
};

struct HaloPlan {
  std::vector<long long> row_start;  // every rank's first row (nranks + 1)
  std::vector<HaloRange> peer;       // per rank (empty ranges for self)
};

}  // namespace ks

// Transport of a split solve. Every call is queued on the rank's context
// stream in the same order on every rank.
struct ks_comm {
  ks_ctx *ctx = nullptr;
  int nranks = 1, rank = 0;
  virtual ~ks_comm() = default;
  // buf[0..count) summed over the ranks, in place
  virtual ks_status allreduce(double *buf, int count) = 0;
  // receive the halo of x (the local part's pointer; elem bytes per entry)
  virtual ks_status exchange(const ks::HaloPlan &plan, void *x, size_t elem) = 0;
  // host values of every rank, rank-major (setup only; synchronous)
  virtual ks_status allgather_host(const long long *mine, int count, long long *all) = 0;
};

namespace ks {

struct DistInfo {
  ks_comm *comm = nullptr;
  long long n_global = 0, r0 = 0, r1 = 0;
  long long lo = 0, hi = 0;    // window of A's local rows
  long long tlo = 0, thi = 0;  // window of A^T's local rows (if any)
  long long ext_lo = 0, ext_hi = 0;  // union: the vector layout
  HaloPlan planA, planT;
  long long off() const { return r0 - ext_lo; }   // local part's offset in a slot
  long long ld() const { return ext_hi - ext_lo; }  // slot length
};

}  // namespace ks
