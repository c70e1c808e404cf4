// Host-side plan of a solve split over several GPUs by rows.
//
// The reference splits the rows of A over two GPUs at N1 = ceil(N/2)
// (solver_collection.cpp:1022-1031) and gathers the whole of x through the
// host before every split SpMV (cudaFunction.cu:1942-2226). Here every rank
// owns a contiguous block of rows and keeps x only over the contiguous
// window of columns its rows read; before each SpMV it receives the part of
// that window owned by other ranks (for a stencil matrix split on grid
// planes: one plane from each neighbour) straight into device memory.
#include <algorithm>
#include <cstdint>

#include "krylov_sm100.h"

extern "C" {

ks_status ks_partition_rows(int64_t n, int nranks, int64_t align, int64_t *row_start) {
  if (n < 1 || nranks < 1 || align < 1 || !row_start) return KS_BAD_INPUT;
  const int64_t units = (n + align - 1) / align;
  row_start[0] = 0;
  for (int p = 1; p < nranks; p++) {
    // ceil(p * units / nranks) units, so that two ranks split n rows at ceil(n / 2)
    const int64_t u = (int64_t)(((__int128)p * units + nranks - 1) / nranks);
    row_start[p] = std::min<int64_t>(n, u * align);
  }
  row_start[nranks] = n;
  for (int p = 1; p <= nranks; p++)
    if (row_start[p] < row_start[p - 1]) return KS_BAD_INPUT;
  return KS_OK;
}

ks_status ks_halo_window(int64_t r0, int64_t r1, const int32_t *ptr, const int32_t *col, int64_t *lo,
                         int64_t *hi) {
  if (r0 < 0 || r1 < r0 || !ptr || !lo || !hi) return KS_BAD_INPUT;
  int64_t a = r0, b = r1;
  const int64_t j0 = ptr[0], j1 = ptr[r1 - r0];
  if (j1 < j0 || (j1 > j0 && !col)) return KS_BAD_INPUT;
  for (int64_t j = j0; j < j1; j++) {
    a = std::min<int64_t>(a, col[j - j0]);
    b = std::max<int64_t>(b, (int64_t)col[j - j0] + 1);
  }
  if (a < 0) return KS_BAD_INPUT;
  *lo = a;
  *hi = b;
  return KS_OK;
}

ks_status ks_halo_plan(int nranks, int rank, const int64_t *row_start, const int64_t *win_lo,
                       const int64_t *win_hi, int64_t *send_lo, int64_t *send_hi, int64_t *recv_lo,
                       int64_t *recv_hi) {
  if (nranks < 1 || rank < 0 || rank >= nranks || !row_start || !win_lo || !win_hi || !send_lo || !send_hi ||
      !recv_lo || !recv_hi)
    return KS_BAD_INPUT;
  for (int p = 0; p < nranks; p++)
    if (win_lo[p] > row_start[p] || win_hi[p] < row_start[p + 1]) return KS_BAD_INPUT;
  // One contiguous range each way per peer: the peer's rows lie wholly below
  // or wholly above this rank's rows, and the windows are contiguous.
  auto cut = [](int64_t a0, int64_t a1, int64_t b0, int64_t b1, int64_t *lo, int64_t *hi) {
    *lo = std::max(a0, b0);
    *hi = std::min(a1, b1);
    if (*hi < *lo) *hi = *lo;
  };
  const int64_t r0 = row_start[rank], r1 = row_start[rank + 1];
  for (int q = 0; q < nranks; q++) {
    if (q == rank) {
      send_lo[q] = send_hi[q] = recv_lo[q] = recv_hi[q] = r0;
      continue;
    }
    const int64_t q0 = row_start[q], q1 = row_start[q + 1];
    cut(win_lo[rank], win_hi[rank], q0, q1, &recv_lo[q], &recv_hi[q]);  // q's rows this rank reads
    cut(win_lo[q], win_hi[q], r0, r1, &send_lo[q], &send_hi[q]);        // this rank's rows q reads
  }
  return KS_OK;
}

}  // extern "C"
