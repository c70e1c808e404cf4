// Host-only stand-in for the reference's `class cuda` (cudaFunction.hpp:7-129).
//
// TEST INFRASTRUCTURE ONLY. This file lets the reference's own CPU path
// (blas.cpp, the solver classes, solver_collection.cpp, main.cpp) be compiled
// unmodified with g++ and run on the host as an oracle and CPU baseline. It is
// linked into oracle/_ref/Solver only; nothing in the product library uses it.
//
// In CPU mode (no -c flag) the reference touches `cuda` only for buffer
// management (d_Malloc/d_MallocHost/i_Malloc/i_MallocHost/Free/FreeHost,
// cudaFunction.cu:413-536), device queries (GetDeviceNum/Reset,
// cudaFunction.cu:571-578,1905-1909) and the CSR->CSC transpose used by the
// BiCG family (solver_collection.cpp:857-868 -> cudaFunction.cu:933-982). The
// transpose here is a stable counting sort, which yields the same ordering as
// cuSPARSE csr2csc: inside each column, row indices ascend.
//
// Every device compute entry (MtxVec_mult, dot, Kskip_*, dot_gmres*, *_Multi)
// is only reachable with -c / -g; here they stop the program with a message.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cudaFunction.hpp"

namespace {

[[noreturn]] void device_path_unavailable(const char *what) {
  std::fprintf(stderr,
               "[host-only reference build] %s needs the GPU path (-c/-g), "
               "which this build does not provide\n",
               what);
  std::exit(3);
}

template <typename T>
T *host_alloc(unsigned long int count) {
  void *p = std::calloc(count ? count : 1, sizeof(T));
  if (!p) {
    std::fprintf(stderr, "[host-only reference build] out of host memory\n");
    std::exit(4);
  }
  return static_cast<T *>(p);
}

// Transpose of a square CSR matrix (n x n, nnz entries) by counting sort over
// the column index. Stable in the row index, so each output column lists its
// rows in ascending order.
void csr_transpose(const double *val, const int *col, const int *ptr,
                   double *tval, int *trow, int *tptr, unsigned long int n,
                   unsigned long int nnz) {
  std::vector<unsigned long int> count(n + 1, 0);
  for (unsigned long int j = 0; j < nnz; ++j) count[col[j] + 1]++;
  for (unsigned long int c = 0; c < n; ++c) count[c + 1] += count[c];
  for (unsigned long int c = 0; c <= n; ++c) tptr[c] = (int)count[c];
  for (unsigned long int r = 0; r < n; ++r) {
    for (int j = ptr[r]; j < ptr[r + 1]; ++j) {
      unsigned long int dst = count[col[j]]++;
      trow[dst] = (int)r;
      tval[dst] = val[j];
    }
  }
}

}  // namespace

cuda::cuda(times *t) {
  time = t;
  cu_d1 = cu_d2 = cu_d3 = cu_h1 = NULL;
  cu_d4 = cu_d5 = cu_d6 = cu_d7 = cu_d8 = cu_h2 = cu_h3 = cu_h4 = NULL;
  cu_d9 = cu_h5 = NULL;
  cu_d10 = cu_h6 = cu_d11 = cu_h7 = NULL;
  cu_d100 = cu_d101 = NULL;
  cu_d200 = cu_d201 = cu_h8 = NULL;
  cu_d1_1 = cu_d1_2 = cu_d2_1 = cu_d2_2 = NULL;
  cu_d4_1 = cu_d4_2 = cu_d5_1 = cu_d5_2 = NULL;
  size = size1 = size2 = 0;
  k = 0;
  restart = 0;
  isMulti = false;
}

cuda::cuda(times *t, unsigned long int n, unsigned long int n1,
           unsigned long int n2)
    : cuda(t) {
  size = n;
  size1 = n1;
  size2 = n2;
  isMulti = !(n1 == 0 && n2 == 0);
}

cuda::cuda(times *t, unsigned long int n, int kk, unsigned long int n1,
           unsigned long int n2)
    : cuda(t, n, n1, n2) {
  k = kk;
}

cuda::cuda(times *t, unsigned long int n, double r, unsigned long int n1,
           unsigned long int n2)
    : cuda(t, n, n1, n2) {
  restart = (int)r;
}

cuda::cuda(times *t, unsigned long int n, int kk, double r,
           unsigned long int n1, unsigned long int n2)
    : cuda(t, n, kk, n1, n2) {
  restart = (int)r;
}

cuda::~cuda() {}

double *cuda::d_Malloc(unsigned long int n, int) { return host_alloc<double>(n); }
double *cuda::d_MallocHost(unsigned long int n, int) { return host_alloc<double>(n); }
int *cuda::i_Malloc(unsigned long int n, int) { return host_alloc<int>(n); }
int *cuda::i_MallocHost(unsigned long int n, int) { return host_alloc<int>(n); }

void cuda::H2D(double *from, double *to, unsigned long int n, bool, int) {
  std::memcpy(to, from, n * sizeof(double));
}
void cuda::D2H(double *from, double *to, unsigned long int n, bool, int) {
  std::memcpy(to, from, n * sizeof(double));
}
void cuda::H2D(int *from, int *to, unsigned long int n, bool, int) {
  std::memcpy(to, from, n * sizeof(int));
}
void cuda::D2H(int *from, int *to, unsigned long int n, bool, int) {
  std::memcpy(to, from, n * sizeof(int));
}

void cuda::Free(void *p) { std::free(p); }
void cuda::FreeHost(void *p) { std::free(p); }

void cuda::Memset(double *p, double v, unsigned long int n, bool, int) {
  for (unsigned long int i = 0; i < n; ++i) p[i] = v;
}
void cuda::Memset(int *p, int v, unsigned long int n, bool, int) {
  for (unsigned long int i = 0; i < n; ++i) p[i] = v;
}

void cuda::Reset(int) {}
int cuda::GetDeviceNum() { return 1; }
void cuda::ShowDevice() {}
void cuda::EnableP2P() {}
void cuda::SetSize_Multi(int s1, int s2) {
  size1 = (unsigned long int)s1;
  size2 = (unsigned long int)s2;
}
void cuda::HostRegister(void *, int) {}
void cuda::HostUnregister(void *) {}

void cuda::CSR2CSC(double *CSRval, int *CSRcol, int *CSRptr, double *CSCval,
                   int *CSCrow, int *CSCptr, unsigned long int N,
                   unsigned long int NNZ) {
  csr_transpose(CSRval, CSRcol, CSRptr, CSCval, CSCrow, CSCptr, N, NNZ);
}

void cuda::CSR2CSC(double *, int *, int *, double *, int *, int *, double *,
                   int *, int *, unsigned long int, unsigned long int) {
  device_path_unavailable("CSR2CSC (device arrays)");
}

void cuda::MtxVec_mult(double *, double *, unsigned long int, double *, int *,
                       int *) {
  device_path_unavailable("MtxVec_mult");
}
void cuda::MtxVec_mult(double *, double *, double *, int *, int *) {
  device_path_unavailable("MtxVec_mult");
}
void cuda::MtxVec_mult(double *, unsigned long int, unsigned long int, double *,
                       unsigned long int, unsigned long int, double *, int *,
                       int *) {
  device_path_unavailable("MtxVec_mult");
}
void cuda::MtxVec_mult(double *, unsigned long int, unsigned long int, double *,
                       double *, int *, int *) {
  device_path_unavailable("MtxVec_mult");
}

double cuda::dot(double *, double *, unsigned long int) { device_path_unavailable("dot"); }
double cuda::dot(double *, double *) { device_path_unavailable("dot"); }
double cuda::dot(double *, unsigned long int, unsigned long int, double *,
                 unsigned long int, unsigned long int) {
  device_path_unavailable("dot");
}
double cuda::dot(double *, double *, unsigned long int, unsigned long int) {
  device_path_unavailable("dot");
}
double cuda::dot(double *, unsigned long int, unsigned long int, double *) {
  device_path_unavailable("dot");
}

void cuda::Kskip_cg_bicg_base(double *, double *, double *, double *, const int,
                              double *, int *, int *) {
  device_path_unavailable("Kskip_cg_bicg_base");
}
void cuda::Kskip_cg_bicg_base2(double *, double *, double *, double *,
                               const int, double *, int *, int *) {
  device_path_unavailable("Kskip_cg_bicg_base2");
}
void cuda::Kskip_cg_innerProduce(double *, double *, double *, double *,
                                 double *, double *, double *, int, double *,
                                 int *, int *) {
  device_path_unavailable("Kskip_cg_innerProduce");
}
void cuda::Kskip_cg_innerProduce2(double *, double *, double *, double *,
                                  double *, double *, double *, int, double *,
                                  int *, int *) {
  device_path_unavailable("Kskip_cg_innerProduce2");
}
void cuda::Kskip_cg_innerProduce3(double *, double *, double *, double *,
                                  double *, double *, double *, int, double *,
                                  int *, int *) {
  device_path_unavailable("Kskip_cg_innerProduce3");
}
void cuda::Kskip_bicg_innerProduce(double *, double *, double *, double *,
                                   double *, double *, double *, double *, int,
                                   double *, int *, int *) {
  device_path_unavailable("Kskip_bicg_innerProduce");
}
void cuda::Kskip_bicg_innerProduce2(double *, double *, double *, double *,
                                    double *, double *, double *, double *, int,
                                    double *, int *, int *) {
  device_path_unavailable("Kskip_bicg_innerProduce2");
}
void cuda::Kskip_bicg_innerProduce3(double *, double *, double *, double *,
                                    double *, double *, double *, double *, int,
                                    double *, int *, int *) {
  device_path_unavailable("Kskip_bicg_innerProduce3");
}
void cuda::dot_gmres(double *, double *, double *, int, unsigned long int) {
  device_path_unavailable("dot_gmres");
}
void cuda::dot_gmres2(double *, double *, double *, int, unsigned long int) {
  device_path_unavailable("dot_gmres2");
}
void cuda::dot_gmres3(double *, double *, double *, int, unsigned long int) {
  device_path_unavailable("dot_gmres3");
}
void cuda::MtxVec_mult_Multi(double *, double *, double *, int *, int *,
                             double *, int *, int *) {
  device_path_unavailable("MtxVec_mult_Multi");
}
void cuda::Kskip_cg_bicg_base_Multi(double *, double *, double *, double *,
                                    const int, double *, int *, int *, double *,
                                    int *, int *) {
  device_path_unavailable("Kskip_cg_bicg_base_Multi");
}
