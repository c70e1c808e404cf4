// The reference's CRS text format (collection::checkCRSMatrix / readMatrix,
// solver_collection.cpp:655-828):
//   <dir>/ColVal.txt  "N M NNZ" then NNZ lines "col val"  (0-based)
//   <dir>/Ptr.txt     "N M NNZ" then N+1 lines "ptr"
//   <dir>/bx.txt      "N M NNZ" then N lines "b x"
// Reading parses whole files from memory; writing uses 17 significant digits
// so values round-trip exactly through the reference's fscanf("%le").
#include <cerrno>
#include <cstdarg>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "krylov_sm100.h"

namespace {

bool slurp(const std::string &path, std::vector<char> &buf) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return false;
  }
  buf.resize((size_t)sz + 1);
  size_t got = std::fread(buf.data(), 1, (size_t)sz, f);
  std::fclose(f);
  buf[got] = '\0';
  buf.resize(got + 1);
  return true;
}

struct Cursor {
  char *p;
  bool ok = true;
  long long next_int() {
    char *e = nullptr;
    errno = 0;
    long long v = std::strtoll(p, &e, 10);
    if (e == p || errno) ok = false;
    p = e;
    return v;
  }
  double next_double() {
    char *e = nullptr;
    double v = std::strtod(p, &e);
    if (e == p) ok = false;
    p = e;
    return v;
  }
};

bool header(const std::string &path, long long h[3]) {
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  int got = std::fscanf(f, "%lld %lld %lld", &h[0], &h[1], &h[2]);
  std::fclose(f);
  return got == 3;
}

struct Writer {
  FILE *f;
  std::vector<char> buf;
  size_t used = 0;
  explicit Writer(FILE *fp) : f(fp), buf(1 << 22) {}
  void flush() {
    if (used) std::fwrite(buf.data(), 1, used, f);
    used = 0;
  }
  void put(const char *fmt, ...) __attribute__((format(printf, 2, 3)));
};

void Writer::put(const char *fmt, ...) {
  if (buf.size() - used < 256) flush();
  va_list ap;
  va_start(ap, fmt);
  int k = std::vsnprintf(buf.data() + used, buf.size() - used, fmt, ap);
  va_end(ap);
  if (k > 0) used += (size_t)k;
}

}  // namespace

extern "C" {

ks_status ks_crs_read_header(const char *dir, int64_t *n, int64_t *nnz) {
  if (!dir || !n || !nnz) return KS_BAD_INPUT;
  const std::string d(dir);
  long long h[3][3];
  const char *names[3] = {"/ColVal.txt", "/Ptr.txt", "/bx.txt"};
  for (int i = 0; i < 3; i++)
    if (!header(d + names[i], h[i])) return KS_IO_ERROR;
  for (int c = 0; c < 3; c++)
    if (h[0][c] != h[1][c] || h[1][c] != h[2][c]) return KS_IO_ERROR;  // "Three N/M/NNZ ... not same"
  if (h[0][0] != h[0][1]) return KS_IO_ERROR;                           // "N != M"
  *n = h[0][0];
  *nnz = h[0][2];
  return KS_OK;
}

ks_status ks_crs_read(const char *dir, int64_t n, int64_t nnz, int32_t *ptr, int32_t *col, double *val,
                      double *b, double *x) {
  if (!dir || n < 1 || nnz < 0) return KS_BAD_INPUT;
  const std::string d(dir);
  std::vector<char> buf;
  if (col || val) {
    if (!slurp(d + "/ColVal.txt", buf)) return KS_IO_ERROR;
    Cursor c{buf.data()};
    for (int i = 0; i < 3; i++) c.next_int();
    for (int64_t j = 0; j < nnz && c.ok; j++) {
      long long cj = c.next_int();
      double vj = c.next_double();
      if (col) col[j] = (int32_t)cj;
      if (val) val[j] = vj;
    }
    if (!c.ok) return KS_IO_ERROR;
  }
  if (ptr) {
    if (!slurp(d + "/Ptr.txt", buf)) return KS_IO_ERROR;
    Cursor c{buf.data()};
    for (int i = 0; i < 3; i++) c.next_int();
    for (int64_t i = 0; i <= n && c.ok; i++) ptr[i] = (int32_t)c.next_int();
    if (!c.ok) return KS_IO_ERROR;
  }
  if (b || x) {
    if (!slurp(d + "/bx.txt", buf)) return KS_IO_ERROR;
    Cursor c{buf.data()};
    for (int i = 0; i < 3; i++) c.next_int();
    for (int64_t i = 0; i < n && c.ok; i++) {
      double bi = c.next_double();
      double xi = c.next_double();
      if (b) b[i] = bi;
      if (x) x[i] = xi;
    }
    if (!c.ok) return KS_IO_ERROR;
  }
  return KS_OK;
}

ks_status ks_crs_write(const char *dir, int64_t n, int64_t nnz, const int32_t *ptr, const int32_t *col,
                       const double *val, const double *b, const double *x) {
  if (!dir || n < 1 || nnz < 0 || !ptr || (nnz > 0 && (!col || !val))) return KS_BAD_INPUT;
  const std::string d(dir);
  {
    FILE *f = std::fopen((d + "/ColVal.txt").c_str(), "w");
    if (!f) return KS_IO_ERROR;
    Writer w(f);
    w.put("%" PRId64 " %" PRId64 " %" PRId64 "\n", n, n, nnz);
    for (int64_t j = 0; j < nnz; j++) w.put("%d %.17e\n", col[j], val[j]);
    w.flush();
    std::fclose(f);
  }
  {
    FILE *f = std::fopen((d + "/Ptr.txt").c_str(), "w");
    if (!f) return KS_IO_ERROR;
    Writer w(f);
    w.put("%" PRId64 " %" PRId64 " %" PRId64 "\n", n, n, nnz);
    for (int64_t i = 0; i <= n; i++) w.put("%d\n", ptr[i]);
    w.flush();
    std::fclose(f);
  }
  {
    FILE *f = std::fopen((d + "/bx.txt").c_str(), "w");
    if (!f) return KS_IO_ERROR;
    Writer w(f);
    w.put("%" PRId64 " %" PRId64 " %" PRId64 "\n", n, n, nnz);
    for (int64_t i = 0; i < n; i++) w.put("%.17e %.17e\n", b ? b[i] : 0.0, x ? x[i] : 0.0);
    w.flush();
    std::fclose(f);
  }
  return KS_OK;
}

}  // extern "C"
