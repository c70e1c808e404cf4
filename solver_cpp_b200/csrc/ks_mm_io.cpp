// Matrix Market coordinate input. The reference declares a Matrix Market
// source (-P / -D / -M, solver_collection.cpp:278-286 and 505-601: it looks
// for <MM_Path>/<L1_Dir>/<MM_Dir>/<name>/<name>.mtx) but never reads the
// file; this reader makes that input source work.
//
// Supported: "%%MatrixMarket matrix coordinate <field> <symmetry>" with field
// real, double, integer or pattern (pattern entries are 1.0) and symmetry
// general, symmetric or skew-symmetric (the stored triangle is mirrored, with
// the sign flipped for skew-symmetric). The matrix must be square. Entries
// are ordered by row, then column; entries repeated at one position are
// summed in file order. Complex fields and the dense "array" format are
// rejected with KS_BAD_INPUT.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "krylov_sm100.h"

namespace {

struct Triplet {
  int64_t row, col;
  double val;
};

bool read_file(const char *path, std::vector<char> &buf) {
  FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return false;
  }
  buf.resize((size_t)sz + 1);
  const size_t got = std::fread(buf.data(), 1, (size_t)sz, f);
  std::fclose(f);
  buf.resize(got + 1);
  buf[got] = '\0';
  return true;
}

std::string lower(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// Parses the whole file into CSR arrays (ptr has n + 1 entries).
ks_status parse_mm_body(const char *file, int64_t &n, std::vector<int32_t> &ptr, std::vector<int32_t> &col,
                        std::vector<double> &val) {
  if (!file) return KS_BAD_INPUT;
  std::vector<char> buf;
  if (!read_file(file, buf)) return KS_IO_ERROR;
  char *p = buf.data();
  // banner
  char *eol = std::strchr(p, '\n');
  std::string banner(p, eol ? (size_t)(eol - p) : std::strlen(p));
  char w[5][64] = {{0}};
  if (std::sscanf(banner.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5)
    return KS_BAD_INPUT;
  if (lower(w[0]) != "%%matrixmarket" || lower(w[1]) != "matrix" || lower(w[2]) != "coordinate")
    return KS_BAD_INPUT;
  const std::string field = lower(w[3]), sym = lower(w[4]);
  const bool pattern = field == "pattern";
  if (!(field == "real" || field == "double" || field == "integer" || pattern)) return KS_BAD_INPUT;
  const int mirror = sym == "general" ? 0 : sym == "symmetric" ? 1 : sym == "skew-symmetric" ? -1 : 2;
  if (mirror == 2) return KS_BAD_INPUT;
  p = eol ? eol + 1 : p + std::strlen(p);
  // comment and blank lines, then the size line
  for (;;) {
    while (*p == ' ' || *p == '\t' || *p == '\r') p++;
    if (*p == '%') {
      char *e = std::strchr(p, '\n');
      p = e ? e + 1 : p + std::strlen(p);
    } else if (*p == '\n') {
      p++;
    } else {
      break;
    }
  }
  char *e = nullptr;
  errno = 0;
  const long long rows = std::strtoll(p, &e, 10);
  if (e == p) return KS_BAD_INPUT;
  p = e;
  const long long cols = std::strtoll(p, &e, 10);
  if (e == p) return KS_BAD_INPUT;
  p = e;
  const long long entries = std::strtoll(p, &e, 10);
  if (e == p || errno) return KS_BAD_INPUT;
  p = e;
  if (rows != cols || rows < 1 || rows >= (1LL << 31) - 1 || entries < 0) return KS_BAD_INPUT;
  n = rows;
  std::vector<Triplet> t;
  t.reserve((size_t)entries * (mirror ? 2 : 1));
  for (long long k = 0; k < entries; k++) {
    const long long i = std::strtoll(p, &e, 10);
    if (e == p) return KS_BAD_INPUT;
    p = e;
    const long long j = std::strtoll(p, &e, 10);
    if (e == p) return KS_BAD_INPUT;
    p = e;
    double v = 1.0;
    if (!pattern) {
      v = std::strtod(p, &e);
      if (e == p) return KS_BAD_INPUT;
      p = e;
    }
    if (i < 1 || i > rows || j < 1 || j > cols) return KS_BAD_INPUT;
    t.push_back({i - 1, j - 1, v});
    if (mirror && i != j) t.push_back({j - 1, i - 1, mirror < 0 ? -v : v});
    if (mirror < 0 && i == j) return KS_BAD_INPUT;  // skew-symmetric stores no diagonal
  }
  // order by (row, column), keeping file order among repeats, then sum repeats
  std::stable_sort(t.begin(), t.end(), [](const Triplet &a, const Triplet &b) {
    return a.row != b.row ? a.row < b.row : a.col < b.col;
  });
  ptr.assign((size_t)n + 1, 0);
  col.clear();
  val.clear();
  col.reserve(t.size());
  val.reserve(t.size());
  for (size_t k = 0; k < t.size(); k++) {
    if (k > 0 && t[k].row == t[k - 1].row && t[k].col == t[k - 1].col) {
      val.back() += t[k].val;
      continue;
    }
    if (col.size() >= (size_t)((1LL << 31) - 1)) return KS_BAD_INPUT;
    col.push_back((int32_t)t[k].col);
    val.push_back(t[k].val);
    ptr[(size_t)t[k].row + 1]++;
  }
  for (int64_t r = 0; r < n; r++) ptr[(size_t)r + 1] += ptr[(size_t)r];
  return KS_OK;
}

// Running out of host memory for the entries is KS_OUT_OF_MEMORY; no
// exception leaves the C entry points.
ks_status parse_mm(const char *file, int64_t &n, std::vector<int32_t> &ptr, std::vector<int32_t> &col,
                   std::vector<double> &val) {
  try {
    return parse_mm_body(file, n, ptr, col, val);
  } catch (const std::bad_alloc &) {
    return KS_OUT_OF_MEMORY;
  } catch (...) {
    return KS_BAD_INPUT;
  }
}

}  // namespace

extern "C" {

ks_status ks_mm_read_header(const char *file, int64_t *n, int64_t *nnz) {
  if (!n || !nnz) return KS_BAD_INPUT;
  int64_t rows = 0;
  std::vector<int32_t> ptr, col;
  std::vector<double> val;
  const ks_status s = parse_mm(file, rows, ptr, col, val);
  if (s != KS_OK) return s;
  *n = rows;
  *nnz = (int64_t)col.size();
  return KS_OK;
}

ks_status ks_mm_read(const char *file, int64_t n, int64_t nnz, int32_t *ptr, int32_t *col, double *val) {
  if (!ptr || (nnz > 0 && (!col || !val))) return KS_BAD_INPUT;
  int64_t rows = 0;
  std::vector<int32_t> p, c;
  std::vector<double> v;
  const ks_status s = parse_mm(file, rows, p, c, v);
  if (s != KS_OK) return s;
  if (rows != n || (int64_t)c.size() != nnz) return KS_BAD_INPUT;
  std::memcpy(ptr, p.data(), sizeof(int32_t) * (size_t)(n + 1));
  if (nnz > 0) {
    std::memcpy(col, c.data(), sizeof(int32_t) * (size_t)nnz);
    std::memcpy(val, v.data(), sizeof(double) * (size_t)nnz);
  }
  return KS_OK;
}

}  // extern "C"
