// The reference's CRS text format (collection::checkCRSMatrix / readMatrix,
// solver_collection.cpp:655-828):
//   <dir>/ColVal.txt  "N M NNZ" then NNZ lines "col val"  (0-based)
//   <dir>/Ptr.txt     "N M NNZ" then N+1 lines "ptr"
//   <dir>/bx.txt      "N M NNZ" then N lines "b x"
// Reading parses whole files from memory, in parallel over chunks of the text
// (parse_tokens); writing uses 17 significant digits so values round-trip
// exactly through the reference's fscanf("%le").
#include <cerrno>
#include <cinttypes>
#include <new>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
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

// Whitespace as strtoll / strtod skip it (isspace in the C locale).
inline bool is_ws(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// Threads for the parse: KS_IO_THREADS if set (tests force several chunks on
// small files with it), else one per 4 MB of text up to the host's cores.
int io_threads(size_t bytes) {
  if (const char *e = std::getenv("KS_IO_THREADS")) {
    const int t = std::atoi(e);
    if (t >= 1) return std::min(t, 256);
  }
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)std::min(hw, 64), bytes >> 22));
}

// Runs fn(k) for k = 0 .. T-1: chunk 0 here, the others on threads of their
// own; a chunk whose thread cannot be started runs here too.
template <class F>
void run_chunks(int T, const F &fn) {
  std::vector<std::thread> pool;
  std::vector<int> here;
  for (int k = 1; k < T; k++) {
    try {
      pool.emplace_back(fn, k);
    } catch (...) {
      here.push_back(k);
    }
  }
  fn(0);
  for (int k : here) fn(k);
  for (auto &t : pool) t.join();
}

// The whitespace-separated tokens of [body, end) (end points at the buffer's
// terminating NUL), the first `want` of them handed to put(t, p) in parallel:
// put parses token t at p, advances p past it and returns false on a parse
// error. The text is cut into chunks at whitespace characters, so no token
// straddles two chunks; a first pass counts each chunk's tokens, their
// prefix sums give each chunk the index of its first token. Tokens are what
// fscanf("%d %le") would read one after another, whatever whitespace (lines,
// blanks, tabs) separates them. Returns false when the text holds fewer than
// `want` tokens or a token does not parse.
template <class Put>
bool parse_tokens(char *body, char *end, long long want, const Put &put) {
  if (want <= 0) return true;
  const size_t len = (size_t)(end - body);
  const int T = io_threads(len);
  std::vector<char *> cut(T + 1);
  cut[0] = body;
  cut[T] = end;
  for (int k = 1; k < T; k++) {
    char *q = std::max(body + len * (size_t)k / (size_t)T, cut[k - 1]);
    while (q < end && !is_ws(*q)) q++;
    cut[k] = q;
  }
  auto starts_token = [&](const char *q) { return !is_ws(*q) && (q == body || is_ws(q[-1])); };
  std::vector<long long> first(T + 1, 0);
  run_chunks(T, [&](int k) {
    long long c = 0;
    for (const char *q = cut[k]; q < cut[k + 1]; q++) c += starts_token(q) ? 1 : 0;
    first[k + 1] = c;
  });
  for (int k = 0; k < T; k++) first[k + 1] += first[k];
  if (first[T] < want) return false;
  std::atomic<bool> ok{true};
  run_chunks(T, [&](int k) {
    char *q = cut[k];
    for (long long t = first[k]; t < std::min(first[k + 1], want); t++) {
      while (is_ws(*q)) q++;
      if (!put(t, q)) {
        ok = false;
        return;
      }
    }
  });
  return ok;
}

bool parse_ll(char *&p, long long *v) {
  char *e = nullptr;
  errno = 0;
  *v = std::strtoll(p, &e, 10);
  if (e == p || errno) return false;
  p = e;
  return true;
}

bool parse_d(char *&p, double *v) {
  char *e = nullptr;
  *v = std::strtod(p, &e);
  if (e == p) return false;
  p = e;
  return true;
}

bool header(const std::string &path, long long h[3]) {
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  int got = std::fscanf(f, "%lld %lld %lld", &h[0], &h[1], &h[2]);
  std::fclose(f);
  return got == 3;
}

// Formats records [0, count) with fmt_one(i, out) into text, in parallel
// over ranges of records, and writes the ranges in order after `head`.
template <class Fmt>
bool write_records(const std::string &path, const std::string &head, long long count, const Fmt &fmt_one) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return false;
  const int T = io_threads((size_t)count * 24);
  std::vector<std::string> part(T);
  auto work = [&](int k) {
    const long long i0 = count * k / T, i1 = count * (k + 1) / T;
    std::string &o = part[k];
    o.reserve((size_t)(i1 - i0) * 32);
    char line[96];
    for (long long i = i0; i < i1; i++) {
      const int m = fmt_one(i, line, sizeof(line));
      if (m > 0) o.append(line, (size_t)m);
    }
  };
  run_chunks(T, work);
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  for (int k = 0; k < T && ok; k++) ok = std::fwrite(part[k].data(), 1, part[k].size(), f) == part[k].size();
  return std::fclose(f) == 0 && ok;
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

static ks_status crs_read(const char *dir, int64_t n, int64_t nnz, int32_t *ptr, int32_t *col, double *val,
                          double *b, double *x);

// Host memory for the text (and the writer's formatted ranges) can run out;
// no exception leaves these entry points.
ks_status ks_crs_read(const char *dir, int64_t n, int64_t nnz, int32_t *ptr, int32_t *col, double *val,
                      double *b, double *x) {
  try {
    return crs_read(dir, n, nnz, ptr, col, val, b, x);
  } catch (const std::bad_alloc &) {
    return KS_OUT_OF_MEMORY;
  } catch (...) {
    return KS_IO_ERROR;
  }
}

static ks_status crs_read(const char *dir, int64_t n, int64_t nnz, int32_t *ptr, int32_t *col, double *val,
                          double *b, double *x) {
  if (!dir || n < 1 || nnz < 0) return KS_BAD_INPUT;
  const std::string d(dir);
  std::vector<char> buf;
  // After the "N M NNZ" header: the file's body and its end.
  auto body = [&](const char *name, char **b0, char **b1) {
    if (!slurp(d + name, buf)) return false;
    Cursor c{buf.data()};
    for (int i = 0; i < 3; i++) c.next_int();
    *b0 = c.p;
    *b1 = buf.data() + buf.size() - 1;
    return c.ok;
  };
  char *b0 = nullptr, *b1 = nullptr;
  if (col || val) {
    if (!body("/ColVal.txt", &b0, &b1)) return KS_IO_ERROR;
    const bool good = parse_tokens(b0, b1, 2 * (long long)nnz, [&](long long t, char *&p) {
      const long long j = t >> 1;
      if ((t & 1) == 0) {
        long long cj;
        if (!parse_ll(p, &cj)) return false;
        if (col) col[j] = (int32_t)cj;
      } else {
        double vj;
        if (!parse_d(p, &vj)) return false;
        if (val) val[j] = vj;
      }
      return true;
    });
    if (!good) return KS_IO_ERROR;
  }
  if (ptr) {
    if (!body("/Ptr.txt", &b0, &b1)) return KS_IO_ERROR;
    const bool good = parse_tokens(b0, b1, (long long)n + 1, [&](long long t, char *&p) {
      long long v;
      if (!parse_ll(p, &v)) return false;
      ptr[t] = (int32_t)v;
      return true;
    });
    if (!good) return KS_IO_ERROR;
  }
  if (b || x) {
    if (!body("/bx.txt", &b0, &b1)) return KS_IO_ERROR;
    const bool good = parse_tokens(b0, b1, 2 * (long long)n, [&](long long t, char *&p) {
      double v;
      if (!parse_d(p, &v)) return false;
      double *out = (t & 1) == 0 ? b : x;
      if (out) out[t >> 1] = v;
      return true;
    });
    if (!good) return KS_IO_ERROR;
  }
  return KS_OK;
}

static ks_status crs_write(const char *dir, int64_t n, int64_t nnz, const int32_t *ptr, const int32_t *col,
                           const double *val, const double *b, const double *x);

ks_status ks_crs_write(const char *dir, int64_t n, int64_t nnz, const int32_t *ptr, const int32_t *col,
                       const double *val, const double *b, const double *x) {
  try {
    return crs_write(dir, n, nnz, ptr, col, val, b, x);
  } catch (const std::bad_alloc &) {
    return KS_OUT_OF_MEMORY;
  } catch (...) {
    return KS_IO_ERROR;
  }
}

static ks_status crs_write(const char *dir, int64_t n, int64_t nnz, const int32_t *ptr, const int32_t *col,
                           const double *val, const double *b, const double *x) {
  if (!dir || n < 1 || nnz < 0 || !ptr || (nnz > 0 && (!col || !val))) return KS_BAD_INPUT;
  const std::string d(dir);
  char head[96];
  std::snprintf(head, sizeof(head), "%" PRId64 " %" PRId64 " %" PRId64 "\n", n, n, nnz);
  const bool ok =
      write_records(d + "/ColVal.txt", head, nnz,
                    [&](long long j, char *o, size_t cap) {
                      return std::snprintf(o, cap, "%d %.17e\n", col[j], val[j]);
                    }) &&
      write_records(d + "/Ptr.txt", head, n + 1,
                    [&](long long i, char *o, size_t cap) { return std::snprintf(o, cap, "%d\n", ptr[i]); }) &&
      write_records(d + "/bx.txt", head, n, [&](long long i, char *o, size_t cap) {
        return std::snprintf(o, cap, "%.17e %.17e\n", b ? b[i] : 0.0, x ? x[i] : 0.0);
      });
  return ok ? KS_OK : KS_IO_ERROR;
}

}  // extern "C"
