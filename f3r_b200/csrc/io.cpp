// io.cpp -- Matrix Market ingest and output: the on-disk formats on either
// side of the solve.
//
// Reading follows kmm::io::mm (umineko-sparse/matrix/io.hpp):
//  - read_matrix + io::CSR(COO) (io.hpp:91-96, 44-60, 129-192): coordinate
//    real/integer files, general or symmetric; an off-diagonal entry whose
//    value is exactly 0 is dropped; a symmetric file's off-diagonal entry is
//    mirrored right after itself; rows are filled in file order and then
//    sorted by column; duplicate entries are kept as separate entries;
//  - read_system's right-hand side (io.hpp:104-126): "<stem>_b.mtx" (the
//    matrix path with "_b" inserted before its last four characters), an
//    n x 1 "array real general" file, or, when that file does not exist, n
//    values U(0, 1) from std::mt19937_64(0), the drivers' init (f3r-gpu.cpp:60,
//    core/tensor.hpp:253-265).
// Where the reference exits or misreads (a malformed header, a pattern or
// complex file, an index out of range, a short file, a right-hand side of the
// wrong length) these functions return F3R_ERROR_INVALID_VALUE with a message.
//
// The data section is parsed by OpenMP threads over newline-aligned chunks
// of the file image; the chunks are concatenated in file order, so the
// result does not depend on the thread count.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <omp.h>

#include "internal.hpp"

using namespace f3r;

namespace {

// Whole-file image, NUL-terminated.
Status slurp(const char *path, std::vector<char> &buf, bool *missing = nullptr) {
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    if (missing) {
      *missing = true;
      return F3R_SUCCESS;
    }
    return fail(F3R_ERROR_INVALID_VALUE, std::string("cannot open ") + path + ": " + std::strerror(errno));
  }
  if (missing) *missing = false;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return fail(F3R_ERROR_INVALID_VALUE, std::string("cannot size ") + path);
  }
  buf.resize((size_t)sz + 1);
  size_t got = sz ? std::fread(buf.data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if (got != (size_t)sz) return fail(F3R_ERROR_INVALID_VALUE, std::string("short read of ") + path);
  buf[(size_t)sz] = '\0';
  return F3R_SUCCESS;
}

std::string lower(std::string s) {
  for (auto &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

struct Header {
  std::string object, format, field, symmetry;
};

// Banner "%%MatrixMarket object format field symmetry" (keywords are
// case-insensitive in the Matrix Market definition).  Returns the offset just
// past the comment lines, i.e. at the size line.
Status parse_header(const std::vector<char> &buf, const char *path, Header &h, size_t &pos) {
  const char *p = buf.data();
  const char *eol = std::strchr(p, '\n');
  std::string line(p, eol ? (size_t)(eol - p) : std::strlen(p));
  char t[5][64];
  if (std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", t[0], t[1], t[2], t[3], t[4]) != 5 ||
      lower(t[0]) != "%%matrixmarket")
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": not a Matrix Market file (banner: '" + line + "')");
  h.object = lower(t[1]);
  h.format = lower(t[2]);
  h.field = lower(t[3]);
  h.symmetry = lower(t[4]);
  // skip the banner and every following line that starts with '%' (or is blank)
  pos = eol ? (size_t)(eol - p) + 1 : line.size();
  const size_t end = buf.size() - 1;
  while (pos < end) {
    size_t q = pos;
    while (q < end && (buf[q] == ' ' || buf[q] == '\t' || buf[q] == '\r')) q++;
    if (q < end && buf[q] != '%' && buf[q] != '\n') break;
    while (q < end && buf[q] != '\n') q++;
    pos = q + 1;
  }
  return F3R_SUCCESS;
}

// Reads one number the way the reference does (strtod), advancing p.
inline bool next_num(const char *&p, double &v) {
  char *e;
  v = std::strtod(p, &e);
  if (e == p) return false;
  p = e;
  return true;
}

// An integer-valued field (an index or a size).
inline bool next_int(const char *&p, int64_t &v) {
  double d;
  if (!next_num(p, d) || !(d == std::floor(d)) || std::fabs(d) > 9.0e18) return false;
  v = (int64_t)d;
  return true;
}

struct Chunk {
  std::vector<int32_t> row, col;
  std::vector<double> val;
  int64_t lines = 0;        // data lines parsed
  int64_t bad_line = -1;    // first malformed line (chunk-local line number)
  std::string why;
};

// Parses the data lines in [b, e): "row col value" per line, 1-based.
void parse_chunk(const char *b, const char *e, int64_t nrow, int64_t ncol, bool sym, Chunk &c) {
  const char *p = b;
  while (p < e) {
    // skip blank lines
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) p++;
    if (p >= e) break;
    const char *eol = (const char *)std::memchr(p, '\n', (size_t)(e - p));
    if (!eol) eol = e;
    int64_t i, j;
    double v;
    const char *q = p;
    // strtod skips newlines, so a short line shows up as q past its end
    if (!next_int(q, i) || !next_int(q, j) || !next_num(q, v) || q > eol) {
      if (c.bad_line < 0) c.bad_line = c.lines, c.why = "expected 'row col value'";
    } else if (i < 1 || i > nrow || j < 1 || j > ncol) {
      if (c.bad_line < 0) c.bad_line = c.lines, c.why = "index out of range";
    } else if (!(v == 0.0 && i != j)) {  // io.hpp:177-180: explicit off-diagonal zeros dropped
      c.row.push_back((int32_t)(i - 1));
      c.col.push_back((int32_t)(j - 1));
      c.val.push_back(v);
      if (sym && i != j) {  // io.hpp:183-188: the mirrored entry follows
        c.row.push_back((int32_t)(j - 1));
        c.col.push_back((int32_t)(i - 1));
        c.val.push_back(v);
      }
    }
    c.lines++;
    p = eol + 1;
  }
}

}  // namespace

extern "C" {

f3r_status f3r_mm_read(const char *path, f3r_host_matrix **out) {
  if (!path || !out) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  std::vector<char> buf;
  F3R_TRY(slurp(path, buf));
  Header h;
  size_t pos = 0;
  F3R_TRY(parse_header(buf, path, h, pos));
  if (h.object != "matrix" || h.format != "coordinate")
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": need a 'matrix coordinate' file, got '" +
                                             h.object + " " + h.format + "'");
  if (h.field != "real" && h.field != "integer" && h.field != "double")
    return fail(F3R_ERROR_UNSUPPORTED, std::string(path) + ": field '" + h.field +
                                           "' (only real and integer matrices are read)");
  if (h.symmetry != "general" && h.symmetry != "symmetric")
    return fail(F3R_ERROR_UNSUPPORTED, std::string(path) + ": symmetry '" + h.symmetry +
                                           "' (only general and symmetric are read)");
  const bool sym = h.symmetry == "symmetric";
  const char *p = buf.data() + pos;
  int64_t nrow, ncol, nlines;
  if (!next_int(p, nrow) || !next_int(p, ncol) || !next_int(p, nlines) || nrow < 0 || ncol < 0 || nlines < 0)
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": bad size line");
  if (nrow > INT32_MAX - 1 || ncol > INT32_MAX - 1)
    return fail(F3R_ERROR_UNSUPPORTED, std::string(path) + ": more than 2^31-2 rows or columns");
  while (*p && *p != '\n') p++;
  const char *data = *p ? p + 1 : p;
  const char *end = buf.data() + buf.size() - 1;

  // newline-aligned chunks, one per thread
  const int T = std::max(1, std::min(omp_get_max_threads(), (int)((end - data) / (1 << 20) + 1)));
  std::vector<const char *> cut(T + 1);
  cut[0] = data;
  cut[T] = end;
  for (int t = 1; t < T; t++) {
    const char *c = data + (end - data) * t / T;
    if (c < cut[t - 1]) c = cut[t - 1];
    const char *nl = (const char *)std::memchr(c, '\n', (size_t)(end - c));
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<Chunk> ch(T);
#pragma omp parallel for schedule(static, 1) num_threads(T)
  for (int t = 0; t < T; t++) parse_chunk(cut[t], cut[t + 1], nrow, ncol, sym, ch[t]);

  int64_t lines = 0, nnz = 0;
  for (int t = 0; t < T; t++) {
    if (ch[t].bad_line >= 0)
      return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": entry " + std::to_string(lines + ch[t].bad_line + 1) +
                                               ": " + ch[t].why);
    lines += ch[t].lines;
    nnz += (int64_t)ch[t].val.size();
  }
  if (lines != nlines)
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": the size line announces " + std::to_string(nlines) +
                                             " entries, the file holds " + std::to_string(lines));
  if (nnz > INT32_MAX)
    return fail(F3R_ERROR_UNSUPPORTED, std::string(path) + ": more than 2^31-1 stored entries");

  // CSR: rows in file order (a stable counting sort, io.hpp:47-56), then each
  // row sorted by column (io.hpp:57-59)
  auto *m = new HostCSR((int32_t)nrow, (int32_t)ncol, nnz);
  std::fill(m->rptr.begin(), m->rptr.end(), 0);
  for (auto &c : ch)
    for (int32_t r : c.row) m->rptr[r + 1]++;
  for (int64_t i = 0; i < nrow; i++) m->rptr[i + 1] += m->rptr[i];
  {
    std::vector<int32_t> fill(m->rptr.begin(), m->rptr.end() - 1);
    for (auto &c : ch)
      for (size_t k = 0; k < c.row.size(); k++) {
        const int32_t at = fill[c.row[k]]++;
        m->idx[at] = c.col[k];
        m->val[at] = c.val[k];
      }
  }
  ch.clear();
#pragma omp parallel
  {
    std::vector<std::pair<int32_t, double>> tmp;
#pragma omp for schedule(dynamic, 4096)
    for (int64_t i = 0; i < nrow; i++) {
      const int32_t b = m->rptr[i], e = m->rptr[i + 1];
      bool sorted = true;
      for (int32_t k = b + 1; k < e && sorted; k++) sorted = m->idx[k - 1] <= m->idx[k];
      if (sorted) continue;
      tmp.clear();
      for (int32_t k = b; k < e; k++) tmp.emplace_back(m->idx[k], m->val[k]);
      std::stable_sort(tmp.begin(), tmp.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
      for (int32_t k = b; k < e; k++) m->idx[k] = tmp[k - b].first, m->val[k] = tmp[k - b].second;
    }
  }
  *out = new f3r_host_matrix;
  (*out)->m.reset(m);
  return F3R_SUCCESS;
}

f3r_status f3r_mm_read_vector(const char *path, int64_t n, double *x) {
  if (!path || (!x && n > 0)) return fail(F3R_ERROR_INVALID_VALUE, "null argument");
  std::vector<char> buf;
  F3R_TRY(slurp(path, buf));
  Header h;
  size_t pos = 0;
  F3R_TRY(parse_header(buf, path, h, pos));
  // io.hpp:200-216: "matrix array real general", one column
  if (h.object != "matrix" || h.format != "array" || h.symmetry != "general" ||
      (h.field != "real" && h.field != "integer" && h.field != "double"))
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": need a 'matrix array real general' file");
  const char *p = buf.data() + pos;
  int64_t nrow, ncol;
  if (!next_int(p, nrow) || !next_int(p, ncol) || ncol != 1)
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": need an n x 1 array");
  if (nrow != n)
    return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": " + std::to_string(nrow) + " values for a system of " +
                                             std::to_string(n) + " rows");
  for (int64_t i = 0; i < n; i++)
    if (!next_num(p, x[i]))
      return fail(F3R_ERROR_INVALID_VALUE, std::string(path) + ": value " + std::to_string(i + 1) + " missing");
  return F3R_SUCCESS;
}

f3r_status f3r_mm_read_rhs(const char *matrix_path, int64_t n, double *b, int32_t *from_file) {
  if (!matrix_path || (!b && n > 0) || n < 0) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  std::string pb = matrix_path;
  if (pb.size() < 4) return fail(F3R_ERROR_INVALID_VALUE, std::string("matrix path too short: ") + matrix_path);
  pb.insert(pb.size() - 4, "_b");  // io.hpp:111-112
  std::vector<char> probe;
  bool missing = false;
  F3R_TRY(slurp(pb.c_str(), probe, &missing));
  if (from_file) *from_file = missing ? 0 : 1;
  if (!missing) return f3r_mm_read_vector(pb.c_str(), n, b);
  // the drivers' init: v.random<0, 1>(std::mt19937_64(0))
  std::mt19937_64 eng(0);
  std::uniform_real_distribution<double> d(0, 1);
  for (int64_t i = 0; i < n; i++) b[i] = d(eng);
  return F3R_SUCCESS;
}

f3r_status f3r_mm_write(const char *path, const f3r_csr *a) {
  if (!path) return fail(F3R_ERROR_INVALID_VALUE, "null path");
  F3R_TRY(check_csr(a));
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(F3R_ERROR_INVALID_VALUE, std::string("cannot create ") + path + ": " + std::strerror(errno));
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %d\n", a->nrows, a->ncols, a->nnz);
  char line[96];
  std::string blk;
  blk.reserve(1 << 20);
  for (int32_t i = 0; i < a->nrows; i++)
    for (int32_t k = a->rptr[i]; k < a->rptr[i + 1]; k++) {
      int len = std::snprintf(line, sizeof line, "%d %d %.17g\n", i + 1, a->idx[k] + 1, a->val[k]);
      blk.append(line, (size_t)len);
      if (blk.size() > (1u << 20) - 128) {
        std::fwrite(blk.data(), 1, blk.size(), f);
        blk.clear();
      }
    }
  std::fwrite(blk.data(), 1, blk.size(), f);
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) return fail(F3R_ERROR_INVALID_VALUE, std::string("write failed: ") + path);
  return F3R_SUCCESS;
}

f3r_status f3r_mm_write_vector(const char *path, int64_t n, const double *x) {
  if (!path || n < 0 || (!x && n > 0)) return fail(F3R_ERROR_INVALID_VALUE, "bad argument");
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(F3R_ERROR_INVALID_VALUE, std::string("cannot create ") + path + ": " + std::strerror(errno));
  std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%lld 1\n", (long long)n);
  for (int64_t i = 0; i < n; i++) std::fprintf(f, "%.17g\n", x[i]);
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) return fail(F3R_ERROR_INVALID_VALUE, std::string("write failed: ") + path);
  return F3R_SUCCESS;
}

}  // extern "C"
