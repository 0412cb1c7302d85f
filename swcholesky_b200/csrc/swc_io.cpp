// Host I/O of the numeric phase's inputs: Matrix Market files and permutation files.
//
// The reference reads its matrices with readMatrix (common/Util.h:77-179), which needs the
// exact header "%%MatrixMarket matrix coordinate real symmetric", lower-triangle entries
// sorted by column and then row, and a non-empty column everywhere (an empty column shifts
// every later column); its return value is ignored by the driver.  The permutation comes
// from a raw file of n native size_t values read with fread
// (examples/sw_choleskyTest01.cpp:70-82), unchecked.
//
// This reader accepts any coordinate file of a square real (or integer) matrix, symmetric
// or general: comment and blank lines anywhere before the entries, any entry order,
// duplicates (summed), upper-triangle entries of a symmetric file (mirrored to the lower
// triangle) and, for a general file, both triangles (the lower one is kept; a value that
// differs from its mirror is reported as an error).  Empty columns are fine, and a column
// without a diagonal entry gets an explicit zero one, so the result is always a lower CSC
// matrix with sorted rows and the diagonal first in every column -- the form the
// reference's reader produces for well-formed files.  Every malformed input (bad header,
// complex / pattern / Hermitian / skew-symmetric data, non-square size, index out of range,
// missing or extra entries, unparsable numbers) is an error with a message.
//
// Permutation files hold n native-endian size_t values, as the reference's driver reads
// them; the reader checks the file size and that the values form a permutation.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "swc_internal.h"

namespace swc {

namespace {

struct Entry {
  int col, row;
  double val;
};

std::string lower(std::string s) {
  for (char &ch : s) ch = (char)std::tolower((unsigned char)ch);
  return s;
}

// Next line of the file without its line break; false at end of file.
bool next_line(FILE *f, std::string &line) {
  line.clear();
  int ch;
  bool any = false;
  while ((ch = std::fgetc(f)) != EOF) {
    any = true;
    if (ch == '\n') break;
    if (ch != '\r') line.push_back((char)ch);
  }
  return any;
}

bool blank(const std::string &s) {
  for (char ch : s)
    if (!std::isspace((unsigned char)ch)) return false;
  return true;
}

}  // namespace

bool read_matrix_market(const char *path, MtxLower &out, std::string &err) {
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path + ": " + std::strerror(errno);
    return false;
  }
  struct Closer {
    FILE *f;
    ~Closer() { std::fclose(f); }
  } closer{f};
  std::string line;
  if (!next_line(f, line)) { err = "empty file"; return false; }
  char b0[64] = {0}, b1[64] = {0}, b2[64] = {0}, b3[64] = {0}, b4[64] = {0};
  if (std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", b0, b1, b2, b3, b4) != 5) {
    err = "header line does not hold 5 tokens (%%MatrixMarket matrix coordinate <field> <symmetry>)";
    return false;
  }
  const std::string banner = lower(b0), object = lower(b1), format = lower(b2),
                    field = lower(b3), symmetry = lower(b4);
  if (banner != "%%matrixmarket") { err = "first token is not %%MatrixMarket"; return false; }
  if (object != "matrix") { err = "object is not a matrix"; return false; }
  if (format != "coordinate") { err = "not in coordinate format (array format is not supported)"; return false; }
  if (field != "real" && field != "integer" && field != "double") {
    err = "field '" + field + "' is not supported (needs real or integer values)";
    return false;
  }
  const bool sym = symmetry == "symmetric";
  if (!sym && symmetry != "general") {
    err = "symmetry '" + symmetry + "' is not supported (needs symmetric or general)";
    return false;
  }
  // size line: first non-comment, non-blank line
  long long nr = -1, nc = -1, nz = -1;
  while (next_line(f, line)) {
    if (line.empty() || line[0] == '%' || blank(line)) continue;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &nr, &nc, &nz) != 3) {
      err = "size line does not hold rows, columns and entries";
      return false;
    }
    break;
  }
  if (nr < 0) { err = "missing size line"; return false; }
  if (nr != nc) { err = "matrix is not square"; return false; }
  if (nr <= 0 || nr > INT32_MAX || nz < 0) { err = "invalid matrix size"; return false; }
  const int n = (int)nr;
  std::vector<Entry> ent;
  ent.reserve((size_t)nz + n);
  long long seen = 0;
  std::vector<Entry> upper;   // general files: entries above the diagonal, for the check
  while (seen < nz && next_line(f, line)) {
    if (line.empty() || line[0] == '%' || blank(line)) continue;
    long long i = 0, j = 0;
    double v = 0.0;
    char *p = const_cast<char *>(line.c_str()), *q = nullptr;
    i = std::strtoll(p, &q, 10);
    if (q == p) { err = "entry " + std::to_string(seen + 1) + ": missing row index"; return false; }
    p = q;
    j = std::strtoll(p, &q, 10);
    if (q == p) { err = "entry " + std::to_string(seen + 1) + ": missing column index"; return false; }
    p = q;
    v = std::strtod(p, &q);
    if (q == p) { err = "entry " + std::to_string(seen + 1) + ": missing value"; return false; }
    if (i < 1 || i > n || j < 1 || j > n) {
      err = "entry " + std::to_string(seen + 1) + ": index out of range";
      return false;
    }
    if (!std::isfinite(v)) { err = "entry " + std::to_string(seen + 1) + ": value is not finite"; return false; }
    int r = (int)(i - 1), c = (int)(j - 1);
    if (r < c) {
      if (sym) std::swap(r, c);          // upper entry of a symmetric file: its mirror
      else { upper.push_back({c, r, v}); ++seen; continue; }
    }
    ent.push_back({c, r, v});
    ++seen;
  }
  if (seen < nz) {
    err = "file ends after " + std::to_string(seen) + " of " + std::to_string(nz) + " entries";
    return false;
  }
  while (next_line(f, line))
    if (!(line.empty() || line[0] == '%' || blank(line))) {
      err = "more entries than the size line states";
      return false;
    }
  for (int j = 0; j < n; ++j) ent.push_back({j, j, 0.0});   // every diagonal present
  std::sort(ent.begin(), ent.end(), [](const Entry &a, const Entry &b) {
    return a.col != b.col ? a.col < b.col : a.row < b.row;
  });
  // merge duplicates (the explicit zero diagonals merge into a given one)
  std::vector<Entry> merged;
  merged.reserve(ent.size());
  for (const Entry &e : ent) {
    if (!merged.empty() && merged.back().col == e.col && merged.back().row == e.row)
      merged.back().val += e.val;
    else
      merged.push_back(e);
  }
  if (!sym) {
    // a general file must be symmetric: its upper entries mirror its lower ones one to one
    std::sort(upper.begin(), upper.end(), [](const Entry &a, const Entry &b) {
      return a.row != b.row ? a.row < b.row : a.col < b.col;   // (row, col) of the mirror
    });
    std::vector<Entry> um;
    for (const Entry &e : upper) {
      if (!um.empty() && um.back().col == e.col && um.back().row == e.row) um.back().val += e.val;
      else um.push_back(e);
    }
    for (const Entry &e : um) {
      // mirror of upper (r, c) with r < c is lower (c, r): column r, row c
      const int col = e.row, row = e.col;
      auto it = std::lower_bound(merged.begin(), merged.end(), Entry{col, row, 0.0},
                                 [](const Entry &a, const Entry &b) {
                                   return a.col != b.col ? a.col < b.col : a.row < b.row;
                                 });
      const bool found = it != merged.end() && it->col == col && it->row == row;
      const double lv = found ? it->val : 0.0;
      if (!found || std::fabs(lv - e.val) > 1e-12 * std::max(std::fabs(lv), std::fabs(e.val))) {
        err = "general matrix is not symmetric (entry " + std::to_string(row + 1) + ", " +
              std::to_string(col + 1) + ")";
        return false;
      }
    }
    size_t off_lower = 0;
    for (const Entry &e : merged) off_lower += e.row != e.col;
    if (off_lower != um.size()) {
      err = "general matrix is not symmetric (a lower entry has no upper mirror)";
      return false;
    }
  }
  if (merged.size() > (size_t)INT32_MAX) { err = "too many entries"; return false; }
  out.n = n;
  out.colptr.assign((size_t)n + 1, 0);
  out.rowind.resize(merged.size());
  out.values.resize(merged.size());
  for (size_t k = 0; k < merged.size(); ++k) {
    out.colptr[merged[k].col + 1]++;
    out.rowind[k] = merged[k].row;
    out.values[k] = merged[k].val;
  }
  for (int j = 0; j < n; ++j) out.colptr[j + 1] += out.colptr[j];
  return true;
}

bool write_matrix_market(const char *path, int n, const int *c, const int *r, const double *v,
                         std::string &err) {
  if (n <= 0 || !c || !r || !v) { err = "empty matrix"; return false; }
  for (int j = 0; j < n; ++j) {
    if (c[j + 1] < c[j]) { err = "column pointers not monotone"; return false; }
    for (int p = c[j]; p < c[j + 1]; ++p)
      if (r[p] < j || r[p] >= n || (p > c[j] && r[p] <= r[p - 1])) {
        err = "not a lower CSC matrix with sorted rows";
        return false;
      }
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) { err = std::string("cannot create ") + path + ": " + std::strerror(errno); return false; }
  bool ok = std::fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n%d %d %d\n", n, n,
                         c[n]) > 0;
  for (int j = 0; j < n && ok; ++j)
    for (int p = c[j]; p < c[j + 1] && ok; ++p)
      ok = std::fprintf(f, "%d %d %.17g\n", r[p] + 1, j + 1, v[p]) > 0;
  if (std::fclose(f) != 0) ok = false;
  if (!ok) err = std::string("write to ") + path + " failed";
  return ok;
}

bool read_perm_file(const char *path, int n, std::vector<int64_t> &perm, std::string &err) {
  if (n <= 0) { err = "n must be positive"; return false; }
  FILE *f = std::fopen(path, "rb");
  if (!f) { err = std::string("cannot open ") + path + ": " + std::strerror(errno); return false; }
  std::vector<size_t> raw((size_t)n);
  const size_t got = std::fread(raw.data(), sizeof(size_t), raw.size(), f);
  const bool extra = std::fgetc(f) != EOF;
  std::fclose(f);
  if (got != raw.size()) {
    err = "permutation file holds " + std::to_string(got) + " of " + std::to_string(n) + " values";
    return false;
  }
  if (extra) { err = "permutation file is longer than n values"; return false; }
  std::vector<char> seen((size_t)n, 0);
  perm.resize((size_t)n);
  for (int k = 0; k < n; ++k) {
    if (raw[k] >= (size_t)n || seen[raw[k]]) { err = "file does not hold a permutation of 0..n-1"; return false; }
    seen[raw[k]] = 1;
    perm[k] = (int64_t)raw[k];
  }
  return true;
}

bool write_perm_file(const char *path, int n, const int64_t *perm, std::string &err) {
  if (n <= 0 || !perm) { err = "empty permutation"; return false; }
  std::vector<char> seen((size_t)n, 0);
  std::vector<size_t> raw((size_t)n);
  for (int k = 0; k < n; ++k) {
    if (perm[k] < 0 || perm[k] >= n || seen[perm[k]]) { err = "not a permutation of 0..n-1"; return false; }
    seen[perm[k]] = 1;
    raw[k] = (size_t)perm[k];
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) { err = std::string("cannot create ") + path + ": " + std::strerror(errno); return false; }
  bool ok = std::fwrite(raw.data(), sizeof(size_t), raw.size(), f) == raw.size();
  if (std::fclose(f) != 0) ok = false;
  if (!ok) err = std::string("write to ") + path + " failed";
  return ok;
}

}  // namespace swc
