// hostutil.cpp -- host-side parts of the engine: the rank readout and the
// .wdm / SMS file formats.
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rr_internal.h"

namespace rr {

namespace {

// src/modular_linalg.rs:132-183 modular_rank on a small dense matrix.
int64_t small_rank(std::vector<uint64_t> a, int rows, int cols, uint64_t p) {
  auto at = [&](int i, int j) -> uint64_t& { return a[(size_t)i * cols + j]; };
  for (auto& v : a) v %= p;
  int rank = 0;
  for (int c = 0; c < cols; ++c) {
    int pr = -1;
    for (int r = rank; r < rows; ++r)
      if (at(r, c)) { pr = r; break; }
    if (pr < 0) continue;
    for (int j = 0; j < cols; ++j) std::swap(at(rank, j), at(pr, j));
    const uint64_t inv = host_invmod((uint32_t)at(rank, c), (uint32_t)p);
    for (int j = c; j < cols; ++j) at(rank, j) = at(rank, j) * inv % p;
    for (int r = rank + 1; r < rows; ++r) {
      const uint64_t f = at(r, c);
      if (!f) continue;
      for (int j = c; j < cols; ++j) at(r, j) = (at(r, j) + p - f * at(rank, j) % p) % p;
    }
    if (++rank == rows) break;
  }
  return rank;
}

}  // namespace

// src/sigma_basis.rs:71-152 (analyze_pm_basis: reverse row i of the upper-left
// b x b block over its degree -delta_i, pack by degree) followed by
// src/blockbmtest.rs:574-599 (rank = b (k-3) + rank(P[k-1]) + rank(P[0])).
int rank_from_basis_host(const uint32_t* M, const int64_t* delta, int b, int64_t len, uint32_t p, int64_t* rank) {
  const int n2 = 2 * b;
  int64_t maxdel = 0;
  for (int i = 0; i < b; ++i) {
    const int64_t del = -delta[i];
    if (del < 0 || del >= len) return fail(RR_EINVAL, "delta[%d] = %lld outside the basis degree range", i, (long long)delta[i]);
    maxdel = std::max(maxdel, del);
  }
  std::vector<uint64_t> P0((size_t)b * b, 0), Pk((size_t)b * b, 0);
  int64_t maxdeg = 0;
  for (int i = 0; i < b; ++i) {
    const int64_t del = -delta[i];
    for (int j = 0; j < b; ++j)
      for (int64_t k = 0; k <= del; ++k)
        if (M[((size_t)i * n2 + j) * len + (del - k)] != 0) maxdeg = std::max(maxdeg, k);
  }
  const int64_t kk = maxdeg + 1;
  if (kk < 3) return fail(RR_ESTATE, "generator degree %lld too small for a rank estimate", (long long)maxdeg);
  for (int i = 0; i < b; ++i) {
    const int64_t del = -delta[i];
    for (int j = 0; j < b; ++j) {
      P0[(size_t)i * b + j] = M[((size_t)i * n2 + j) * len + del];
      const int64_t k = kk - 1;
      Pk[(size_t)i * b + j] = (k <= del) ? M[((size_t)i * n2 + j) * len + (del - k)] : 0;
    }
  }
  *rank = (int64_t)b * (kk - 3) + small_rank(Pk, b, b, p) + small_rank(P0, b, b, p);
  return RR_OK;
}

}  // namespace rr

using namespace rr;

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(FILE* ff) : f(ff) {}
  ~File() { if (f) fclose(f); }
};

bool read_line(FILE* f, std::string& line) {
  line.clear();
  int ch;
  while ((ch = fgetc(f)) != EOF) {
    if (ch == '\n') return true;
    line.push_back((char)ch);
  }
  return !line.empty();
}

// Parse whitespace-separated unsigned integers of one line into out (at most
// max values are stored; count receives how many were present).
bool parse_u32_line(const std::string& line, uint32_t* out, int64_t max, int64_t* count) {
  const char* s = line.c_str();
  int64_t c = 0;
  while (*s) {
    while (*s == ' ' || *s == '\t' || *s == '\r') ++s;
    if (!*s) break;
    char* e = nullptr;
    errno = 0;
    const unsigned long long v = strtoull(s, &e, 10);
    if (e == s || errno || v > 0xffffffffull) return false;
    if (out && c < max) out[c] = (uint32_t)v;
    ++c;
    s = e;
  }
  *count = c;
  return true;
}

int write_u32_line(FILE* f, const uint32_t* v, int64_t n, uint32_t p, bool prettify) {
  for (int64_t i = 0; i < n; ++i) {
    // prettify_vect (src/matrices.rs:67-71): (x + p) % p
    const uint32_t x = prettify ? (uint32_t)(((uint64_t)v[i] + p) % p) : v[i];
    if (fprintf(f, i ? " %u" : "%u", x) < 0) return -1;
  }
  return fputc('\n', f) == EOF ? -1 : 0;
}

}  // namespace

extern "C" {

int rr_wdm_save(const char* path, int64_t m, int64_t n, uint32_t p, int32_t b, const uint32_t* row_precond,
                const uint32_t* col_precond, const uint32_t* v, const uint32_t* curv, const uint32_t* seq,
                int64_t seq_stride, int64_t nlen) {
  if (!path || !row_precond || !col_precond || !v || !curv || (!seq && nlen > 0)) return fail(RR_EINVAL, "NULL argument");
  if (b < 1 || m < 1 || n < 1 || nlen < 0 || seq_stride < nlen) return fail(RR_EINVAL, "bad sizes");
  File F(fopen(path, "w"));
  if (!F.f) return fail(RR_EIO, "cannot open %s for writing: %s", path, strerror(errno));
  // src/wdm_files.rs:144-205
  if (fprintf(F.f, "%lld %lld %u %lld %d\n", (long long)m, (long long)n, p, (long long)nlen, b) < 0) return fail(RR_EIO, "write failed");
  if (write_u32_line(F.f, row_precond, m, p, false) || write_u32_line(F.f, col_precond, n, p, false))
    return fail(RR_EIO, "write failed");
  for (int i = 0; i < b; ++i)
    if (write_u32_line(F.f, v + (size_t)i * n, n, p, true)) return fail(RR_EIO, "write failed");
  for (int i = 0; i < b; ++i)
    if (write_u32_line(F.f, curv + (size_t)i * n, n, p, true)) return fail(RR_EIO, "write failed");
  for (int q = 0; q < b * (b + 1) / 2; ++q)
    if (write_u32_line(F.f, seq + (size_t)q * seq_stride, nlen, p, false)) return fail(RR_EIO, "write failed");
  if (fflush(F.f)) return fail(RR_EIO, "flush failed");
  return RR_OK;
}

int rr_wdm_load(const char* path, int64_t* m, int64_t* n, uint32_t* p, int32_t* b, int64_t* nlen,
                uint32_t* row_precond, uint32_t* col_precond, uint32_t* v, uint32_t* curv, uint32_t* seq,
                int64_t seq_stride) {
  if (!path || !m || !n || !p || !b || !nlen) return fail(RR_EINVAL, "NULL argument");
  File F(fopen(path, "r"));
  if (!F.f) return fail(RR_EIO, "cannot open %s: %s", path, strerror(errno));
  std::string line;
  // src/wdm_files.rs:36-46
  if (!read_line(F.f, line)) return fail(RR_EIO, "%s: missing header", path);
  long long hm, hn, hl;
  unsigned long long hp;
  int hb;
  if (sscanf(line.c_str(), "%lld %lld %llu %lld %d", &hm, &hn, &hp, &hl, &hb) != 5 || hm < 1 || hn < 1 || hl < 0 ||
      hb < 1 || hp > 0xffffffffull)
    return fail(RR_EIO, "%s: malformed header '%s'", path, line.c_str());
  *m = hm; *n = hn; *p = (uint32_t)hp; *b = hb; *nlen = hl;
  if (!row_precond) return RR_OK;  // header query
  if (!col_precond || !v || !curv || (!seq && hl > 0) || seq_stride < hl) return fail(RR_EINVAL, "NULL array or short stride");
  int64_t cnt = 0;
  if (!read_line(F.f, line) || !parse_u32_line(line, row_precond, hm, &cnt) || cnt != hm)
    return fail(RR_EIO, "%s: row preconditioner length does not match matrix rows", path);
  if (!read_line(F.f, line) || !parse_u32_line(line, col_precond, hn, &cnt) || cnt != hn)
    return fail(RR_EIO, "%s: column preconditioner length does not match matrix columns", path);
  for (int i = 0; i < hb; ++i)
    if (!read_line(F.f, line) || !parse_u32_line(line, v + (size_t)i * hn, hn, &cnt) || cnt != hn)
      return fail(RR_EIO, "%s: v vector length does not match matrix columns", path);
  for (int i = 0; i < hb; ++i)
    if (!read_line(F.f, line) || !parse_u32_line(line, curv + (size_t)i * hn, hn, &cnt) || cnt != hn)
      return fail(RR_EIO, "%s: curv vector length does not match matrix columns", path);
  // sequence lines: the first nlen values are taken (src/wdm_files.rs:99-111)
  for (int q = 0; q < hb * (hb + 1) / 2; ++q)
    if (!read_line(F.f, line) || !parse_u32_line(line, seq + (size_t)q * seq_stride, hl, &cnt) || cnt < hl)
      return fail(RR_EIO, "%s: seq vector length does not match expected sequence length", path);
  return RR_OK;
}

// src/matrices.rs:662-732: "%" comments and blank lines skipped; the first
// 3-field line is the header; entries with a non-positive index are skipped;
// values are reduced mod p with the sign handled as in the reference.  The
// reference expects the entries sorted by row; here they are grouped by row
// with a stable counting sort, so a row-sorted file gives the same CSR and an
// unsorted one still gives a valid matrix.
int rr_sms_load(const char* path, uint32_t p, int64_t* m, int64_t* n, int64_t* nnz, int64_t* rowptr, int32_t* col,
                uint32_t* val) {
  if (!path || !m || !n || !nnz) return fail(RR_EINVAL, "NULL argument");
  if (p < 2 || p >= (1u << 31)) return fail(RR_EPRIME, "p must be in [2, 2^31)");
  File F(fopen(path, "r"));
  if (!F.f) return fail(RR_EIO, "cannot open %s: %s", path, strerror(errno));
  std::string line;
  bool header = false;
  long long hm = 0, hn = 0;
  std::vector<int64_t> rows;
  std::vector<int32_t> cols;
  std::vector<uint32_t> vals;
  while (read_line(F.f, line)) {
    size_t a = line.find_first_not_of(" \t\r");
    if (a == std::string::npos || line[a] == '%') continue;
    char t0[64], t1[64], t2[64], t3[8];
    const int k = sscanf(line.c_str() + a, "%63s %63s %63s %7s", t0, t1, t2, t3);
    if (k != 3) continue;
    if (!header) {
      hm = strtoll(t0, nullptr, 10);
      hn = strtoll(t1, nullptr, 10);
      header = true;
      continue;
    }
    const long long r = strtoll(t0, nullptr, 10), c = strtoll(t1, nullptr, 10);
    const long long x = strtoll(t2, nullptr, 10);
    if (r <= 0 || c <= 0) continue;
    if (r > hm || c > hn) return fail(RR_EIO, "%s: entry (%lld, %lld) outside %lld x %lld", path, r, c, hm, hn);
    long long v = x % (long long)p;
    if (v < 0) v += p;
    rows.push_back(r - 1);
    cols.push_back((int32_t)(c - 1));
    vals.push_back((uint32_t)v);
  }
  if (!header) return fail(RR_EIO, "%s: no header line", path);
  *m = hm;
  *n = hn;
  *nnz = (int64_t)vals.size();
  if (!rowptr) return RR_OK;
  if (!col || !val) return fail(RR_EINVAL, "NULL col/val");
  std::vector<int64_t> cnt(hm + 1, 0);
  for (int64_t r : rows) cnt[r + 1]++;
  for (int64_t i = 0; i < hm; ++i) cnt[i + 1] += cnt[i];
  for (int64_t i = 0; i <= hm; ++i) rowptr[i] = cnt[i];
  // entries keep their file order within a row (stable by row)
  std::vector<int64_t> next(cnt.begin(), cnt.end() - 1);
  for (size_t k = 0; k < rows.size(); ++k) {
    const int64_t pos = next[rows[k]]++;
    col[pos] = cols[k];
    val[pos] = vals[k];
  }
  return RR_OK;
}

}  // extern "C"
