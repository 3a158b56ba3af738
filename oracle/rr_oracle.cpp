// rr_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference (wilthoma/rust_rank) block-Wiedemann rank
// path, used as the parity checker for the CUDA engine and as the timed CPU
// baseline ("port" of the reference CPU algorithm).  Only tests/, the smoke
// entry and bench.py's cpu-baseline / reference arm may load this library;
// the product never links or calls it.
//
// Every function follows the reference function named beside it
// (paths relative to the reference repository root).  All arithmetic is exact
// modulo p: products are reduced through 128-bit intermediates, so the results
// equal the reference's "exact integer, then reduce mod p" semantics wherever
// the reference itself is exact.
//
// Parity pins: the PM-basis / LSP / inverse / rank pieces are pinned against
// the reference's own C++ headers (cuda_test/*.h, built by oracle/Makefile
// into oracle/_ref/) at a small prime; the Krylov sequence is pinned by the
// mathematical identity S_t = V^T B^t V checked with dense big-integer
// arithmetic in the tests and by the known rank of cuda_test/matrix.txt.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef int64_t i64;
typedef unsigned __int128 u128;

namespace {

inline u64 mulmod(u64 a, u64 b, u64 p) {
  // residues are < 2^31, so the product fits in 64 bits (one 64-bit division)
  if ((a | b) < (1ull << 32)) return a * b % p;
  return (u64)((u128)a * b % p);
}
inline u64 addmod(u64 a, u64 b, u64 p) { u64 s = a + b; return s >= p ? s - p : s; }
inline u64 submod(u64 a, u64 b, u64 p) { return a >= b ? a - b : a + p - b; }

// src/ntt.rs:133-151 (mod_pow / modinv by Fermat's little theorem)
u64 powmod(u64 base, u64 e, u64 p) {
  u64 r = 1 % p;
  base %= p;
  while (e) {
    if (e & 1) r = mulmod(r, base, p);
    base = mulmod(base, base, p);
    e >>= 1;
  }
  return r;
}
u64 invmod(u64 a, u64 p) { return powmod(a, p - 2, p); }

// ---------------------------------------------------------------------------
// Sparse matrices (src/matrices.rs:53-64 CsrMatrix, 734-778 transpose)
// ---------------------------------------------------------------------------
struct Csr {
  i64 rows = 0, cols = 0;
  std::vector<i64> ptr;
  std::vector<int32_t> idx;
  std::vector<u64> val;
};

// src/matrices.rs:734-778: counting-sort transpose, stable in the row order.
Csr transpose(const Csr& a) {
  Csr t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.ptr.assign(a.cols + 1, 0);
  for (int32_t c : a.idx) t.ptr[c + 1]++;
  for (i64 i = 0; i < a.cols; ++i) t.ptr[i + 1] += t.ptr[i];
  std::vector<i64> next(t.ptr.begin(), t.ptr.end() - 1);
  t.idx.resize(a.idx.size());
  t.val.resize(a.val.size());
  for (i64 r = 0; r < a.rows; ++r)
    for (i64 k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
      i64 pos = next[a.idx[k]]++;
      t.idx[pos] = (int32_t)r;
      t.val[pos] = a.val[k];
    }
  return t;
}

// src/matrices.rs:780-809 (sparse mat-vec per row, reduced once per row),
// applied to an interleaved block x[col*b + lane] of b vectors at once; every
// lane is the reference's scalar mat-vec of one vector.
void spmm(const Csr& a, const std::vector<u64>& x, std::vector<u64>& y, int b, u64 p) {
  y.assign((size_t)a.rows * b, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (i64 r = 0; r < a.rows; ++r) {
    u128 acc[64];
    for (int l = 0; l < b; ++l) acc[l] = 0;
    for (i64 k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
      const u64 v = a.val[k];
      const u64* xr = &x[(size_t)a.idx[k] * b];
      for (int l = 0; l < b; ++l) acc[l] += (u128)v * xr[l];
    }
    for (int l = 0; l < b; ++l) y[(size_t)r * b + l] = (u64)(acc[l] % p);
  }
}

// src/matrices.rs:152-187 dot_product_mod_p_*: <u, v> mod p.  The reference
// reduces every 100 terms; the value mod p is the same for any grouping.
// Computes all pairs (i <= j) of <x_i, y_j> in the pair order of
// src/main.rs:114-127 (row-major over the upper triangle).
void gram_pairs(const std::vector<u64>& x, const std::vector<u64>& y, i64 len, int b, u64 p,
                std::vector<u64>& out) {
  const int np = b * (b + 1) / 2;
  out.assign(np, 0);
  std::vector<std::pair<int, int>> pairs;
  for (int i = 0; i < b; ++i)
    for (int j = i; j < b; ++j) pairs.push_back({i, j});
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < np; ++q) {
    const int i = pairs[q].first, j = pairs[q].second;
    u128 acc = 0;
    u64 red = 0;
    for (i64 r = 0; r < len; ++r) {
      acc += (u128)x[(size_t)r * b + i] * y[(size_t)r * b + j];
      if ((r & 1023) == 1023) { red = addmod(red, (u64)(acc % p), p); acc = 0; }
    }
    out[q] = addmod(red, (u64)(acc % p), p);
  }
}

// ---------------------------------------------------------------------------
// Dense modular linear algebra (src/modular_linalg.rs)
// ---------------------------------------------------------------------------
struct Mat {
  int r = 0, c = 0;
  std::vector<u64> a;
  Mat() {}
  Mat(int r_, int c_) : r(r_), c(c_), a((size_t)r_ * c_, 0) {}
  u64& operator()(int i, int j) { return a[(size_t)i * c + j]; }
  u64 operator()(int i, int j) const { return a[(size_t)i * c + j]; }
};

// src/modular_linalg.rs:188-239 lsp_decomposition: for each row k, the pivot
// is the first column j >= rank (in the current, swapped column order) with a
// non-zero entry; columns rank and j are swapped, rows below are eliminated and
// the factors are stored in L[i][k].
void lsp_decomposition(const Mat& in, u64 p, Mat& L, Mat& S, std::vector<int>& perm) {
  const int m = in.r;
  Mat a = in;
  L = Mat(m, m);
  for (int i = 0; i < m; ++i) L(i, i) = 1;
  perm.resize(m);
  std::iota(perm.begin(), perm.end(), 0);
  int rank = 0;
  for (int k = 0; k < m; ++k) {
    int pc = -1;
    for (int j = rank; j < m; ++j)
      if (a(k, j) % p != 0) { pc = j; break; }
    if (pc < 0) continue;
    for (int i = 0; i < m; ++i) std::swap(a(i, rank), a(i, pc));
    std::swap(perm[rank], perm[pc]);
    const u64 pinv = invmod(a(k, rank), p);
    for (int i = k + 1; i < m; ++i) {
      const u64 f = mulmod(a(i, rank), pinv, p);
      L(i, k) = f;
      for (int col = rank; col < m; ++col) {
        const u64 sub = mulmod(f, a(k, col), p);
        a(i, col) = submod(a(i, col) % p, sub, p);
      }
    }
    ++rank;
  }
  S = a;
  for (auto& v : S.a) v %= p;
}

// src/modular_linalg.rs:10-69 matrix_inverse: Gauss-Jordan on [A | I].
// Returns false when the matrix is singular (the reference panics).
bool matrix_inverse(const Mat& m_in, u64 p, Mat& out) {
  const int n = m_in.r;
  Mat aug(n, 2 * n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) aug(i, j) = m_in(i, j) % p;
    aug(i, n + i) = 1;
  }
  for (int i = 0; i < n; ++i) {
    if (aug(i, i) == 0) {
      bool found = false;
      for (int j = i + 1; j < n; ++j)
        if (aug(j, i) != 0) {
          for (int k = 0; k < 2 * n; ++k) std::swap(aug(i, k), aug(j, k));
          found = true;
          break;
        }
      if (!found) return false;
    }
    const u64 inv = invmod(aug(i, i), p);
    for (int k = 0; k < 2 * n; ++k) aug(i, k) = mulmod(aug(i, k), inv, p);
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const u64 f = aug(j, i);
      for (int k = 0; k < 2 * n; ++k) {
        const u64 t = mulmod(aug(i, k), f, p);
        aug(j, k) = submod(aug(j, k), t, p);
      }
    }
  }
  out = Mat(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out(i, j) = aug(i, n + j);
  return true;
}

// src/modular_linalg.rs:132-183 modular_rank: column-by-column pivot search
// from row `rank`, row swap, normalise, eliminate below.
i64 modular_rank(Mat mat, u64 p) {
  const int nr = mat.r, nc = mat.c;
  for (auto& v : mat.a) v %= p;
  int rank = 0;
  for (int col = 0; col < nc; ++col) {
    int pr = -1;
    for (int row = rank; row < nr; ++row)
      if (mat(row, col) != 0) { pr = row; break; }
    if (pr < 0) continue;
    for (int j = 0; j < nc; ++j) std::swap(mat(rank, j), mat(pr, j));
    const u64 inv = invmod(mat(rank, col), p);
    for (int j = col; j < nc; ++j) mat(rank, j) = mulmod(mat(rank, j), inv, p);
    for (int row = rank + 1; row < nr; ++row) {
      const u64 f = mat(row, col);
      if (!f) continue;
      for (int j = col; j < nc; ++j) {
        const u64 sub = mulmod(f, mat(rank, j), p);
        mat(row, j) = submod(mat(row, j), sub, p);
      }
    }
    ++rank;
    if (rank == nr) break;
  }
  return rank;
}

// ---------------------------------------------------------------------------
// Polynomial matrices and NTT products (src/poly_mat_mul.rs, src/ntt.rs)
// ---------------------------------------------------------------------------
// PolyMat: rows x cols x len, flat [i][j][k].
struct PolyMat {
  int rows = 0, cols = 0;
  i64 len = 0;
  std::vector<u64> a;
  PolyMat() {}
  PolyMat(int r, int c, i64 l) : rows(r), cols(c), len(l), a((size_t)r * c * l, 0) {}
  u64* at(int i, int j) { return &a[((size_t)i * cols + j) * len]; }
  const u64* at(int i, int j) const { return &a[((size_t)i * cols + j) * len]; }
};

// Smallest generator of F_p^* (p prime).  For p = 2013265921 this is 31, the
// root the reference uses (src/ntt.rs:51-53).
u64 find_generator(u64 p) {
  std::vector<u64> fac;
  u64 t = p - 1;
  for (u64 q = 2; q * q <= t; ++q)
    if (t % q == 0) { fac.push_back(q); while (t % q == 0) t /= q; }
  if (t > 1) fac.push_back(t);
  for (u64 g = 2; g < p; ++g) {
    bool ok = true;
    for (u64 q : fac)
      if (powmod(g, (p - 1) / q, p) == 1) { ok = false; break; }
    if (ok) return g;
  }
  return 0;
}

// src/ntt.rs:164-211: radix-2 decimation-in-time NTT, bit reversal first,
// per-stage root wlen = root^(n/len); inverse uses root^-1 and scales by n^-1.
void ntt(u64* a, i64 n, bool invert, u64 p, u64 g) {
  int bits = 0;
  while ((1LL << bits) < n) ++bits;
  for (i64 i = 0, j = 0; i < n; ++i) {
    if (i < j) std::swap(a[i], a[j]);
    i64 bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
  }
  u64 root = powmod(g, (p - 1) / n, p);
  if (invert) root = invmod(root, p);
  for (i64 len = 2; len <= n; len <<= 1) {
    const u64 wlen = powmod(root, n / len, p);
    for (i64 s = 0; s < n; s += len) {
      u64 w = 1;
      for (i64 k = 0; k < len / 2; ++k) {
        const u64 u = a[s + k], v = mulmod(a[s + k + len / 2], w, p);
        a[s + k] = addmod(u, v, p);
        a[s + k + len / 2] = submod(u, v, p);
        w = mulmod(w, wlen, p);
      }
    }
  }
  if (invert) {
    const u64 ninv = invmod((u64)n % p, p);
    for (i64 i = 0; i < n; ++i) a[i] = mulmod(a[i], ninv, p);
  }
}

// Product modulo the NTT prime q (q - 1 divisible by L): out[i][j][0..lres).
// Inputs are reduced mod q first (they are residues mod p, p < 2^31).
void ntt_matmul(const PolyMat& A, const PolyMat& B, i64 b_start, i64 lb, i64 L, u64 q, std::vector<u64>& out) {
  const int m = A.rows, n = A.cols, k = B.cols;
  const i64 la = A.len, lres = la + lb - 1;
  const u64 g = find_generator(q);
  std::vector<u64> fa((size_t)m * n * L, 0), fb((size_t)n * k * L, 0);
  out.assign((size_t)m * k * lres, 0);
#pragma omp parallel for collapse(2)
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      u64* d = &fa[((size_t)i * n + j) * L];
      for (i64 t = 0; t < la; ++t) d[t] = A.at(i, j)[t] % q;
      ntt(d, L, false, q, g);
    }
#pragma omp parallel for collapse(2)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) {
      u64* d = &fb[((size_t)i * k + j) * L];
      for (i64 t = 0; t < lb; ++t) d[t] = B.at(i, j)[b_start + t] % q;
      ntt(d, L, false, q, g);
    }
#pragma omp parallel for collapse(2)
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j) {
      // lazy sums: three products (< 3 q^2 < 2^64 - q) between reductions
      std::vector<u64> d(L, 0);
      for (int r = 0; r < n; ++r) {
        const u64* x = &fa[((size_t)i * n + r) * L];
        const u64* y = &fb[((size_t)r * k + j) * L];
        for (i64 l = 0; l < L; ++l) d[l] += x[l] * y[l];
        if (r % 3 == 2 || r == n - 1)
          for (i64 l = 0; l < L; ++l) d[l] %= q;
      }
      ntt(d.data(), L, true, q, g);
      std::memcpy(&out[((size_t)i * k + j) * lres], d.data(), sizeof(u64) * lres);
    }
}

// src/poly_mat_mul.rs:89-101, 113-256: C = A * B where only coefficients
// [b_start, b_end) of B take part; output length la + nlenb - 1, reduced mod p.
// The reference multiplies exactly over a large NTT prime and then reduces
// (src/poly_mat_mul.rs:240-256 over the prime of src/ntt.rs:60-75).  Here:
// directly mod p when p is NTT-friendly for the padded length; otherwise the
// exact integer product by CRT over three NTT primes (their product, ~2^92.9,
// exceeds inner dimension x length x (p-1)^2 for every size used here), reduced
// mod p; schoolbook for short products.  All give the same value mod p.
PolyMat poly_mat_mul_red(const PolyMat& A, const PolyMat& B, u64 p, i64 b_start, i64 b_end) {
  const int m = A.rows, n = A.cols, k = B.cols;
  const i64 la = A.len;
  const i64 lb = std::min(B.len, b_end - b_start);
  const i64 lres = la + lb - 1;
  PolyMat C(m, k, lres);
  i64 L = 1;
  while (L < lres) L <<= 1;
  if (lres > 32 && (p - 1) % (u64)L == 0) {
    std::vector<u64> out;
    ntt_matmul(A, B, b_start, lb, L, p, out);
    C.a = std::move(out);
  } else if (lres > 32) {
    static const u64 Q[3] = {2013265921ull, 2113929217ull, 2130706433ull};
    std::vector<u64> r[3];
    for (int i = 0; i < 3; ++i) ntt_matmul(A, B, b_start, lb, L, Q[i], r[i]);
    const u128 q01 = (u128)Q[0] * Q[1];
    const u64 c01 = invmod(Q[0] % Q[1], Q[1]), c02 = invmod(Q[0] % Q[2], Q[2]), c12 = invmod(Q[1] % Q[2], Q[2]);
#pragma omp parallel for
    for (i64 t = 0; t < (i64)C.a.size(); ++t) {
      const u64 x0 = r[0][t];
      const u64 x1 = mulmod(submod(r[1][t], x0 % Q[1], Q[1]), c01, Q[1]);
      const u64 t2 = mulmod(submod(r[2][t], x0 % Q[2], Q[2]), c02, Q[2]);
      const u64 x2 = mulmod(submod(t2, x1 % Q[2], Q[2]), c12, Q[2]);
      const u128 v = (u128)x0 + (u128)x1 * Q[0] + (u128)x2 * q01;
      C.a[t] = (u64)(v % p);
    }
  } else {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < k; ++j) {
        std::vector<u128> acc(lres, 0);
        for (int r = 0; r < n; ++r) {
          const u64* x = A.at(i, r);
          const u64* y = B.at(r, j) + b_start;
          for (i64 s = 0; s < la; ++s) {
            if (!x[s]) continue;
            for (i64 t = 0; t < lb; ++t) acc[s + t] += (u128)x[s] * y[t];
          }
          if (((r + 1) & 15) == 0)
            for (auto& v : acc) v %= p;
        }
        u64* c = C.at(i, j);
        for (i64 s = 0; s < lres; ++s) c[s] = (u64)(acc[s] % p);
      }
  }
  return C;
}

// src/sigma_basis.rs:283-294 shift_trunc_in.
void shift_trunc_in(PolyMat& M, i64 shiftd, i64 truncd) {
  PolyMat R(M.rows, M.cols, truncd + 1);
  for (int i = 0; i < M.rows; ++i)
    for (int j = 0; j < M.cols; ++j)
      for (i64 k = 0; k <= truncd; ++k) R.at(i, j)[k] = (k + shiftd < M.len) ? M.at(i, j)[k + shiftd] : 0;
  M = std::move(R);
}

// src/sigma_basis.rs:348-416 M_Basis: order-1 basis of the constant
// coefficient of G under the shift delta.
bool M_Basis(const PolyMat& G, std::vector<i64>& delta, u64 p, PolyMat& out) {
  const int m = G.rows, n = G.cols;
  // stable sort of the row indices by delta, descending (Rust sort_by is stable)
  std::vector<int> perm(m);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return delta[a] > delta[b]; });
  std::vector<i64> sdelta(m);
  for (int i = 0; i < m; ++i) sdelta[i] = delta[perm[i]];
  // Delta = pi * G[.][.][0], augmented to m x m with zero columns
  Mat Daug(m, m);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) Daug(i, j) = G.at(perm[i], j)[0];
  Mat L, S;
  std::vector<int> cperm;
  lsp_decomposition(Daug, p, L, S, cperm);
  Mat Linv;
  if (!matrix_inverse(L, p, Linv)) return false;
  out = PolyMat(m, m, 2);
  for (int i = 0; i < m; ++i) {
    bool zero_row = true;
    for (int j = 0; j < m; ++j)
      if (S(i, j)) { zero_row = false; break; }
    // row i of Linv * pi: (Linv*pi)[i][perm[t]] = Linv[i][t]
    for (int t = 0; t < m; ++t) out.at(i, perm[t])[zero_row ? 0 : 1] = Linv(i, t);
    if (!zero_row) sdelta[i] -= 1;
  }
  delta = sdelta;
  return true;
}

// src/sigma_basis.rs:190-219 _PM_Basis divide and conquer.
bool PM_rec(const PolyMat& G, i64 d, std::vector<i64>& delta, u64 p, PolyMat& out) {
  if (d == 0) {  // unit_mat, src/sigma_basis.rs:274-280
    out = PolyMat(G.rows, G.rows, 1);
    for (int i = 0; i < G.rows; ++i) out.at(i, i)[0] = 1;
    return true;
  }
  if (d == 1) return M_Basis(G, delta, p, out);
  PolyMat MM;
  if (!PM_rec(G, d / 2, delta, p, MM)) return false;
  PolyMat GG = poly_mat_mul_red(MM, G, p, 0, d + 1);
  shift_trunc_in(GG, d / 2, d / 2);
  PolyMat MMM;
  if (!PM_rec(GG, d / 2, delta, p, MMM)) return false;
  out = poly_mat_mul_red(MMM, MM, p, 0, MM.len);
  return true;
}

}  // namespace

extern "C" {

int orc_num_threads(int nt) {
#ifdef _OPENMP
  if (nt > 0) omp_set_num_threads(nt);
  return omp_get_max_threads();
#else
  (void)nt;
  return 1;
#endif
}

// Krylov sequence, restating src/main.rs:88-216 (main_loop_s_mt2) fed by
// src/vectorstream.rs:46-91 (one worker per vector: curw = a*v, then
// repeatedly vec = at*curw, curw = a*vec) with the operator prepared as in
// src/main.rs:522-526 (at = transpose(A) before scaling; a = D_r A D_c;
// at = D_c A^T).
//
// val holds matrix entries already reduced to [0, p).  curv (b x n,
// vector-major, like Vec<Vec<T>>) is the current block and is updated in
// place.  seq is [b(b+1)/2][seq_stride]; entries [seq_len, result) are written.
// Returns the new sequence length, or -1 on bad arguments.
i64 orc_krylov(i64 m, i64 n, const i64* rowptr, const int32_t* col, const uint32_t* val, uint32_t p_,
               int b, const uint32_t* row_precond, const uint32_t* col_precond, uint32_t* curv,
               i64 seq_len, i64 max_nlen, uint32_t* seq, i64 seq_stride) {
  const u64 p = p_;
  if (b < 1 || b > 64 || m < 1 || n < 1) return -1;
  Csr a;
  a.rows = m;
  a.cols = n;
  a.ptr.assign(rowptr, rowptr + m + 1);
  const i64 nnz = rowptr[m];
  a.idx.assign(col, col + nnz);
  a.val.assign(val, val + nnz);
  Csr at = transpose(a);
  // scale_csr_matrix_rows / columns (src/matrices.rs:813-840)
  for (i64 r = 0; r < m; ++r)
    for (i64 k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
      a.val[k] = mulmod(a.val[k], row_precond[r], p);
      a.val[k] = mulmod(a.val[k], col_precond[a.idx[k]], p);
    }
  for (i64 c = 0; c < n; ++c)
    for (i64 k = at.ptr[c]; k < at.ptr[c + 1]; ++k) at.val[k] = mulmod(at.val[k], col_precond[c], p);

  const int np = b * (b + 1) / 2;
  std::vector<u64> x((size_t)n * b), y, w, g;
  for (int l = 0; l < b; ++l)
    for (i64 c = 0; c < n; ++c) x[(size_t)c * b + l] = curv[(size_t)l * n + c] % p;

  i64 len = seq_len;
  const i64 to_be_produced = max_nlen - seq_len;
  if (to_be_produced < 0) return -1;
  if (len == 0) {
    gram_pairs(x, x, n, b, p, g);
    for (int q = 0; q < np; ++q) seq[(size_t)q * seq_stride + len] = (uint32_t)g[q];
    ++len;
  }
  for (i64 it = 0; it < to_be_produced / 2; ++it) {
    spmm(a, x, y, b, p);   // curw = a * curv
    spmm(at, y, w, b, p);  // vec = at * curw
    gram_pairs(x, w, n, b, p, g);
    for (int q = 0; q < np; ++q) seq[(size_t)q * seq_stride + len] = (uint32_t)g[q];
    gram_pairs(w, w, n, b, p, g);
    for (int q = 0; q < np; ++q) seq[(size_t)q * seq_stride + len + 1] = (uint32_t)g[q];
    len += 2;
    x.swap(w);
  }
  for (int l = 0; l < b; ++l)
    for (i64 c = 0; c < n; ++c) curv[(size_t)l * n + c] = (uint32_t)x[(size_t)c * b + l];
  return len;
}

// The same Krylov step as orc_krylov, split so the CPU baseline can time
// individual applications of B: orc_op_create prepares a = D_r A D_c and
// at = D_c A^T once (src/main.rs:522-526); orc_op_step runs one worker
// iteration plus the consumer's two dot-product terms (src/vectorstream.rs:63-64,
// src/main.rs:138-156) on an interleaved block x (n x b), in place.
struct OrcOp {
  Csr a, at;
  u64 p;
  int b;
  std::vector<u64> x, y, w, g;
};

void* orc_op_create(i64 m, i64 n, const i64* rowptr, const int32_t* col, const uint32_t* val, uint32_t p, int b,
                    const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* curv) {
  OrcOp* op = new OrcOp;
  op->p = p;
  op->b = b;
  op->a.rows = m;
  op->a.cols = n;
  op->a.ptr.assign(rowptr, rowptr + m + 1);
  op->a.idx.assign(col, col + rowptr[m]);
  op->a.val.assign(val, val + rowptr[m]);
  op->at = transpose(op->a);
  for (i64 r = 0; r < m; ++r)
    for (i64 k = op->a.ptr[r]; k < op->a.ptr[r + 1]; ++k)
      op->a.val[k] = mulmod(mulmod(op->a.val[k], row_precond[r], p), col_precond[op->a.idx[k]], p);
  for (i64 c = 0; c < n; ++c)
    for (i64 k = op->at.ptr[c]; k < op->at.ptr[c + 1]; ++k) op->at.val[k] = mulmod(op->at.val[k], col_precond[c], p);
  op->x.resize((size_t)n * b);
  for (int l = 0; l < b; ++l)
    for (i64 c = 0; c < n; ++c) op->x[(size_t)c * b + l] = curv[(size_t)l * n + c] % p;
  return op;
}

int orc_op_step(void* h, uint32_t* gram_odd, uint32_t* gram_even) {
  OrcOp* op = static_cast<OrcOp*>(h);
  const int b = op->b, np = b * (b + 1) / 2;
  spmm(op->a, op->x, op->y, b, op->p);
  spmm(op->at, op->y, op->w, b, op->p);
  gram_pairs(op->x, op->w, op->a.cols, b, op->p, op->g);
  for (int q = 0; q < np; ++q) gram_odd[q] = (uint32_t)op->g[q];
  gram_pairs(op->w, op->w, op->a.cols, b, op->p, op->g);
  for (int q = 0; q < np; ++q) gram_even[q] = (uint32_t)op->g[q];
  op->x.swap(op->w);
  return 0;
}

void orc_op_destroy(void* h) { delete static_cast<OrcOp*>(h); }

// src/modular_linalg.rs:188-239.  a, L, S are m x m row-major; perm gets the
// column permutation (perm[i] = original column now at position i).
int orc_lsp(int m, const uint64_t* a, uint64_t p, uint64_t* L, uint64_t* S, int32_t* perm) {
  Mat A(m, m);
  std::copy(a, a + (size_t)m * m, A.a.begin());
  Mat Lm, Sm;
  std::vector<int> pr;
  lsp_decomposition(A, p, Lm, Sm, pr);
  std::copy(Lm.a.begin(), Lm.a.end(), L);
  std::copy(Sm.a.begin(), Sm.a.end(), S);
  for (int i = 0; i < m; ++i) perm[i] = pr[i];
  return 0;
}

// src/modular_linalg.rs:10-69.  Returns 0, or 1 when singular.
int orc_matrix_inverse(int n, const uint64_t* a, uint64_t p, uint64_t* out) {
  Mat A(n, n);
  std::copy(a, a + (size_t)n * n, A.a.begin());
  Mat R;
  if (!matrix_inverse(A, p, R)) return 1;
  std::copy(R.a.begin(), R.a.end(), out);
  return 0;
}

// src/modular_linalg.rs:132-183.
i64 orc_modular_rank(int rows, int cols, const uint64_t* a, uint64_t p) {
  Mat A(rows, cols);
  std::copy(a, a + (size_t)rows * cols, A.a.begin());
  return modular_rank(A, p);
}

// Dense rank of a sparse matrix given in CSR (values in [0,p)), by the same
// elimination as modular_rank; used for known-rank checks of small matrices.
i64 orc_dense_rank_csr(i64 m, i64 n, const i64* rowptr, const int32_t* col, const uint32_t* val,
                       uint64_t p) {
  if ((double)m * (double)n > 6e8) return -1;
  // eliminate on rows (rank(A) = rank(A^T)); use the smaller side as columns
  const bool tr = n > m;
  const int R = (int)(tr ? n : m), C = (int)(tr ? m : n);
  std::vector<uint32_t> d((size_t)R * C, 0);
  for (i64 r = 0; r < m; ++r)
    for (i64 k = rowptr[r]; k < rowptr[r + 1]; ++k) {
      size_t pos = tr ? (size_t)col[k] * C + r : (size_t)r * C + col[k];
      d[pos] = (uint32_t)(((u64)d[pos] + val[k]) % p);
    }
  int rank = 0;
  for (int c = 0; c < C && rank < R; ++c) {
    int pr = -1;
    for (int r = rank; r < R; ++r)
      if (d[(size_t)r * C + c]) { pr = r; break; }
    if (pr < 0) continue;
    if (pr != rank)
      for (int j = 0; j < C; ++j) std::swap(d[(size_t)rank * C + j], d[(size_t)pr * C + j]);
    const u64 inv = invmod(d[(size_t)rank * C + c], p);
    uint32_t* prow = &d[(size_t)rank * C];
    for (int j = c; j < C; ++j) prow[j] = (uint32_t)mulmod(prow[j], inv, p);
#pragma omp parallel for schedule(static)
    for (int r = rank + 1; r < R; ++r) {
      uint32_t* row = &d[(size_t)r * C];
      const u64 f = row[c];
      if (!f) continue;
      const u64 nf = p - f;
      for (int j = c; j < C; ++j) row[j] = (uint32_t)((row[j] + (u128)nf * prow[j]) % p);
    }
    ++rank;
  }
  return rank;
}

// src/poly_mat_mul.rs:240-256 (poly_mat_mul_fft_red).  a: m x n x la,
// b: n x k x lb; out: m x k x (la + min(lb, b_end-b_start) - 1).
int orc_poly_mat_mul(int m, int n, int k, i64 la, i64 lb, const uint64_t* a, const uint64_t* b, uint64_t p,
                     i64 b_start, i64 b_end, uint64_t* out) {
  PolyMat A(m, n, la), B(n, k, lb);
  std::copy(a, a + A.a.size(), A.a.begin());
  std::copy(b, b + B.a.size(), B.a.begin());
  PolyMat C = poly_mat_mul_red(A, B, p, b_start, b_end);
  std::copy(C.a.begin(), C.a.end(), out);
  return 0;
}

// src/ntt.rs:164-211 on one array (length a power of two dividing p-1).
int orc_ntt(uint64_t* a, i64 n, int invert, uint64_t p) {
  if (n < 1 || (n & (n - 1)) || (p - 1) % (u64)n) return 1;
  ntt(a, n, invert != 0, p, find_generator(p));
  return 0;
}

uint64_t orc_generator(uint64_t p) { return find_generator(p); }

// src/sigma_basis.rs:9-54 PM_Basis.  seq is [b(b+1)/2][seq_stride] with nlen
// valid terms.  d is enlarged to a power of two and must be < nlen.
// M_out: [2b][2b][d+1]; delta_out: 2b.  Returns 0, 1 on bad arguments,
// 2 when a leaf basis hits a singular L (cannot happen for exact arithmetic).
int orc_pm_basis(const uint32_t* seq, int b, i64 nlen, i64 seq_stride, i64 d, uint32_t p, uint64_t* M_out,
                 int64_t* delta_out) {
  i64 dd = 1;
  while (dd < d) dd *= 2;
  d = dd;
  if (d >= nlen || b < 1) return 1;
  PolyMat G(2 * b, b, nlen);
  int ii = 0;
  for (int i = 0; i < b; ++i)
    for (int j = i; j < b; ++j) {
      for (i64 k = 0; k < nlen; ++k) {
        G.at(i, j)[k] = seq[(size_t)ii * seq_stride + k] % p;
        G.at(j, i)[k] = G.at(i, j)[k];
      }
      ++ii;
    }
  for (int i = 0; i < b; ++i) G.at(b + i, i)[0] = 1;
  std::vector<i64> delta(2 * b, 0);
  PolyMat M;
  if (!PM_rec(G, d, delta, p, M)) return 2;
  if (M.len != d + 1) return 3;
  std::copy(M.a.begin(), M.a.end(), M_out);
  for (int i = 0; i < 2 * b; ++i) delta_out[i] = delta[i];
  return 0;
}

// src/sigma_basis.rs:71-152 analyze_pm_basis followed by
// src/blockbmtest.rs:574-599 analyze_min_generators: the estimated rank
// b*(k-3) + rank(P[k-1]) + rank(P[0]) of the reversed upper-left block.
// M: [2b][2b][len].  Returns the rank, or -1 when k < 3 (the reference's
// unsigned arithmetic has no meaningful value there).
i64 orc_rank_from_basis(const uint64_t* M, const int64_t* delta, int b, i64 len, uint64_t p) {
  const int n2 = 2 * b;
  i64 maxdel = 0;
  for (int i = 0; i < b; ++i) {
    if (-delta[i] < 0 || -delta[i] >= len) return -2;
    maxdel = std::max<i64>(maxdel, -delta[i]);
  }
  // basisrev[i][j][k] = basis[i][j][del_i - k], k <= del_i
  std::vector<u64> rev((size_t)(maxdel + 1) * b * b, 0);  // [k][i][j]
  i64 maxdeg = 0;
  for (int i = 0; i < b; ++i) {
    const i64 del = -delta[i];
    for (int j = 0; j < b; ++j)
      for (i64 k = 0; k <= del; ++k) {
        const u64 v = M[((size_t)i * n2 + j) * len + (del - k)];
        rev[((size_t)k * b + i) * b + j] = v;
        if (v != 0 && k > maxdeg) maxdeg = k;
      }
  }
  const i64 kk = maxdeg + 1;
  if (kk < 3) return -1;
  Mat P0(b, b), Pk(b, b);
  for (int i = 0; i < b; ++i)
    for (int j = 0; j < b; ++j) {
      P0(i, j) = rev[((size_t)0 * b + i) * b + j];
      Pk(i, j) = rev[((size_t)(kk - 1) * b + i) * b + j];
    }
  return (i64)b * (kk - 3) + modular_rank(Pk, p) + modular_rank(P0, p);
}

}  // extern "C"
