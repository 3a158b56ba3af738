// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Thin extern "C" wrapper around the reference's own host C++ PM-basis code
// (cuda_test/sigma_basis.h, poly_mat_mul.h, ntt.h, modular_linalg.h of
// wilthoma/rust_rank), compiled in place from the reference checkout by
// oracle/Makefile into oracle/_ref/libref.so.  It exists to pin the oracle's
// restatement (rr_oracle.cpp) against the reference itself: the tests call
// both on the same inputs and require identical outputs.
//
// Validity of the reference code paths used here (u64 instantiation):
//  * its NTT works over 2^61 - 2^26 + 1, so products are exact only while
//    p^2 * len * inner < 2^61 (small primes such as 3323);
//  * M_Basis sorts delta with std::sort, which equals the stable sort of the
//    Rust original only for at most 16 rows (2b <= 16).
// The tests stay inside both limits.

#include <chrono>
#include <cstdint>
#include <iomanip>
#include <map>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>
using namespace std;
#include "sigma_basis.h"

typedef uint64_t u64;

extern "C" {

// PM_Basis<u64,u64> (cuda_test/sigma_basis.h:214-263).  seq: [b(b+1)/2][stride].
int ref_pm_basis(const u64* seq, int b, int64_t nlen, int64_t stride, int64_t d, u64 p, u64* M_out,
                 int64_t* delta_out, int64_t* len_out) {
  vector<vector<u64>> s(b * (b + 1) / 2, vector<u64>(nlen));
  for (size_t q = 0; q < s.size(); ++q)
    for (int64_t k = 0; k < nlen; ++k) s[q][k] = seq[q * stride + k];
  auto res = PM_Basis<u64, u64>(s, (size_t)d, p);
  auto& M = res.first;
  auto& delta = res.second;
  const size_t n2 = M.size(), len = M[0][0].size();
  for (size_t i = 0; i < n2; ++i)
    for (size_t j = 0; j < n2; ++j)
      for (size_t k = 0; k < len; ++k) M_out[(i * n2 + j) * len + k] = M[i][j][k];
  for (size_t i = 0; i < n2; ++i) delta_out[i] = delta[i];
  *len_out = (int64_t)len;
  return 0;
}

// analyze_pm_basis<u64> (cuda_test/sigma_basis.h:305-360); the estimated rank
// is read back from the text the reference prints.
int64_t ref_rank_from_basis(const u64* M, const int64_t* delta, int b, int64_t len, u64 p) {
  const int n2 = 2 * b;
  vector<vector<vector<u64>>> basis(n2, vector<vector<u64>>(n2, vector<u64>(len)));
  for (int i = 0; i < n2; ++i)
    for (int j = 0; j < n2; ++j)
      for (int64_t k = 0; k < len; ++k) basis[i][j][k] = M[((size_t)i * n2 + j) * len + k];
  vector<int64_t> dl(delta, delta + n2);
  std::ostringstream cap;
  auto* old = std::cout.rdbuf(cap.rdbuf());
  analyze_pm_basis<u64>(basis, dl, p);
  std::cout.rdbuf(old);
  const string text = cap.str();
  const string key = "Estimated matrix rank: ";
  const size_t pos = text.rfind(key);
  if (pos == string::npos) return -1;
  return (int64_t)std::stoull(text.substr(pos + key.size()));
}

// lsp_decomposition<u64> (cuda_test/modular_linalg.h:287-360).
int ref_lsp(int m, const u64* a, u64 p, u64* L, u64* S, u64* P) {
  DMatrix<u64> A(m, m);
  for (int i = 0; i < m * m; ++i) A.data[i] = a[i];
  auto [l, s, pm] = lsp_decomposition(A, p);
  for (int i = 0; i < m * m; ++i) { L[i] = l.data[i]; S[i] = s.data[i]; P[i] = pm.data[i]; }
  return 0;
}

// matrix_inverse<u64> (cuda_test/modular_linalg.h:107-171).
int ref_matrix_inverse(int n, const u64* a, u64 p, u64* out) {
  DMatrix<u64> A(n, n);
  for (int i = 0; i < n * n; ++i) A.data[i] = a[i];
  auto r = matrix_inverse(A, p);
  for (int i = 0; i < n * n; ++i) out[i] = r.data[i];
  return 0;
}

// modular_rank<u64> (cuda_test/modular_linalg.h:234-285).
int64_t ref_modular_rank(int rows, int cols, const u64* a, u64 p) {
  DMatrix<u64> A(rows, cols);
  for (int i = 0; i < rows * cols; ++i) A.data[i] = a[i];
  return (int64_t)modular_rank(A, p);
}

// poly_mat_mul_fft_red<u64> (cuda_test/poly_mat_mul.h:226-250).
int ref_poly_mat_mul(int m, int n, int k, int64_t la, int64_t lb, const u64* a, const u64* b, u64 p,
                     int64_t b_start, int64_t b_end, u64* out, int64_t* len_out) {
  vector<vector<vector<u64>>> A(m, vector<vector<u64>>(n, vector<u64>(la)));
  vector<vector<vector<u64>>> B(n, vector<vector<u64>>(k, vector<u64>(lb)));
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j)
      for (int64_t l = 0; l < la; ++l) A[i][j][l] = a[((size_t)i * n + j) * la + l];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j)
      for (int64_t l = 0; l < lb; ++l) B[i][j][l] = b[((size_t)i * k + j) * lb + l];
  auto C = poly_mat_mul_fft_red(A, B, p, (size_t)b_start, (size_t)b_end);
  const size_t len = C[0][0].size();
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < k; ++j)
      for (size_t l = 0; l < len; ++l) out[((size_t)i * k + j) * len + l] = C[i][j][l];
  *len_out = (int64_t)len;
  return 0;
}

}  // extern "C"
