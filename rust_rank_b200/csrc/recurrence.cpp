// recurrence.cpp -- host checks around the minimal generator: the generator
// test of src/blockbmtest.rs:445-461 and the scalar Berlekamp-Massey call
// surface of src/block_berlekamp_massey.rs:104-131 (block width 1).
//
// Both are verification / small-case utilities in the reference (the rank
// driver uses the PM-basis), so they run on the host: the generator test is
// split over the host's threads, Berlekamp-Massey is inherently sequential.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "rr_internal.h"

using namespace rr;

extern "C" {

int rr_is_generating_poly(const uint32_t* poly, int64_t k, const uint32_t* seq, int64_t N, int32_t n, uint32_t p,
                          int32_t* is_gen) {
  if (!poly || !seq || !is_gen) return fail(RR_EINVAL, "NULL argument");
  RR_TRY(rr_prime_check(p));
  if (n < 1 || k < 1) return fail(RR_EINVAL, "n = %d and k = %lld must be positive", n, (long long)k);
  // the reference iterates l in 0..N-k (an unsigned range): N < k has no meaning there
  if (N < k) return fail(RR_EINVAL, "sequence of %lld terms shorter than the polynomial (%lld)", (long long)N, (long long)k);
  const int64_t nn = (int64_t)n * n;
  for (int64_t i = 0; i < k * nn; ++i)
    if (poly[i] >= p) return fail(RR_EINVAL, "poly entry %lld not reduced mod p", (long long)i);
  for (int64_t i = 0; i < N * nn; ++i)
    if (seq[i] >= p) return fail(RR_EINVAL, "seq entry %lld not reduced mod p", (long long)i);
  const int64_t windows = N - k;
  // the first failing window (windows = none); threads skip windows past it
  std::atomic<int64_t> first_bad{windows};
  auto check = [&](int64_t l) {
    // sum_{i<k} seq[l+i] * poly[i] (n x n); every entry < 2^62 * k * n fits
    // an unsigned 128-bit accumulator
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) {
        unsigned __int128 acc = 0;
        for (int64_t i = 0; i < k; ++i) {
          const uint32_t* S = seq + (l + i) * nn + (int64_t)r * n;
          const uint32_t* Q = poly + i * nn + c;
          for (int t = 0; t < n; ++t) acc += (uint64_t)S[t] * Q[(int64_t)t * n];
        }
        if ((uint64_t)(acc % p) != 0) return false;
      }
    return true;
  };
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(windows, std::max(1u, std::thread::hardware_concurrency())));
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (int64_t l = next.fetch_add(1); l < windows; l = next.fetch_add(1)) {
      if (l >= first_bad.load()) break;
      if (!check(l)) {
        int64_t cur = first_bad.load();
        while (l < cur && !first_bad.compare_exchange_weak(cur, l)) {
        }
      }
    }
  };
  if (nt == 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
  }
  *is_gen = first_bad.load() == windows ? 1 : 0;
  return RR_OK;
}

int rr_berlekamp_massey(const uint32_t* seq, int64_t n, uint32_t p, uint32_t* conn, int64_t* L_out) {
  if ((!seq && n > 0) || !conn || !L_out) return fail(RR_EINVAL, "NULL argument");
  RR_TRY(rr_prime_check(p));
  if (n < 0) return fail(RR_EINVAL, "n < 0");
  for (int64_t i = 0; i < n; ++i)
    if (seq[i] >= p) return fail(RR_EINVAL, "seq entry %lld not reduced mod p", (long long)i);
  // Massey (1969): C is the current connection polynomial of length L, B the
  // one before the last length change, bd its discrepancy, m the steps since.
  std::vector<uint64_t> C(n + 1, 0), B(n + 1, 0), T;
  C[0] = 1;
  B[0] = 1;
  int64_t L = 0, m = 1;
  uint64_t bd = 1;
  for (int64_t j = 0; j < n; ++j) {
    uint64_t d = seq[j];
    for (int64_t i = 1; i <= L; ++i) d = (d + C[i] * seq[j - i]) % p;
    if (d == 0) {
      ++m;
      continue;
    }
    const uint64_t coef = d * host_invmod((uint32_t)bd, p) % p;  // C <- C - (d / bd) x^m B
    const bool grow = 2 * L <= j;
    if (grow) T = C;
    for (int64_t i = 0; i + m <= n; ++i)
      if (B[i]) C[i + m] = (C[i + m] + (p - coef) * B[i]) % p;
    if (grow) {
      L = j + 1 - L;
      B = T;
      bd = d;
      m = 1;
    } else {
      ++m;
    }
  }
  for (int64_t i = 0; i <= L; ++i) conn[i] = (uint32_t)C[i];
  *L_out = L;
  return RR_OK;
}

}  // extern "C"
