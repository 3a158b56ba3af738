// rr_modp.cuh -- exact arithmetic modulo a prime p < 2^31 on sm_100a.
//
// Values are kept as uint32 in [0, p).  Dot products and sparse row sums are
// accumulated lazily in 64 bits: a product of two residues is < p^2 < 2^62,
// and an accumulator is "folded" (hi * (2^32 mod p) + lo) after every
// `fold_every` products so that it never wraps.  The final residue comes from
// a Barrett reduction with mu = floor(2^64 / p) (Barrett, CRYPTO '86).
#pragma once
#include <cstdint>

namespace rr {

struct ModP {
  uint32_t p;      // the prime, p < 2^31
  uint32_t c32;    // 2^32 mod p
  uint64_t mu;     // floor(2^64 / p)
  uint32_t pinv;   // -p^{-1} mod 2^32 (Montgomery reduction with R = 2^32)
  uint32_t r1;     // R mod p
};

#ifdef __CUDACC__
// a * b + c exactly (mod 2^64), as a carry chain of 32-bit multiply-adds
// (mad.lo.cc / madc.hi): on sm_100 this issues at about 1.6x the rate of the
// 64-bit wide multiply-add the compiler emits for (uint64_t)a * b + c.
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t c) {
  uint32_t lo = (uint32_t)c, hi = (uint32_t)(c >> 32);
  asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.u32 %1, %2, %3, %1;" : "+r"(lo), "+r"(hi) : "r"(a), "r"(b));
  return ((uint64_t)hi << 32) | lo;
}

// Fold a 64-bit accumulator: result == x (mod p) and result < 2^32 * c32 + 2^32.
__device__ __forceinline__ uint64_t fold(uint64_t x, const ModP& M) {
  return mad_wide((uint32_t)(x >> 32), M.c32, (uint32_t)x);
}

// Exact x mod p for any 64-bit x.  q = floor(x*mu / 2^64) is at most 2 below
// floor(x/p), so r = x - q*p < 3p and two conditional subtractions finish.
__device__ __forceinline__ uint32_t reduce(uint64_t x, const ModP& M) {
  const uint64_t q = __umul64hi(x, M.mu);
  uint64_t r = x - q * (uint64_t)M.p;
  if (r >= M.p) r -= M.p;
  if (r >= M.p) r -= M.p;
  return (uint32_t)r;
}

// Montgomery reduction (Montgomery 1985), R = 2^32: for T < p * 2^32 returns
// T * R^{-1} mod p in [0, p).  m = T * (-p^{-1}) mod R makes T + m p divisible
// by R, and T + m p < 2 p R < 2^64.  A folded accumulator always satisfies
// the bound, since fold() < (2^32 - 1) * c32 + 2^32 <= (2^32 - 1) * p + 2^32 - 1.
__device__ __forceinline__ uint32_t redc(uint64_t T, const ModP& M) {
  const uint32_t m = (uint32_t)T * M.pinv;
  const uint64_t s = (uint64_t)m * M.p + T;
  const uint32_t t = (uint32_t)(s >> 32);
  return t >= M.p ? t - M.p : t;
}

__device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b, const ModP& M) {
  return reduce((uint64_t)a * b, M);
}

__device__ __forceinline__ uint32_t addmod(uint32_t a, uint32_t b, uint32_t p) {
  const uint32_t s = a + b;  // a, b < 2^31 so no wrap
  return s >= p ? s - p : s;
}

__device__ __forceinline__ uint32_t submod(uint32_t a, uint32_t b, uint32_t p) {
  return a >= b ? a - b : a + p - b;
}

// (hi:lo) += a * b with a carry chain of 32-bit multiply-adds; on sm_100 this
// runs at about 1.6x the rate of the 64-bit wide multiply-add above.
__device__ __forceinline__ void mac_cc(uint32_t a, uint32_t b, uint32_t& lo, uint32_t& hi) {
  asm("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.u32 %1, %2, %3, %1;" : "+r"(lo), "+r"(hi) : "r"(a), "r"(b));
}

// Montgomery reduction of T = (hi:lo) < p * 2^32: T * 2^-32 mod p, in [0, p).
__device__ __forceinline__ uint32_t redc_cc(uint32_t lo, uint32_t hi, const ModP& M) {
  const uint32_t q = lo * M.pinv;
  mac_cc(q, M.p, lo, hi);  // lo becomes 0; T + q p < 2 p 2^32 <= 2^64
  return hi >= M.p ? hi - M.p : hi;
}

// (a b + c d) * 2^-32 mod p for residues a, b, c, d < p < 2^31.
__device__ __forceinline__ uint32_t redc_2mac(uint32_t a, uint32_t b, uint32_t c, uint32_t d, const ModP& M) {
  uint32_t lo = 0, hi = 0;
  mac_cc(a, b, lo, hi);
  mac_cc(c, d, lo, hi);
  return redc_cc(lo, hi, M);
}
#endif  // __CUDACC__

}  // namespace rr
