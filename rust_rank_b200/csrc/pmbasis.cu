// pmbasis.cu -- the minimal matrix generator (PM-basis) on the device.
//
// Reference: src/sigma_basis.rs:9-54 (PM_Basis), 190-219 (_PM_Basis),
// 283-294 (shift_trunc_in), 348-416 (M_Basis); src/modular_linalg.rs:188-239
// (lsp_decomposition), 10-69 (matrix_inverse); src/poly_mat_mul.rs:113-256.
//
// With exact arithmetic, _PM_Basis(G, d) equals the ordered product of d
// order-1 bases m_{d-1} ... m_0, where m_k = M_Basis(coefficient k of
// (m_{k-1}...m_0) G).  The engine keeps the reference's divide and conquer
// above blocks of K leaves and runs each block of K leaves iteratively inside
// one CTA:
//
//   * a leaf sorts delta stably (descending), eliminates the permuted
//     coefficient matrix row by row with the reference's pivot rule (first
//     non-zero column from `rank` in the swapped column order) and records
//     which rows hold a pivot (the "x" rows of Dx) -- identical decisions to
//     M_Basis;
//   * it forms T = L^{-1} pi by applying the same row operations to pi.
//     Rows are eliminated fraction-free (row_i <- piv*row_i - a_ic*row_k),
//     which leaves row i of the result scaled by a non-zero c_i; c_i is read
//     off T[i][perm[i]] (L^{-1} has a unit diagonal).  Scaled rows commute
//     with the leaf recurrence (T' R' = D T R for row-scaled R' = D R), so the
//     block carries a row scale sigma and normalises its product once at the
//     end instead of inverting per leaf;
//   * m_k = D1 T + x Dx T is applied to the residual series and to the block's
//     accumulated basis.
//
// Products above the blocks are exact NTT products modulo p itself (p must
// admit the transform length), which equal the reference's exact integer
// products reduced mod p.  NTTs are decimation-in-frequency forward (natural
// in, bit-reversed out) and decimation-in-time inverse (bit-reversed in,
// natural out), so no bit-reversal pass is needed; twiddles use Shoup's
// precomputed quotients.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>

#include "rr_internal.h"

namespace rr {

namespace {

constexpr int kNttBlock = 4096;  // elements transformed per CTA in shared memory
constexpr int kBaseThreads = 512;
constexpr size_t kBaseSmemBudget = 220 * 1024;  // dynamic shared memory of one block kernel

struct Twiddles {
  const uint32_t* w;   // omega^j, j < Nmax/2
  const uint32_t* ws;  // floor(w * 2^32 / p)
  int64_t nmax;
};

__device__ __forceinline__ uint32_t mul_shoup(uint32_t a, uint32_t w, uint32_t ws, uint32_t p) {
  const uint32_t q = __umulhi(a, ws);
  uint32_t r = a * w - q * p;  // in [0, 2p), computed mod 2^32
  return r >= p ? r - p : r;
}

// A batch of strided polynomial matrices seen as a flat list of polynomials:
// polynomial q is entry (qi / cols, qi % cols) of matrix q / npb (qi = q % npb),
// starting at p + (q / npb) * bs + (qi / cols) * rs + (qi % cols) * cs.
struct PolyView {
  uint32_t* p;
  int cols, npb;
  int64_t rs, cs, bs;
  __host__ __device__ uint32_t* at(int64_t q) const {
    const int64_t bi = q / npb, qi = q % npb;
    return p + bi * bs + (qi / cols) * rs + (qi % cols) * cs;
  }
};

// ---------------------------------------------------------------- NTT kernels
// Forward DIF stage with butterfly span `len` (len > kNttBlock) in global memory.
__global__ void ntt_fwd_stage_kernel(uint32_t* a, int64_t N, int64_t npoly, int64_t len, Twiddles tw, uint32_t p) {
  const int64_t half = len / 2;
  const int lh = __ffsll(half) - 1, lp = __ffsll(N / 2) - 1;
  const int64_t total = npoly * (N / 2);
  const int64_t tstep = tw.nmax / len;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t poly = t >> lp, b = t & (N / 2 - 1);
    const int64_t j = b & (half - 1);
    uint32_t* x = a + poly * N + ((b >> lh) << (lh + 1)) + j;
    const uint32_t u = x[0], v = x[half];
    x[0] = addmod(u, v, p);
    x[half] = mul_shoup(submod(u, v, p), tw.w[j * tstep], tw.ws[j * tstep], p);
  }
}

// Inverse DIT stage with span len (len > kNttBlock) in global memory.
__global__ void ntt_inv_stage_kernel(uint32_t* a, int64_t N, int64_t npoly, int64_t len, Twiddles tw, uint32_t p) {
  const int64_t half = len / 2;
  const int lh = __ffsll(half) - 1, lp = __ffsll(N / 2) - 1;
  const int64_t total = npoly * (N / 2);
  const int64_t tstep = tw.nmax / len;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t poly = t >> lp, b = t & (N / 2 - 1);
    const int64_t j = b & (half - 1);
    uint32_t* x = a + poly * N + ((b >> lh) << (lh + 1)) + j;
    const uint32_t u = x[0];
    const uint32_t v = mul_shoup(x[half], tw.w[j * tstep], tw.ws[j * tstep], p);
    x[0] = addmod(u, v, p);
    x[half] = submod(u, v, p);
  }
}

// Shared-memory NTT of the last (forward) or first (inverse) stages, span up
// to T = 2^logT <= kNttBlock.  A CTA transforms G = max(1, kNttGroup / T)
// consecutive T-blocks (several short polynomials per CTA), with the twiddles
// of span T staged in shared memory (span 2^lg uses entry j << (logT - lg))
// and power-of-two index arithmetic.  Dynamic shared memory: (G + 1) * T words.
constexpr int kNttGroup = 2048;

__device__ __forceinline__ void ntt_load_twiddles(uint32_t* W, uint32_t* WS, int logT, const Twiddles& tw) {
  const int64_t tstep = tw.nmax >> logT;
  for (int j = threadIdx.x; j < (1 << (logT - 1)); j += blockDim.x) {
    W[j] = tw.w[j * tstep];
    WS[j] = tw.ws[j * tstep];
  }
}

// Forward DIF.  When src.p != nullptr the blocks are first loaded from the
// polynomials of src (t < src_len, zero padded) -- only valid when N <= kNttBlock.
__global__ void __launch_bounds__(512) ntt_fwd_smem_kernel(uint32_t* a, int64_t N, int logT, int64_t nblocks,
                                                           PolyView src, int64_t src_len, Twiddles tw, uint32_t p) {
  extern __shared__ uint32_t nsm[];
  const int T = 1 << logT, G = T >= kNttGroup ? 1 : kNttGroup / T;
  uint32_t* s = nsm;
  uint32_t* W = s + G * T;
  uint32_t* WS = W + T / 2;
  const int64_t blk0 = (int64_t)blockIdx.x * G;
  ntt_load_twiddles(W, WS, logT, tw);
  for (int e = threadIdx.x; e < G * T; e += blockDim.x) {
    const int g = e >> logT, t = e & (T - 1);
    const int64_t blk = blk0 + g;
    uint32_t v = 0;
    if (blk < nblocks) {
      if (src.p) {  // N == T: block = polynomial; residues mod p < 2^31 < 2q, one subtraction reduces them mod q
        v = t < src_len ? src.at(blk)[t] : 0u;
        v = v >= p ? v - p : v;
      } else {
        v = a[(blk << logT) + t];
      }
    }
    s[e] = v;
  }
  __syncthreads();
  const int nbf = G * T / 2;
  for (int lg = logT; lg >= 1; --lg) {
    const int lh = lg - 1, half = 1 << lh, sh = logT - lg;
    for (int bf = threadIdx.x; bf < nbf; bf += blockDim.x) {
      const int j = bf & (half - 1);
      const int i0 = ((bf >> lh) << lg) | j;
      const uint32_t u = s[i0], v = s[i0 + half];
      s[i0] = addmod(u, v, p);
      s[i0 + half] = mul_shoup(submod(u, v, p), W[j << sh], WS[j << sh], p);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < G * T; e += blockDim.x) {
    const int64_t blk = blk0 + (e >> logT);
    if (blk < nblocks) a[(blk << logT) + (e & (T - 1))] = s[e];
  }
}

// Inverse DIT of the first stages.  When dst.p != nullptr (only valid when
// N <= T) the result is scaled by N^{-1} and coefficients [lo, lo + cnt) go to
// the polynomials of dst.
__global__ void __launch_bounds__(512) ntt_inv_smem_kernel(uint32_t* a, int64_t N, int logT, int64_t nblocks,
                                                           PolyView dst, int64_t lo, int64_t cnt, uint32_t ninv,
                                                           uint32_t ninv_s, Twiddles tw, uint32_t p) {
  extern __shared__ uint32_t nsm[];
  const int T = 1 << logT, G = T >= kNttGroup ? 1 : kNttGroup / T;
  uint32_t* s = nsm;
  uint32_t* W = s + G * T;
  uint32_t* WS = W + T / 2;
  const int64_t blk0 = (int64_t)blockIdx.x * G;
  ntt_load_twiddles(W, WS, logT, tw);
  for (int e = threadIdx.x; e < G * T; e += blockDim.x) {
    const int64_t blk = blk0 + (e >> logT);
    s[e] = blk < nblocks ? a[(blk << logT) + (e & (T - 1))] : 0u;
  }
  __syncthreads();
  const int nbf = G * T / 2;
  for (int lg = 1; lg <= logT; ++lg) {
    const int lh = lg - 1, half = 1 << lh, sh = logT - lg;
    for (int bf = threadIdx.x; bf < nbf; bf += blockDim.x) {
      const int j = bf & (half - 1);
      const int i0 = ((bf >> lh) << lg) | j;
      const uint32_t u = s[i0];
      const uint32_t v = mul_shoup(s[i0 + half], W[j << sh], WS[j << sh], p);
      s[i0] = addmod(u, v, p);
      s[i0 + half] = submod(u, v, p);
    }
    __syncthreads();
  }
  if (dst.p) {
    for (int e = threadIdx.x; e < G * cnt; e += blockDim.x) {
      const int g = (int)(e / cnt);
      const int64_t t = e - (int64_t)g * cnt;
      const int64_t blk = blk0 + g;
      if (blk < nblocks) dst.at(blk)[t] = mul_shoup(s[(g << logT) + lo + t], ninv, ninv_s, p);
    }
  } else {
    for (int e = threadIdx.x; e < G * T; e += blockDim.x) {
      const int64_t blk = blk0 + (e >> logT);
      if (blk < nblocks) a[(blk << logT) + (e & (T - 1))] = s[e];
    }
  }
}

// Copy poly q of a strided source into a dense N-length slot with zero
// padding, reduced modulo the transform prime qp (sources are < 2^31 < 2 qp).
__global__ void pad_copy_kernel(uint32_t* a, int64_t N, int64_t npoly, PolyView src, int64_t src_len, uint32_t qp) {
  const int64_t total = npoly * N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / N, k = t % N;
    const uint32_t v = (k < src_len) ? src.at(q)[k] : 0u;
    a[t] = v >= qp ? v - qp : v;
  }
}

__global__ void extract_scale_kernel(const uint32_t* a, int64_t N, int64_t npoly, PolyView dst, int64_t lo, int64_t cnt,
                                     uint32_t ninv, uint32_t ninv_s, uint32_t p) {
  const int64_t total = npoly * cnt;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / cnt, k = t % cnt;
    dst.at(q)[k] = mul_shoup(a[q * N + lo + k], ninv, ninv_s, p);
  }
}

// Exact integer products for primes without a suitable NTT: the product is
// computed modulo two or three NTT primes q0 < q1 < q2 whose product exceeds
// every coefficient of the exact integer product (inner dimension x length x
// (p-1)^2), the residues are combined by Garner's mixed-radix CRT
//   V = x0 + q0 x1 + q0 q1 x2,  x0 = r0,  x1 = (r1 - x0) q0^-1 mod q1,
//   x2 = ((r2 - x0) q0^-1 - x1) q1^-1 mod q2,
// and V is reduced mod p -- the reference's exact-integer-then-reduce
// semantics (src/poly_mat_mul.rs:240-256 over the prime of src/ntt.rs:60-75).
struct CrtParams {
  int k;                  // primes used (2 or 3)
  uint32_t q[3];
  ModP Mq[3];
  uint32_t c01, c02, c12;  // q0^-1 mod q1, q0^-1 mod q2, q1^-1 mod q2
  uint32_t q0p, q01p;      // q0 mod p, q0 q1 mod p
  ModP Mp;
};

__global__ void crt_kernel(const uint32_t* __restrict__ R0, const uint32_t* __restrict__ R1,
                           const uint32_t* __restrict__ R2, int64_t npoly, int64_t cnt, PolyView dst, CrtParams C) {
  const int64_t total = npoly * cnt;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / cnt, j = t - q * cnt;
    const uint32_t x0 = R0[t];
    const uint32_t x0m1 = x0 >= C.q[1] ? x0 - C.q[1] : x0;
    const uint32_t x1 = mulmod(submod(R1[t], x0m1, C.q[1]), C.c01, C.Mq[1]);
    uint64_t v = (uint64_t)x0 + (uint64_t)x1 * C.q0p;
    if (C.k == 3) {
      const uint32_t x0m2 = x0 >= C.q[2] ? x0 - C.q[2] : x0;
      const uint32_t x1m2 = x1 >= C.q[2] ? x1 - C.q[2] : x1;
      const uint32_t t2 = mulmod(submod(R2[t], x0m2, C.q[2]), C.c02, C.Mq[2]);
      const uint32_t x2 = mulmod(submod(t2, x1m2, C.q[2]), C.c12, C.Mq[2]);
      v += (uint64_t)x2 * C.q01p;  // < 2^31 + 2 * 2^62
    }
    dst.at(q)[j] = reduce(v, C.Mp);
  }
}

// Pointwise stage: C[i][j][f] = sum_r A[i][r][f] * B[r][j][f]  (all N-length),
// for nb matrices stored one after the other.  A thread computes a 4 x 4 tile
// of (i, j) at one frequency (consecutive threads take consecutive
// frequencies, so every load is coalesced), 16 carry-chain accumulators,
// folded every 4 steps (every 2 for primes where 4 products do not fit).  m and k are multiples of 4 here (m = 2b, k in {b, 2b}
// with b a multiple of 4); pointwise1_kernel covers the rest.
__global__ void __launch_bounds__(256) pointwise_kernel(const uint32_t* __restrict__ A, const uint32_t* __restrict__ Bm,
                                                        uint32_t* __restrict__ C, int m, int r, int k, int64_t N, int nb,
                                                        int fold_mask, ModP M) {
  const int ti = m / 4, tj = k / 4;
  const int64_t per = (int64_t)ti * tj * N;
  const int64_t total = per * nb;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bi = t / per, tt = t - bi * per;
    const int64_t f = tt % N;
    const int64_t tile = tt / N;
    const int i0 = 4 * (int)(tile / tj), j0 = 4 * (int)(tile % tj);
    const uint32_t* a = A + bi * (int64_t)m * r * N + (int64_t)i0 * r * N + f;
    const uint32_t* b = Bm + bi * (int64_t)r * k * N + (int64_t)j0 * N + f;
    uint32_t lo[4][4], hi[4][4];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) lo[x][y] = hi[x][y] = 0;
    for (int s = 0; s < r; ++s) {
      uint32_t av[4], bv[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) av[x] = a[(int64_t)x * r * N + (int64_t)s * N];
#pragma unroll
      for (int y = 0; y < 4; ++y) bv[y] = b[(int64_t)s * k * N + (int64_t)y * N];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) mac_cc(av[x], bv[y], lo[x][y], hi[x][y]);
      if ((s & fold_mask) == fold_mask) {  // fold (hi:lo) -> hi * (2^32 mod p) + lo every 4 (or 2) products
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            const uint32_t h = hi[x][y];
            hi[x][y] = 0;
            mac_cc(h, M.c32, lo[x][y], hi[x][y]);
          }
      }
    }
    uint32_t* c = C + bi * (int64_t)m * k * N + (int64_t)i0 * k * N + (int64_t)j0 * N + f;
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y)
        c[(int64_t)x * k * N + (int64_t)y * N] = reduce(((uint64_t)hi[x][y] << 32) | lo[x][y], M);
  }
}

// Pointwise stage for shapes that are not multiples of 4 (one output per thread).
__global__ void pointwise1_kernel(const uint32_t* __restrict__ A, const uint32_t* __restrict__ Bm, uint32_t* __restrict__ C,
                                  int m, int r, int k, int64_t N, int nb, ModP M) {
  const int64_t per = (int64_t)m * k * N;
  const int64_t total = per * nb;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bi = t / per, tt = t % per;
    const int64_t f = tt % N;
    const int64_t ij = tt / N;
    const int i = (int)(ij / k), j = (int)(ij % k);
    const uint32_t* a = A + bi * (int64_t)m * r * N + (int64_t)i * r * N + f;
    const uint32_t* b = Bm + bi * (int64_t)r * k * N + (int64_t)j * N + f;
    uint64_t acc = 0;
    int s = 0;
    for (; s + 1 < r; s += 2) {
      acc = mad_wide(a[(int64_t)s * N], b[(int64_t)s * k * N], acc);
      acc = mad_wide(a[(int64_t)(s + 1) * N], b[(int64_t)(s + 1) * k * N], acc);
      acc = fold(acc, M);
    }
    if (s < r) acc = mad_wide(a[(int64_t)s * N], b[(int64_t)s * k * N], acc);
    C[t] = reduce(acc, M);
  }
}

// Direct product for moduli without a suitable NTT: dst coefficient lo + t of
// sum_s A[i][s] * B[s][j], one thread per output coefficient.
__global__ void schoolbook_kernel(const uint32_t* A, int mA, int r, int64_t la, int64_t a_rs, int64_t a_cs,
                                  int64_t a_bs, const uint32_t* Bm, int k, int64_t lb, int64_t b_rs, int64_t b_cs,
                                  int64_t b_bs, uint32_t* dst, int64_t d_rs, int64_t d_cs, int64_t d_bs, int64_t lo,
                                  int64_t cnt, int nb, ModP M) {
  const int64_t per = (int64_t)mA * k * cnt;
  const int64_t total = per * nb;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bi = t / per, tt = t % per;
    const int64_t c = lo + tt % cnt;
    const int64_t ij = tt / cnt;
    const int i = (int)(ij / k), j = (int)(ij % k);
    uint64_t acc = 0;
    int parity = 0;
    for (int s = 0; s < r; ++s) {
      const uint32_t* a = A + bi * a_bs + (int64_t)i * a_rs + (int64_t)s * a_cs;
      const uint32_t* b = Bm + bi * b_bs + (int64_t)s * b_rs + (int64_t)j * b_cs;
      const int64_t u0 = c - (lb - 1) > 0 ? c - (lb - 1) : 0;
      const int64_t u1 = c < la - 1 ? c : la - 1;
      for (int64_t u = u0; u <= u1; ++u) {
        acc = mad_wide(a[u], b[c - u], acc);
        if (++parity == 2) { acc = fold(acc, M); parity = 0; }
      }
    }
    dst[bi * d_bs + (int64_t)i * d_rs + (int64_t)j * d_cs + (c - lo)] = reduce(acc, M);
  }
}

// G[i][j][t] = seq[pair(i,j)][t] for i < b; G[b+i][i][0] = 1 (src/sigma_basis.rs:33-46)
__global__ void build_G_kernel(const uint32_t* seq, int64_t seq_stride, int b, int64_t len, uint32_t* G, uint32_t p) {
  const int64_t total = (int64_t)2 * b * b * len;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = t % len;
    const int64_t ij = t / len;
    const int i = (int)(ij / b), j = (int)(ij % b);
    uint32_t v;
    if (i < b) {
      const int a = min(i, j), c = max(i, j);
      const int q = a * b - a * (a - 1) / 2 + (c - a);
      v = seq[(int64_t)q * seq_stride + k] % p;
    } else {
      v = (i - b == j && k == 0) ? 1u : 0u;
    }
    G[t] = v;
  }
}

// ---------------------------------------------------------------- base block
struct BaseParams {
  const uint32_t* G;   // G[i][c][t] (row stride g_rs, column stride g_cs), t < nleaves
  int64_t g_rs, g_cs;
  int m, n, nleaves;
  int64_t* delta;      // [m], in/out
  uint32_t* Mout;      // Mout[i][j][t], row stride out_rs, column stride out_cs, t <= nleaves
  int64_t out_rs, out_cs;
  uint32_t* Mbuf;      // scratch: 2 x (nleaves+1) x m x m, used unless m_smem
  int m_smem;          // keep the block's basis in shared memory
  ModP M;
  int* status;
};

__device__ uint32_t inv_fermat(uint32_t a, const ModP& M) {
  uint32_t r = 1, b = a;
  uint32_t e = M.p - 2;
  while (e) {
    if (e & 1) r = mulmod(r, b, M);
    b = mulmod(b, b, M);
    e >>= 1;
  }
  return r;
}

// One CTA runs nleaves order-1 leaves on G's first nleaves coefficients.
// VEC = 4 when 4 | b: the residual and basis updates then compute four
// adjacent columns per thread from 128-bit shared-memory reads.
// Arithmetic: every elimination and update ends in a Montgomery reduction, so
// each leaf multiplies the rows of the residual and of the basis by a known
// non-zero factor (c_i R^{-1}); sigma tracks it and the block's basis is
// normalised once at the end.
template <int VEC>
__global__ void __launch_bounds__(kBaseThreads) pm_base_kernel(BaseParams P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = P.m, n = P.n, K = P.nleaves;
  const int W = n + m;  // width of the augmented matrix [pi r | pi]
  const ModP M = P.M;
  const uint32_t p = M.p;
  uint32_t* R0 = reinterpret_cast<uint32_t*>(smem_raw);
  uint32_t* R1 = R0 + (size_t)K * m * n;
  uint32_t* MS = R1 + (size_t)K * m * n;                     // basis in shared memory (2 x (K+1) x m x m) or empty
  uint32_t* A = MS + (P.m_smem ? (size_t)2 * (K + 1) * m * m : 0);  // m x W
  uint32_t* T = A + (size_t)m * W;      // m x m
  uint32_t* fcol = T + (size_t)m * m;   // m
  uint32_t* sigma = fcol + m;           // m
  uint32_t* sig_tmp = sigma + m;        // m
  int64_t* sdelta = reinterpret_cast<int64_t*>(sig_tmp + m + (m & 1));  // m (8-byte aligned)
  int64_t* sdelta_tmp = sdelta + m;
  int* perm = reinterpret_cast<int*>(sdelta_tmp + m);
  int* mask = perm + m;
  int* Lst = mask + m;
  __shared__ int s_pivcol, s_pivflag, s_rank;

  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;

  for (int e = tid; e < K * m * n; e += nt) {
    const int t = e / (m * n), i = (e / n) % m, c = e % n;
    R0[e] = P.G[(int64_t)i * P.g_rs + (int64_t)c * P.g_cs + t];
  }
  for (int i = tid; i < m; i += nt) {
    sdelta[i] = P.delta[i];
    sigma[i] = 1;
  }
  uint32_t* Mc = P.m_smem ? MS : P.Mbuf;                            // current basis [t][i][j]
  uint32_t* Mn = Mc + (size_t)(K + 1) * m * m;                      // next basis
  for (int e = tid; e < m * m; e += nt) Mc[e] = (e / m == e % m) ? 1u : 0u;
  __syncthreads();

  uint32_t* Rc = R0;
  uint32_t* Rn = R1;
  for (int leaf = 0; leaf < K; ++leaf) {
    // stable sort of delta, descending (src/sigma_basis.rs:357-359)
    for (int i = tid; i < m; i += nt) {
      const int64_t di = sdelta[i];
      int pos = 0;
      for (int j = 0; j < m; ++j) {
        const int64_t dj = sdelta[j];
        pos += (dj > di) || (dj == di && j < i);
      }
      perm[pos] = i;
    }
    for (int i = tid; i < n; i += nt) Lst[i] = i;
    if (tid == 0) s_rank = 0;
    __syncthreads();
    // A = [pi r | pi]
    for (int e = tid; e < m * W; e += nt) {
      const int i = e / W, c = e % W;
      A[e] = c < n ? Rc[(size_t)perm[i] * n + c] : ((c - n) == perm[i] ? 1u : 0u);
    }
    __syncthreads();
    // LSP rows (src/modular_linalg.rs:198-226)
    for (int k = 0; k < m; ++k) {
      if (warp == 0) {
        const int rank = s_rank;
        const int len = n - rank;
        int c = -1;
        bool nz = false;
        if (lane < len) {
          c = Lst[lane];
          nz = A[(size_t)k * W + c] != 0;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, nz);
        const int l0 = __shfl_sync(0xffffffffu, c, 0);
        const int nxt = __shfl_down_sync(0xffffffffu, c, 1);
        if (bal) {
          const int ts = __ffs(bal) - 1;
          const int cstar = __shfl_sync(0xffffffffu, c, ts);
          // swap columns rank <-> pivot: the column at the front of the
          // unpivoted list takes the pivot's place, then the front is popped
          __syncwarp();
          if (lane < len - 1) Lst[lane] = (lane == ts - 1) ? l0 : nxt;
          if (lane == 0) {
            s_pivcol = cstar;
            s_pivflag = 1;
            s_rank = rank + 1;
            mask[k] = 1;
          }
        } else if (lane == 0) {
          s_pivflag = 0;
          mask[k] = 0;
        }
      }
      __syncthreads();
      const int pf = s_pivflag, cs = s_pivcol;
      if (pf) {
        for (int i = k + 1 + tid; i < m; i += nt) fcol[i] = A[(size_t)i * W + cs];
        __syncthreads();
        const uint32_t piv = A[(size_t)k * W + cs];
        const uint32_t* ak = A + (size_t)k * W;
        const int rows = m - k - 1;
        for (int e = tid; e < rows * W; e += nt) {
          const int i = k + 1 + e / W, c = e % W;
          // (piv * a_ic - a_ic* * a_kc) R^{-1}: the row keeps a non-zero scale
          const uint64_t acc = mad_wide(piv, A[(size_t)i * W + c], (uint64_t)(p - fcol[i]) * ak[c]);
          A[(size_t)i * W + c] = redc(acc, M);
        }
      }
      // no warp may rewrite the step flags before every warp has read them
      __syncthreads();
    }
    // T = scaled L^{-1} pi; c_i = T[i][perm[i]]; rows of the updates below are
    // multiplied by c_i R^{-1}
    for (int e = tid; e < m * m; e += nt) T[e] = A[(size_t)(e / m) * W + n + (e % m)];
    for (int i = tid; i < m; i += nt) {
      const uint32_t ci = A[(size_t)i * W + n + perm[i]];
      if (ci == 0) atomicExch(P.status, 2);
      sig_tmp[i] = redc((uint64_t)ci * sigma[perm[i]], M);
      sdelta_tmp[i] = sdelta[perm[i]] - mask[i];  // src/sigma_basis.rs:408-411
    }
    __syncthreads();
    for (int i = tid; i < m; i += nt) {
      sigma[i] = sig_tmp[i];
      sdelta[i] = sdelta_tmp[i];
    }
    // residual: Rn[t][i] = T_i . Rc[t + 1 - mask_i], t < K - leaf - 1
    const int rem = K - leaf - 1;
    const int nq = n / VEC;
    for (int e = tid; e < rem * m * nq; e += nt) {
      const int t = e / (m * nq), i = (e / nq) % m, c = (e % nq) * VEC;
      const uint32_t* src = Rc + (size_t)(t + 1 - mask[i]) * m * n + c;
      const uint32_t* ti = T + (size_t)i * m;
      uint64_t acc[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = 0;
      for (int s = 0; s < m; ++s) {
        const uint32_t w = ti[s];
        if (VEC == 4) {
          const uint4 x = *reinterpret_cast<const uint4*>(src + (size_t)s * n);
          acc[0] = mad_wide(w, x.x, acc[0]);
          acc[VEC > 1 ? 1 : 0] = mad_wide(w, x.y, acc[VEC > 1 ? 1 : 0]);
          acc[VEC > 2 ? 2 : 0] = mad_wide(w, x.z, acc[VEC > 2 ? 2 : 0]);
          acc[VEC > 3 ? 3 : 0] = mad_wide(w, x.w, acc[VEC > 3 ? 3 : 0]);
        } else {
          acc[0] = mad_wide(w, src[(size_t)s * n], acc[0]);
        }
        if (s & 1) {
#pragma unroll
          for (int v = 0; v < VEC; ++v) acc[v] = fold(acc[v], M);
        }
      }
      uint32_t* dst = Rn + (size_t)t * m * n + (size_t)i * n + c;
#pragma unroll
      for (int v = 0; v < VEC; ++v) dst[v] = redc(fold(acc[v], M), M);
    }
    // basis: Mn[t][i] = T_i . Mc[t - mask_i], t <= leaf + 1
    const int mq = m / VEC;
    for (int e = tid; e < (leaf + 2) * m * mq; e += nt) {
      const int t = e / (m * mq), i = (e / mq) % m, c = (e % mq) * VEC;
      const int st = t - mask[i];
      uint32_t* dst = Mn + (size_t)t * m * m + (size_t)i * m + c;
      if (st < 0 || st > leaf) {
#pragma unroll
        for (int v = 0; v < VEC; ++v) dst[v] = 0;
        continue;
      }
      const uint32_t* src = Mc + (size_t)st * m * m + c;
      const uint32_t* ti = T + (size_t)i * m;
      uint64_t acc[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = 0;
      for (int s = 0; s < m; ++s) {
        const uint32_t w = ti[s];
        if (VEC == 4) {
          const uint4 x = *reinterpret_cast<const uint4*>(src + (size_t)s * m);
          acc[0] = mad_wide(w, x.x, acc[0]);
          acc[VEC > 1 ? 1 : 0] = mad_wide(w, x.y, acc[VEC > 1 ? 1 : 0]);
          acc[VEC > 2 ? 2 : 0] = mad_wide(w, x.z, acc[VEC > 2 ? 2 : 0]);
          acc[VEC > 3 ? 3 : 0] = mad_wide(w, x.w, acc[VEC > 3 ? 3 : 0]);
        } else {
          acc[0] = mad_wide(w, src[(size_t)s * m], acc[0]);
        }
        if (s & 1) {
#pragma unroll
          for (int v = 0; v < VEC; ++v) acc[v] = fold(acc[v], M);
        }
      }
#pragma unroll
      for (int v = 0; v < VEC; ++v) dst[v] = redc(fold(acc[v], M), M);
    }
    __syncthreads();
    uint32_t* tr = Rc; Rc = Rn; Rn = tr;
    uint32_t* tm = Mc; Mc = Mn; Mn = tm;
  }
  // normalise rows by sigma^{-1} and write out [i][j][t]
  for (int i = tid; i < m; i += nt) sig_tmp[i] = inv_fermat(sigma[i], M);
  __syncthreads();  // every status write of this CTA is visible after the barrier
  // a zero row scale cannot be returned by the asynchronous caller: it marks
  // the output instead, every delta entry INT64_MIN
  const bool failed = *(volatile int*)P.status != 0;
  for (int i = tid; i < m; i += nt) P.delta[i] = failed ? INT64_MIN : sdelta[i];
  for (int e = tid; e < (K + 1) * m * m; e += nt) {
    const int t = e / (m * m), i = (e / m) % m, c = e % m;
    P.Mout[(int64_t)i * P.out_rs + (int64_t)c * P.out_cs + t] = mulmod(Mc[e], sig_tmp[i], M);
  }
}

// Shared-memory bytes of pm_base_kernel for m rows, n columns, K leaves.
size_t base_smem_bytes(int m, int n, int K, bool m_smem) {
  size_t words = (size_t)2 * K * m * n + (m_smem ? (size_t)2 * (K + 1) * m * m : 0) + (size_t)m * (n + m) +
                 (size_t)m * m + 3 * (size_t)m + 1;
  size_t bytes = (words * 4 + 7) & ~(size_t)7;
  bytes += 2 * (size_t)m * 8 + 3 * (size_t)m * 4 + 64;
  return bytes;
}

// ---------------------------------------------------------------- leaves + block basis (main path)
// The main path splits a block of K leaves in two kernels:
//
//   pm_leaves_kernel (one CTA) runs the K order-1 leaves in sequence and, for
//   each, records the stored transform T_k (transposed, Tt[k][s][i]) and its
//   pivot rows; it updates only the residual series, which is what the next
//   leaf depends on.
//   pm_block_basis_kernel (one CTA per basis column) multiplies the recorded
//   factors m_{K-1} ... m_0 (m_k = D1 T_k + x Dx T_k) in parallel and writes the
//   block's basis, normalised by the row scales.
//
// Elimination.  For m <= 32 rows and n + m <= 48 columns (b <= 16) one warp
// eliminates with one row per lane, held in registers: the pivot row is
// broadcast by shuffles, the pivot column is the unpivoted column of least
// list position (one redux.sync), and no CTA barrier is needed.  Larger
// blocks keep the matrix in shared memory and give each warp the rows
// i == warp (mod 16), with one CTA barrier per pivot step.  Either way the
// loop stops once all n columns have pivots: no later row can get one.
//
// Residual update.  The rows are regrouped so that pivot rows ("x" rows,
// shifted by one coefficient) come first, each group padded to a multiple of
// four; a thread then computes a 4 x 4 tile (16 independent 64-bit
// accumulators) whose rows all read the same source coefficient.
constexpr int kLeafThreads = 512;
constexpr int kLeafWarps = kLeafThreads / 32;


struct LeafParams {
  const uint32_t* G;  // G[i][c][t] (row stride g_rs, column stride g_cs), t < K; CTA z takes G + z g_bs
  int64_t g_rs, g_cs, g_bs;
  int m, n, K;
  int64_t cs;                // words per residual coefficient in shared memory (>= m * n, padded)
  int64_t* delta;            // [nb][m], in/out
  uint32_t* Tt;              // [nb][K][m][m]: Tt[k][s][i] = stored T_k[i][s]
  unsigned long long* mask;  // [nb][K]: bit i set when row i of leaf k is a pivot row (an "x" row)
  uint32_t* sigma_inv;       // [nb][m]: inverse row scales of the block's stored basis
  ModP M;
  int* status;
};

// Row stride (words) of the slot-ordered transform in shared memory: room for
// m rows plus the padding of two groups, a multiple of four.
__host__ __device__ constexpr int leaf_tstride(int m) { return (m + 6 + 3) & ~3; }

// Shared-memory bytes of pm_leaves_kernel.
size_t leaves_smem_bytes(int m, int n, int K, int64_t cs) {
  const size_t W = (size_t)n + m, TS = (size_t)leaf_tstride(m);
  size_t words = (size_t)2 * K * cs + (((size_t)m * W + 3) & ~(size_t)3) + (size_t)m * TS + 2 * (size_t)m;
  size_t bytes = (words * 4 + 15) & ~(size_t)15;
  bytes += 2 * (size_t)m * 8 + (3 * (size_t)m + (size_t)n + TS) * 4 + 64;
  return bytes;
}

// Shared-memory bytes of pm_block_basis_kernel.
size_t block_basis_smem_bytes(int m, int K) {
  const size_t S = (size_t)leaf_tstride(m), VS = ((size_t)(K + 1) * (m + 1) + 3) & ~(size_t)3;
  return (2 * VS + (size_t)m * S) * 4 + (size_t)S * 4;
}

// Pivot search of row r by one warp (src/modular_linalg.rs:198-226): the first
// non-zero column of row r in the order of the unpivoted list Lst.  A pivot
// moves the list's front into the pivot's slot and pops the front.
__device__ __forceinline__ void leaf_search(int r, const uint32_t* A, int W, int n, int* Lst, int* s_flag,
                                            int* s_col, int* s_rank, int* rowmask, int lane) {
  const int rank = r == 0 ? 0 : s_rank[(r - 1) & 1];
  const int len = n - rank;
  int c = -1;
  bool nz = false;
  if (lane < len) {
    c = Lst[lane];
    nz = A[r * W + c] != 0;
  }
  const unsigned bal = __ballot_sync(0xffffffffu, nz);
  const int l0 = __shfl_sync(0xffffffffu, c, 0);
  const int nxt = __shfl_down_sync(0xffffffffu, c, 1);
  int col = 0;
  if (bal) {
    const int ts = __ffs(bal) - 1;
    col = __shfl_sync(0xffffffffu, c, ts);
    __syncwarp();
    if (lane < len - 1) Lst[lane] = (lane == ts - 1) ? l0 : nxt;
  }
  if (lane == 0) {
    s_flag[r & 1] = bal ? 1 : 0;
    s_col[r & 1] = col;
    s_rank[r & 1] = rank + (bal ? 1 : 0);
    rowmask[r] = bal ? 1 : 0;
  }
}

// Slot of row i (i < m) in the grouped order: pivot rows first (increasing
// i), padded to a multiple of four, then the other rows.  mx is the pivot-row
// mask; rows past m never get a slot.
__device__ __forceinline__ int leaf_slot(unsigned long long mx, int i, int m) {
  const unsigned long long below = (i == 0) ? 0ull : (~0ull >> (64 - i));
  const int nx = __popcll(mx);
  if ((mx >> i) & 1ull) return __popcll(mx & below);
  const unsigned long long valid = (m == 64) ? ~0ull : ((1ull << m) - 1);
  return ((nx + 3) & ~3) + __popcll(~mx & valid & below);
}

// One matrix of the batch per CTA (blockIdx.x).
__device__ __forceinline__ void leaf_select(LeafParams& P) {
  const int z = blockIdx.x;
  P.G += (int64_t)z * P.g_bs;
  P.delta += (int64_t)z * P.m;
  P.Tt += (int64_t)z * P.K * P.m * P.m;
  P.mask += (int64_t)z * P.K;
  P.sigma_inv += (int64_t)z * P.m;
}

template <int CT, int FE>
__global__ void __launch_bounds__(kLeafThreads) pm_leaves_kernel(LeafParams P) {
  leaf_select(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = P.m, n = P.n, K = P.K;
  const int W = n + m;
  const int TS = leaf_tstride(m);
  const int CS = (int)P.cs;
  const ModP M = P.M;
  const uint32_t p = M.p;
  uint32_t* Rc = reinterpret_cast<uint32_t*>(smem_raw);  // [K][CS]: residual coefficient t, row i, column c
  uint32_t* Rn = Rc + (size_t)K * CS;
  uint32_t* A = Rn + (size_t)K * CS;                      // m x W augmented matrix [pi r | pi] (multi-warp path)
  uint32_t* Tq = A + ((m * W + 3) & ~3);                  // m x TS: Tq[s][slot] = T[row(slot)][s]
  uint32_t* sigma = Tq + m * TS;                          // m
  uint32_t* sig_tmp = sigma + m;                          // m
  const size_t w32 = (size_t)2 * K * CS + (((size_t)m * W + 3) & ~(size_t)3) + (size_t)m * TS + 2 * (size_t)m;
  int64_t* sdelta = reinterpret_cast<int64_t*>(smem_raw + ((w32 * 4 + 15) & ~(size_t)15));
  int64_t* sdelta_tmp = sdelta + m;
  int* perm = reinterpret_cast<int*>(sdelta_tmp + m);
  int* rowmask = perm + m;
  int* slotrow = rowmask + m;  // TS entries: row of a slot, -1 for padding
  int* Lst = slotrow + TS;
  __shared__ int s_flag[2], s_col[2], s_rank[2];
  __shared__ unsigned long long s_mx;

  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;

  for (int i = warp; i < m; i += kLeafWarps)
    for (int c = lane; c < n; c += 32)
      for (int t = 0; t < K; ++t) Rc[t * CS + i * n + c] = P.G[(int64_t)i * P.g_rs + (int64_t)c * P.g_cs + t];
  for (int i = tid; i < m; i += nt) {
    sdelta[i] = P.delta[i];
    sigma[i] = 1;
  }
  __syncthreads();

  for (int leaf = 0; leaf < K; ++leaf) {
    uint32_t* Tg = P.Tt + (size_t)leaf * m * m;
    // stable sort of delta, descending (src/sigma_basis.rs:357-359)
    for (int i = tid; i < m; i += nt) {
      const int64_t di = sdelta[i];
      int pos = 0;
      for (int j = 0; j < m; ++j) {
        const int64_t dj = sdelta[j];
        pos += (dj > di) || (dj == di && j < i);
      }
      perm[pos] = i;
    }
    for (int i = tid; i < n; i += nt) Lst[i] = i;
    for (int i = tid; i < m; i += nt) rowmask[i] = 0;
    __syncthreads();
    // A = [pi r | pi]  (src/sigma_basis.rs:369-380)
    for (int i = warp; i < m; i += kLeafWarps) {
      const int pi = perm[i];
      for (int c = lane; c < W; c += 32) A[i * W + c] = c < n ? Rc[pi * n + c] : ((c - n) == pi ? 1u : 0u);
    }
    __syncthreads();
    if (warp == 0) leaf_search(0, A, W, n, Lst, s_flag, s_col, s_rank, rowmask, lane);
    // LSP elimination, fraction-free: row_i <- (piv row_i - a_i,cs row_k) R^{-1}
    for (int k = 0; k < m; ++k) {
      __syncthreads();  // row k final, its pivot published
      const int flag = s_flag[k & 1], cs = s_col[k & 1];
      const int rank_k = s_rank[k & 1];
      if (flag) {
        const uint32_t* ak = A + k * W;
        const uint32_t piv = ak[cs];
        int i = warp;
        while (i <= k) i += kLeafWarps;
        for (; i < m; i += kLeafWarps) {
          uint32_t* ai = A + i * W;
          const uint32_t f = ai[cs];
          __syncwarp();
          const uint64_t nf = (uint64_t)(p - f);
          for (int c = lane; c < W; c += 32) ai[c] = redc(mad_wide(piv, ai[c], nf * ak[c]), M);
        }
      }
      if (rank_k == n) break;  // every column has its pivot: no later row pivots
      if (k + 1 < m && warp == (k + 1) % kLeafWarps) {
        __syncwarp();
        leaf_search(k + 1, A, W, n, Lst, s_flag, s_col, s_rank, rowmask, lane);
      }
    }
    __syncthreads();
    if (warp == 0) {
      unsigned long long mx = 0;
      for (int i = lane; i < m; i += 32) mx |= (unsigned long long)(rowmask[i] != 0) << i;
#pragma unroll
      for (int off = 16; off; off >>= 1) mx |= __shfl_xor_sync(0xffffffffu, mx, off);
      if (lane == 0) {
        P.mask[leaf] = mx;
        s_mx = mx;
      }
      for (int q = lane; q < TS; q += 32) slotrow[q] = -1;
    }
    __syncthreads();
    const unsigned long long mx = s_mx;
    for (int i = tid; i < m; i += nt) slotrow[leaf_slot(mx, i, m)] = i;
    for (int e = tid; e < m * TS; e += nt) Tq[e] = 0;
    __syncthreads();
    for (int i = warp; i < m; i += kLeafWarps) {
      const int slot = leaf_slot(mx, i, m);
      for (int s = lane; s < m; s += 32) {
        const uint32_t v = A[i * W + n + s];
        Tq[s * TS + slot] = v;
        Tg[s * m + i] = v;
      }
    }
    for (int i = tid; i < m; i += nt) {
      const uint32_t ci = A[i * W + n + perm[i]];
      if (ci == 0) atomicExch(P.status, 2);
      sig_tmp[i] = redc((uint64_t)ci * sigma[perm[i]], M);
      sdelta_tmp[i] = sdelta[perm[i]] - rowmask[i];  // src/sigma_basis.rs:408-411
    }
    __syncthreads();
    for (int i = tid; i < m; i += nt) {
      sigma[i] = sig_tmp[i];
      sdelta[i] = sdelta_tmp[i];
    }
    __syncthreads();
    // residual: Rn[t][i] = T_i . Rc[t + 1 - mask_i], t < K - leaf - 1, in 4 x CT tiles
    const int rem = K - leaf - 1;
    if (rem > 0) {
      const unsigned long long mx = s_mx;
      const int nx = __popcll(mx);
      const int gx = (nx + 3) & ~3;
      const int QG = (gx + ((m - nx + 3) & ~3)) / 4, CG = n / CT;
      const int jobs = rem * QG * CG;
      for (int job = tid; job < jobs; job += nt) {
        const int t = job / (QG * CG);
        const int qg = (job / CG) % QG, cg = job % CG;
        const int q0 = 4 * qg, c0 = CT * cg;
        const int shift = q0 < gx ? 0 : 1;  // pivot rows read coefficient t, the others t + 1
        const uint32_t* w = Tq + q0;
        const uint32_t* x = Rc + (t + shift) * CS + c0;
        uint64_t acc[4][CT];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int v = 0; v < CT; ++v) acc[r][v] = 0;
        int s = 0;
        for (; s + FE <= m; s += FE) {
#pragma unroll
          for (int u = 0; u < FE; ++u) {
            const uint4 wv = *reinterpret_cast<const uint4*>(w);
            uint32_t xv[CT];
            if (CT == 4) {
              const uint4 q = *reinterpret_cast<const uint4*>(x);
              xv[0] = q.x;
              xv[CT > 1 ? 1 : 0] = q.y;
              xv[CT > 2 ? 2 : 0] = q.z;
              xv[CT > 3 ? 3 : 0] = q.w;
            } else {
              xv[0] = *x;
            }
            const uint32_t wr[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
              for (int v = 0; v < CT; ++v) acc[r][v] = mad_wide(wr[r], xv[v], acc[r][v]);
            w += TS;
            x += n;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int v = 0; v < CT; ++v) acc[r][v] = fold(acc[r][v], M);
        }
        for (; s < m; ++s) {
          const uint4 wv = *reinterpret_cast<const uint4*>(w);
          const uint32_t wr[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int v = 0; v < CT; ++v) acc[r][v] = fold(mad_wide(wr[r], x[v], acc[r][v]), M);
          w += TS;
          x += n;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int row = slotrow[q0 + r];
          if (row >= 0) {
            uint32_t* dst = Rn + t * CS + row * n + c0;
#pragma unroll
            for (int v = 0; v < CT; ++v) dst[v] = redc(acc[r][v], M);
          }
        }
      }
    }
    __syncthreads();
    uint32_t* tr = Rc;
    Rc = Rn;
    Rn = tr;
  }
  for (int i = tid; i < m; i += nt) {
    P.sigma_inv[i] = inv_fermat(sigma[i], M);
    P.delta[i] = sdelta[i];
  }
}

// ---------------------------------------------------------------- leaves, tensor-core path (b <= 16)
// For m <= 32 rows and n <= 16 columns the residual update runs on the int8
// tensor cores, exactly: residues are < 2^31, so with byte limbs
//   (T R)[i][c] = sum over a, b of 256^(a+b) (T_a R_b)[i][c],
// and per shift class s = a + b the limb products summed over the 32-long
// inner dimension stay below 4 * 32 * 255^2 < 2^23, exact in int32
// (mma.sync m16n8k32 u8).  Classes 0..3 are recombined exactly in 64 bits
// (< 2^48), classes 4..6 are added with weights 2^(8s) mod p, and one
// Montgomery reduction gives (T R) R^{-1} -- the value the CUDA-core path
// produces.  The residual lives in shared memory only as byte planes,
// plane[t][limb][c][i] (one 32-byte row per column c, K index i), so each B
// fragment is two 32-bit loads; the transform T is staged the same way for
// the A fragments.  Row r of a plane keeps word w at w ^ 4 (r >> 2 & 1), so the
// fragment loads of rows r and r + 4 fall in different banks.
//
// The elimination runs in kElimWarps warps, one row per lane, each warp
// holding kElimColsPerWarp of the 48 columns in registers; every column is
// updated unconditionally (padding columns are zero and stay zero), so the
// updates of a step are independent.  Two warps per SM sub-partition hide
// each other's dependency latencies (the elimination is the serial part of a
// leaf).
constexpr int kMmaRows = 32;
constexpr int kMmaCols = 16;
constexpr int kElimWarps = 8;
constexpr int kRpartStride = kMmaCols + 1;            // row stride of the published columns
constexpr int kRpartSize = kMmaRows * kRpartStride;
constexpr int kElimColsPerWarp = 6;  // 8 x 6 = 48 >= n + m
static_assert(kElimWarps * kElimColsPerWarp >= kMmaRows + kMmaCols, "elimination columns");
static_assert(kElimWarps <= kLeafWarps, "elimination warps");

// Named barriers of the elimination warps and of the update warps.
__device__ __forceinline__ void elim_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kElimWarps * 32) : "memory"); }
__device__ __forceinline__ void upd_bar() {
  asm volatile("bar.sync 2, %0;" ::"n"((kLeafWarps - kElimWarps) * 32) : "memory");
}
constexpr uint64_t kLeafWaitNs = 2000000000ull;  // 2 s of %globaltimer per hand-off wait
__device__ __forceinline__ uint64_t leaf_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void leaf_mma_u8(int (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__host__ __device__ constexpr int plane_word(int r, int w) { return r * 8 + (w ^ (((r >> 2) & 1) << 2)); }

// Words of one residual coefficient in plane form: 4 limbs x (n padded to 8) rows x 8 words.
__host__ __device__ constexpr int leaf_plane_words(int n) { return 32 * 8 * ((n + 7) / 8); }

// Shared-memory bytes of pm_leaves_mma_kernel.
size_t leaves_mma_smem_bytes(int m, int n, int K) {
  size_t words = (size_t)2 * K * leaf_plane_words(n) + 2048 + (size_t)m * (m + 1) + (size_t)m * n + 2 * (size_t)m;
  size_t bytes = (words * 4 + 15) & ~(size_t)15;
  bytes += 2 * (size_t)m * 8 + (size_t)m * 4 + 64;
  return bytes;
}

__device__ __forceinline__ void plane_store(uint32_t* coeff, int NPc, int col, int row, uint32_t v) {
  unsigned char* b = reinterpret_cast<unsigned char*>(coeff);
  const int wo = plane_word(col, row >> 2), bo = row & 3;
#pragma unroll
  for (int l = 0; l < 4; ++l) b[4 * (l * NPc * 8 + wo) + bo] = (unsigned char)(v >> (8 * l));
}

__global__ void __launch_bounds__(kLeafThreads) pm_leaves_mma_kernel(LeafParams P) {
  leaf_select(P);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = P.m, n = P.n, K = P.K;
  const int W = n + m;
  const int NT = (n + 7) / 8, MT = (m + 15) / 16, NPc = 8 * NT;
  const int PW = leaf_plane_words(n);
  const int TQS = m + 1;
  const ModP M = P.M;
  const uint32_t p = M.p;
  uint32_t* Rc = reinterpret_cast<uint32_t*>(smem_raw);  // [K][PW] residual byte planes
  uint32_t* Rn = Rc + K * PW;
  uint32_t* Tp = Rn + K * PW;                             // 2 x [4][32 rows][8 words] byte planes of T
  uint32_t* Tq = Tp + 2048;                               // [m][TQS]: Tq[s][i] = T[i][s]
  uint32_t* R0 = Tq + m * TQS;                            // [m][n]: coefficient 0 of the residual
  uint32_t* sigma = R0 + m * n;                           // m
  uint32_t* sig_tmp = sigma + m;                          // m
  const size_t w32 = (size_t)2 * K * PW + 2048 + (size_t)m * TQS + (size_t)m * n + 2 * (size_t)m;
  int64_t* sdelta = reinterpret_cast<int64_t*>(smem_raw + ((w32 * 4 + 15) & ~(size_t)15));
  int64_t* sdelta_tmp = sdelta + m;
  int* perm = reinterpret_cast<int*>(sdelta_tmp + m);
  __shared__ unsigned long long s_mx2[2];     // pivot-row masks of the last two leaves
  __shared__ volatile int s_tready, s_c1, s_abort;
  __shared__ int s_ok_e, s_ok_u;
  __shared__ uint32_t rpart[2 * kRpartSize];  // first n columns of A, all rows, double buffered

  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const uint32_t Wt[3] = {M.c32, (uint32_t)((uint64_t)M.c32 * 256 % p), (uint32_t)((uint64_t)M.c32 * 65536 % p)};

  // padding bytes (rows i >= m of every column, columns c >= n) stay zero for good
  for (int e = tid; e < 2 * K * PW + 2048; e += nt) Rc[e] = 0;
  __syncthreads();
  for (int e = tid; e < K * m * n; e += nt) {
    const int t = e / (m * n), i = (e / n) % m, c = e % n;
    const uint32_t v = P.G[(int64_t)i * P.g_rs + (int64_t)c * P.g_cs + t];
    plane_store(Rc + t * PW, NPc, c, i, v);
    if (t == 0) R0[i * n + c] = v;
  }
  for (int i = tid; i < m; i += nt) {
    sdelta[i] = P.delta[i];
    sigma[i] = 1;
  }
  __syncthreads();

  // Two warp groups overlap consecutive leaves: the elimination warps (E,
  // warps 0 .. kElimWarps-1) run leaf k+1 while the update warps (U, the
  // others) still apply T_k to the remaining coefficients of the residual.
  // Leaf k+1 needs only coefficient 0 of the new residual, which E computes
  // itself (from coefficients 0 and 1 of the old one); U computes the others,
  // coefficient 1 first.  Residual buffer j & 1 holds the residual before leaf
  // j; E writes only coefficient 0 of a buffer and U only coefficients >= 1,
  // and T_k's byte planes and mask are double buffered by k & 1.  Hand-offs are
  // counters in shared memory: s_tready = k + 1 once T_k, its mask and the new
  // coefficient 0 are written (U may start on leaf k), s_c1 = k + 1 once U has
  // written coefficient 1 of the residual after leaf k (E may take T_{k+1} and
  // reuse T_{k-1}'s planes).  A wait gives up after kLeafWaitNs, raises
  // s_abort and sets *P.status = 3; both groups then leave their loops.
  if (tid == 0) {
    s_tready = 0;
    s_c1 = 0;
    s_abort = 0;
  }
  __syncthreads();
  const int tiles = MT * NT;  // 1, 2 or 4: a divisor of the group's warp count
  auto wait_count = [&](volatile int* cnt, int target) -> bool {
    const uint64_t t0 = leaf_ns();
    while (*cnt < target) {
      if (s_abort) return false;
      if (leaf_ns() - t0 > kLeafWaitNs) {
        s_abort = 1;
        atomicExch(P.status, 3);
        return false;
      }
      __nanosleep(32);
    }
    __threadfence_block();
    return true;
  };
  // outputs t in [tmin, tmax] (and < rem) of Rn[t][i] = T_i . Rc[t + 1 - mask_i],
  // from the products T Rc[tq] for the tq of this warp's share
  auto residual = [&](int gw, int gwarps, int tq_first, int tq_last, int tmin, int tmax, const uint32_t* Tpl,
                      const uint32_t* Rcl, uint32_t* Rnl, unsigned long long mx, int rem) {
    const int tile = gw % tiles, tq0 = tq_first + gw / tiles, tqs = gwarps / tiles;
    const int mt = tile / NT, ntl = tile % NT;
    const int r0 = mt * 16 + g, r1 = r0 + 8, col = ntl * 8 + g;
    if (tq0 > tq_last) return;
    uint32_t A[4][4];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      A[l][0] = Tpl[l * 256 + plane_word(r0, t4)];
      A[l][1] = Tpl[l * 256 + plane_word(r1, t4)];
      A[l][2] = Tpl[l * 256 + plane_word(r0, t4 + 4)];
      A[l][3] = Tpl[l * 256 + plane_word(r1, t4 + 4)];
    }
    for (int tq = tq0; tq <= tq_last; tq += tqs) {
      uint32_t Bf[4][2];
      const uint32_t* rc = Rcl + tq * PW;
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        Bf[l][0] = rc[l * NPc * 8 + plane_word(col, t4)];
        Bf[l][1] = rc[l * NPc * 8 + plane_word(col, t4 + 4)];
      }
      int C[7][4];
#pragma unroll
      for (int s = 0; s < 7; ++s)
#pragma unroll
        for (int v = 0; v < 4; ++v) C[s][v] = 0;
#pragma unroll
      for (int l = 0; l < 4; ++l)
#pragma unroll
        for (int r = 0; r < 4; ++r) leaf_mma_u8(C[l + r], A[l], Bf[r][0], Bf[r][1]);
      // classes 0..3 exactly in 64 bits (< 2^48), classes 4..6 with their weights
      uint32_t lo[4], hi[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const uint64_t x = (uint64_t)(uint32_t)C[0][v] + ((uint64_t)(uint32_t)C[1][v] << 8) +
                           ((uint64_t)(uint32_t)C[2][v] << 16) + ((uint64_t)(uint32_t)C[3][v] << 24);
        lo[v] = (uint32_t)x;
        hi[v] = (uint32_t)(x >> 32);
        mac_cc((uint32_t)C[4][v], Wt[0], lo[v], hi[v]);
        mac_cc((uint32_t)C[5][v], Wt[1], lo[v], hi[v]);
        mac_cc((uint32_t)C[6][v], Wt[2], lo[v], hi[v]);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = (v < 2) ? r0 : r1;
        const int c = ntl * 8 + 2 * t4 + (v & 1);
        if (row < m && c < n) {
          const int t = tq - 1 + (int)((mx >> row) & 1ull);
          if (t >= tmin && t <= tmax && t < rem) {
            const uint32_t val = redc_cc(lo[v], hi[v], M);
            plane_store(Rnl + t * PW, NPc, c, row, val);
            if (t == 0) R0[row * n + c] = val;
          }
        }
      }
    }
  };
  uint32_t* const Rbuf[2] = {Rc, Rn};

  if (warp < kElimWarps) {
    for (int leaf = 0; leaf < K; ++leaf) {
      // stable sort of delta, descending (src/sigma_basis.rs:357-359): lane q
      // takes the row of sorted position q
      if (warp == 0 && lane < m) {
        const int64_t di = sdelta[lane];
        int pos = 0;
        for (int j = 0; j < m; ++j) {
          const int64_t dj = sdelta[j];
          pos += (dj > di) || (dj == di && j < lane);
        }
        perm[pos] = lane;
      }
      elim_bar();
      const int myrow = lane < m ? perm[lane] : 0;
      // this warp's columns of row `lane` of A = [pi r | pi] (src/sigma_basis.rs:369-380)
      const int c0 = kElimColsPerWarp * warp;
      uint32_t a[kElimColsPerWarp];
#pragma unroll
      for (int cl = 0; cl < kElimColsPerWarp; ++cl) {
        const int c = c0 + cl;
        uint32_t v = 0;
        if (lane < m && c < W) v = c < n ? R0[myrow * n + c] : ((c - n) == myrow ? 1u : 0u);
        a[cl] = v;
      }
      // LSP elimination (src/modular_linalg.rs:188-239), fraction-free:
      // row_i <- (piv row_i - a_i,cs row_k) R^{-1}.  Every warp keeps the list
      // positions of the unpivoted columns (lane c < n; -1 once pivoted) and
      // picks the non-zero column of least position.  The owners of the first
      // n columns publish them for all rows after every update (double
      // buffered), so one barrier per pivot step lets each warp read both row
      // k and the pivot column.
      int lpos = lane < n ? lane : -1;
      int rank = 0, cur = 0;
      bool piv_row = false;
      auto publish = [&](uint32_t* dst) {
        if (lane < m) {
#pragma unroll
          for (int cl = 0; cl < kElimColsPerWarp; ++cl)
            if (c0 + cl < n) dst[lane * kRpartStride + c0 + cl] = a[cl];
        }
      };
      publish(rpart);
      elim_bar();
      for (int k = 0; k < m && rank < n; ++k) {
        const uint32_t* rp = rpart + cur * kRpartSize;
        const uint32_t mine = lane < n ? rp[k * kRpartStride + lane] : 0u;
        const int key = (lpos >= 0 && mine != 0) ? ((lpos << 5) | lane) : 0x7fffffff;
        const int best = __reduce_min_sync(0xffffffffu, key);
        if (best == 0x7fffffff) continue;  // no pivot in row k (same decision in every warp)
        const int cs = best & 31, ts = best >> 5;
        if (lpos >= 0) lpos = (lane == cs) ? -1 : (lpos == 0 ? ts - 1 : lpos - 1);
        ++rank;
        piv_row = piv_row || (lane == k);
        const uint32_t f = lane < m ? rp[lane * kRpartStride + cs] : 0u;
        const uint32_t piv = rp[k * kRpartStride + cs];
        const uint32_t nf = p - f;
        const bool upd = lane > k && lane < m;
#pragma unroll
        for (int cl = 0; cl < kElimColsPerWarp; ++cl) {
          const uint32_t ak = __shfl_sync(0xffffffffu, a[cl], k);
          const uint32_t nv = redc_2mac(piv, a[cl], nf, ak, M);
          a[cl] = upd ? nv : a[cl];
        }
        if (rank < n) {  // the last pivot's update is final: nobody reads it back
          cur ^= 1;
          publish(rpart + cur * kRpartSize);
          elim_bar();
        }
      }
      // T (transposed) = columns n.. of A; c_i = T[i][perm[i]] (owned by one warp)
      uint32_t* Tg = P.Tt + (size_t)leaf * m * m;
#pragma unroll
      for (int cl = 0; cl < kElimColsPerWarp; ++cl) {
        const int c = c0 + cl;
        if (c >= n && c < W && lane < m) {
          const int s = c - n;
          Tq[s * TQS + lane] = a[cl];
          Tg[s * m + lane] = a[cl];
          if (s == myrow) {
            if (a[cl] == 0) atomicExch(P.status, 2);
            sig_tmp[lane] = redc((uint64_t)a[cl] * sigma[myrow], M);
          }
        }
      }
      if (warp == 0) {
        const unsigned long long mx = (unsigned long long)__ballot_sync(0xffffffffu, piv_row && lane < m);
        if (lane < m) sdelta_tmp[lane] = sdelta[myrow] - (piv_row ? 1 : 0);  // src/sigma_basis.rs:408-411
        if (lane == 0) {
          P.mask[leaf] = mx;
          s_mx2[leaf & 1] = mx;
        }
      }
      elim_bar();
      if (warp == 0 && lane < m) {
        sigma[lane] = sig_tmp[lane];
        sdelta[lane] = sdelta_tmp[lane];
      }
      const int rem = K - leaf - 1;
      if (rem == 0) break;
      // coefficient 1 of this leaf's residual is U's (leaf - 1 > = 0), and
      // U's work on leaf - 1 no longer reads the planes of T_{leaf - 2}
      if (leaf > 0) {
        if (tid == 0) s_ok_e = wait_count(&s_c1, leaf) ? 1 : 0;
        elim_bar();
        if (!s_ok_e) break;
      }
      uint32_t* const Tpl = Tp + (leaf & 1) * 1024;
      // byte planes of T: row i, word w holds limb l of T[i][4w .. 4w+3]
      for (int e = tid; e < m * 8; e += kElimWarps * 32) {
        const int i = e >> 3, w = e & 7;
        uint32_t v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = (4 * w + j < m) ? Tq[(4 * w + j) * TQS + i] : 0u;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const uint32_t lo = __byte_perm(v[0], v[1], 0x40 + 0x11 * l) & 0xffffu;  // byte l of v0, byte l of v1
          const uint32_t hi = __byte_perm(v[2], v[3], 0x40 + 0x11 * l) & 0xffffu;
          Tpl[l * 256 + plane_word(i, w)] = lo | (hi << 16);
        }
      }
      elim_bar();
      // coefficient 0 of the next residual (products with coefficients 0 and 1)
      residual(warp, kElimWarps, 0, std::min(1, rem), 0, 0, Tpl, Rbuf[leaf & 1], Rbuf[(leaf + 1) & 1],
               s_mx2[leaf & 1], rem);
      elim_bar();
      if (tid == 0) {
        __threadfence_block();
        s_tready = leaf + 1;
      }
    }
  } else {
    const int uw = warp - kElimWarps, uwarps = kLeafWarps - kElimWarps;
    for (int leaf = 0; leaf + 1 < K; ++leaf) {
      if (tid == kElimWarps * 32) s_ok_u = wait_count(&s_tready, leaf + 1) ? 1 : 0;
      upd_bar();
      if (!s_ok_u) break;
      const int rem = K - leaf - 1;
      const uint32_t* Tpl = Tp + (leaf & 1) * 1024;
      const uint32_t* Rcl = Rbuf[leaf & 1];
      uint32_t* Rnl = Rbuf[(leaf + 1) & 1];
      const unsigned long long mx = s_mx2[leaf & 1];
      // coefficient 1 first (products with coefficients 1 and 2), then the rest
      residual(uw, uwarps, 1, std::min(2, rem), 1, rem - 1, Tpl, Rcl, Rnl, mx, rem);
      upd_bar();
      if (tid == kElimWarps * 32) {
        __threadfence_block();
        s_c1 = leaf + 1;
      }
      residual(uw, uwarps, 3, rem, 1, rem - 1, Tpl, Rcl, Rnl, mx, rem);
      upd_bar();
    }
  }
  __syncthreads();
  for (int i = tid; i < m; i += nt) {
    P.sigma_inv[i] = inv_fermat(sigma[i], M);
    P.delta[i] = sdelta[i];
  }
}

// Block basis on the int8 tensor cores (2b <= 32): CTA (j, z) keeps column j
// of generator z's block basis as byte planes Vp[limb][t][8 words]
// (coefficient t = plane row, K index s = byte s) and applies
//   V_{k+1}[t' + mask_k(i)][i] = (T_k V_k[t'])[i] 2^-32,
// the same Montgomery convention as the CUDA-core kernel below, with exact
// u8-limb mma.sync products (T_k staged as byte planes as in the leaves kernel).
__device__ __forceinline__ uint32_t plane_load(const uint32_t* coeff, int NPc, int col, int row) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(coeff);
  const int wo = plane_word(col, row >> 2), bo = row & 3;
  uint32_t v = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l) v |= (uint32_t)b[4 * (l * NPc * 8 + wo) + bo] << (8 * l);
  return v;
}

// Plane rows of the block basis kernel: K + 2 coefficients, multiple of 8.
__host__ __device__ constexpr int bb_rows(int K) { return (K + 2 + 7) & ~7; }

size_t block_basis_mma_smem_bytes(int K) { return ((size_t)2 * 4 * bb_rows(K) * 8 + 1024) * 4; }

__global__ void __launch_bounds__(256) pm_block_basis_mma_kernel(const uint32_t* __restrict__ Tt,
                                                                 const unsigned long long* __restrict__ mask,
                                                                 const uint32_t* __restrict__ sigma_inv, int m, int K,
                                                                 uint32_t* Mout, int64_t out_rs, int64_t out_cs,
                                                                 int64_t out_bs, ModP M) {
  extern __shared__ __align__(16) uint32_t bbm_smem[];
  Tt += (int64_t)blockIdx.y * K * m * m;
  mask += (int64_t)blockIdx.y * K;
  sigma_inv += (int64_t)blockIdx.y * m;
  Mout += (int64_t)blockIdx.y * out_bs;
  const int VR = bb_rows(K);
  uint32_t* Vc = bbm_smem;          // [4][VR][8] byte planes of V_k
  uint32_t* Vn = Vc + 4 * VR * 8;   // V_{k+1}
  uint32_t* Tp = Vn + 4 * VR * 8;   // [4][32][8] byte planes of T_k
  const int j = blockIdx.x;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const uint32_t p = M.p;
  const uint32_t Wt[3] = {M.c32, (uint32_t)((uint64_t)M.c32 * 256 % p), (uint32_t)((uint64_t)M.c32 * 65536 % p)};
  const int MT = (m + 15) / 16;
  for (int e = tid; e < 2 * 4 * VR * 8 + 1024; e += nt) bbm_smem[e] = 0;
  __syncthreads();
  if (tid == 0) plane_store(Vc, VR, 0, j, 1u);  // V_0 = e_j
  for (int k = 0; k < K; ++k) {
    const unsigned long long mk = mask[k];
    const uint32_t* Tk = Tt + (size_t)k * m * m;  // Tk[s * m + i] = T_k[i][s]
    for (int e = tid; e < m * 8; e += nt) {
      const int i = e >> 3, w = e & 7;
      uint32_t v[4];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) v[jj] = (4 * w + jj < m) ? Tk[(4 * w + jj) * m + i] : 0u;
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const uint32_t lo = __byte_perm(v[0], v[1], 0x40 + 0x11 * l) & 0xffffu;
        const uint32_t hi = __byte_perm(v[2], v[3], 0x40 + 0x11 * l) & 0xffffu;
        Tp[l * 256 + plane_word(i, w)] = lo | (hi << 16);
      }
    }
    for (int e = tid; e < 4 * (k + 2) * 8; e += nt) {  // rows 0 .. k+1 of V_{k+1}
      const int l = e / ((k + 2) * 8), r = e - l * (k + 2) * 8;
      Vn[l * VR * 8 + r] = 0;
    }
    __syncthreads();
    const int NTk = (k + 1 + 7) / 8;
    for (int job = warp; job < MT * NTk; job += nwarps) {
      const int mt = job / NTk, ntl = job % NTk;
      const int r0 = mt * 16 + g, r1 = r0 + 8, col = ntl * 8 + g;
      uint32_t A[4][4], Bf[4][2];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        A[l][0] = Tp[l * 256 + plane_word(r0, t4)];
        A[l][1] = Tp[l * 256 + plane_word(r1, t4)];
        A[l][2] = Tp[l * 256 + plane_word(r0, t4 + 4)];
        A[l][3] = Tp[l * 256 + plane_word(r1, t4 + 4)];
        Bf[l][0] = Vc[l * VR * 8 + plane_word(col, t4)];
        Bf[l][1] = Vc[l * VR * 8 + plane_word(col, t4 + 4)];
      }
      int C[7][4];
#pragma unroll
      for (int q = 0; q < 7; ++q)
#pragma unroll
        for (int v = 0; v < 4; ++v) C[q][v] = 0;
#pragma unroll
      for (int l = 0; l < 4; ++l)
#pragma unroll
        for (int r = 0; r < 4; ++r) leaf_mma_u8(C[l + r], A[l], Bf[r][0], Bf[r][1]);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int row = (v < 2) ? r0 : r1;
        const int tp = ntl * 8 + 2 * t4 + (v & 1);
        if (row < m && tp <= k) {
          const uint64_t x = (uint64_t)(uint32_t)C[0][v] + ((uint64_t)(uint32_t)C[1][v] << 8) +
                             ((uint64_t)(uint32_t)C[2][v] << 16) + ((uint64_t)(uint32_t)C[3][v] << 24);
          uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
          mac_cc((uint32_t)C[4][v], Wt[0], lo, hi);
          mac_cc((uint32_t)C[5][v], Wt[1], lo, hi);
          mac_cc((uint32_t)C[6][v], Wt[2], lo, hi);
          plane_store(Vn, VR, tp + (int)((mk >> row) & 1ull), row, redc_cc(lo, hi, M));
        }
      }
    }
    __syncthreads();
    uint32_t* tv = Vc;
    Vc = Vn;
    Vn = tv;
  }
  for (int e = tid; e < (K + 1) * m; e += nt) {
    const int t = e / m, r = e % m;
    Mout[(int64_t)r * out_rs + (int64_t)j * out_cs + t] = mulmod(plane_load(Vc, VR, t, r), sigma_inv[r], M);
  }
}

// Block basis, one CTA per column j: V_0 = e_j, V_{k+1}[t][i] = T_k[i] . V_k[t - mask_k(i)]
// (t <= k + 1), with the same Montgomery convention as the residual; then
// Mout[i][j][t] = V_K[t][i] sigma_inv[i].  Rows are taken in the grouped slot
// order of the leaves kernel, four per thread, so the four rows of a thread
// read one source coefficient.
template <int FE>
__global__ void __launch_bounds__(256) pm_block_basis_kernel(const uint32_t* __restrict__ Tt,
                                                             const unsigned long long* __restrict__ mask,
                                                             const uint32_t* __restrict__ sigma_inv, int m, int K,
                                                             uint32_t* Mout, int64_t out_rs, int64_t out_cs,
                                                             int64_t out_bs, ModP M) {
  extern __shared__ __align__(16) uint32_t bb_smem[];
  // matrix blockIdx.y of the batch
  Tt += (int64_t)blockIdx.y * K * m * m;
  mask += (int64_t)blockIdx.y * K;
  sigma_inv += (int64_t)blockIdx.y * m;
  Mout += (int64_t)blockIdx.y * out_bs;
  const int S = m + 1;            // row stride of V
  const int TS = leaf_tstride(m); // row stride of the slot-ordered transform
  const int VS = ((K + 1) * S + 3) & ~3;  // words per V buffer (16-byte multiple)
  uint32_t* Vc = bb_smem;                  // [K+1][S]
  uint32_t* Vn = Vc + VS;                  // [K+1][S]
  uint32_t* Ts = Vn + VS;                  // [m][TS], Ts[s][slot]
  int* srow = reinterpret_cast<int*>(Ts + m * TS);  // [TS]
  const int j = blockIdx.x;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < (K + 1) * S; e += nt) Vc[e] = (e == j) ? 1u : 0u;
  for (int k = 0; k < K; ++k) {
    const unsigned long long mk = mask[k];
    const int nx = __popcll(mk);
    const int gx = (nx + 3) & ~3, QG = (gx + ((m - nx + 3) & ~3)) / 4;
    const uint32_t* Tk = Tt + (size_t)k * m * m;
    for (int q = tid; q < TS; q += nt) srow[q] = -1;
    __syncthreads();
    for (int i = tid; i < m; i += nt) srow[leaf_slot(mk, i, m)] = i;
    __syncthreads();
    for (int e = tid; e < m * TS; e += nt) {
      const int s = e / TS, q = e % TS;
      const int r = srow[q];
      Ts[e] = r >= 0 ? Tk[s * m + r] : 0u;
    }
    __syncthreads();
    const int jobs = (k + 2) * QG;
    for (int job = tid; job < jobs; job += nt) {
      const int t = job / QG, q0 = 4 * (job % QG);
      const int st = t - (q0 < gx ? 1 : 0);
      uint64_t acc[4] = {0, 0, 0, 0};
      if (st >= 0 && st <= k) {
        const uint32_t* w = Ts + q0;
        const uint32_t* x = Vc + st * S;
        int s = 0;
        for (; s + FE <= m; s += FE) {
#pragma unroll
          for (int u = 0; u < FE; ++u) {
            const uint4 wv = *reinterpret_cast<const uint4*>(w);
            const uint32_t xv = x[s + u];
            acc[0] = mad_wide(wv.x, xv, acc[0]);
            acc[1] = mad_wide(wv.y, xv, acc[1]);
            acc[2] = mad_wide(wv.z, xv, acc[2]);
            acc[3] = mad_wide(wv.w, xv, acc[3]);
            w += TS;
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[r] = fold(acc[r], M);
        }
        for (; s < m; ++s) {
          const uint4 wv = *reinterpret_cast<const uint4*>(w);
          const uint32_t xv = x[s];
          acc[0] = fold(mad_wide(wv.x, xv, acc[0]), M);
          acc[1] = fold(mad_wide(wv.y, xv, acc[1]), M);
          acc[2] = fold(mad_wide(wv.z, xv, acc[2]), M);
          acc[3] = fold(mad_wide(wv.w, xv, acc[3]), M);
          w += TS;
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = srow[q0 + r];
        if (row >= 0) Vn[t * S + row] = (st >= 0 && st <= k) ? redc(acc[r], M) : 0u;
      }
    }
    __syncthreads();
    uint32_t* tv = Vc;
    Vc = Vn;
    Vn = tv;
  }
  for (int e = tid; e < (K + 1) * m; e += nt) {
    const int t = e / m, r = e % m;
    Mout[(int64_t)r * out_rs + (int64_t)j * out_cs + t] = mulmod(Vc[t * S + r], sigma_inv[r], M);
  }
}

// ---------------------------------------------------------------- host side
uint32_t find_generator(uint32_t p) {
  std::vector<uint32_t> fac;
  uint32_t t = p - 1;
  for (uint32_t q = 2; (uint64_t)q * q <= t; ++q)
    if (t % q == 0) {
      fac.push_back(q);
      while (t % q == 0) t /= q;
    }
  if (t > 1) fac.push_back(t);
  for (uint32_t g = 2; g < p; ++g) {
    bool ok = true;
    for (uint32_t q : fac)
      if (host_powmod(g, (p - 1) / q, p) == 1) { ok = false; break; }
    if (ok) return g;
  }
  return 0;
}

int grid_for(int64_t work, int threads = 256) {
  const int64_t b = (work + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

// An NTT prime q with its twiddle tables (w^j and Shoup quotients, forward
// and inverse, j < nmax / 2) and the pointwise stage's fold rule.
struct NttPrime {
  uint32_t q = 0;
  ModP M{};
  int fold4 = 0;
  int64_t nmax = 0;
  DevBuf<uint32_t> tw, tws, twi, twis;
  Twiddles fwd() const { return Twiddles{tw.ptr, tws.ptr, nmax}; }
  Twiddles inv() const { return Twiddles{twi.ptr, twis.ptr, nmax}; }
};

// Four products fit between folds of a 64-bit accumulator iff
// (2^32 - 1) * c32 + 2^32 - 1 + 4 (q - 1)^2 < 2^64.
int fold4_ok(uint32_t q, const ModP& M) {
  const unsigned __int128 F = (unsigned __int128)0xffffffffull * M.c32 + 0xffffffffull;
  const unsigned __int128 sq = (unsigned __int128)(q - 1) * (q - 1);
  return (F + 4 * sq) < ((unsigned __int128)1 << 64);
}

// The three largest NTT primes below 2^31 (2-adic orders 27, 25, 24): the
// exact-integer products of primes without a suitable NTT are taken modulo
// the first two or three of them.
constexpr uint32_t kCrtPrimes[3] = {2013265921u, 2113929217u, 2130706433u};

struct Pm {
  rr_ctx* ctx = nullptr;
  cudaStream_t s = nullptr;
  int m = 0, n = 0;
  int nb = 1;  // generators solved together (same b, d, p)
  uint32_t p = 0;
  ModP M{};
  int K = 0;
  bool use_ntt = false;
  int64_t nmax = 0;
  // transform primes: {p} when p - 1 is divisible by nmax, else two or three
  // of kCrtPrimes with the products combined by CRT
  std::vector<std::unique_ptr<NttPrime>> nps;
  bool crt = false;
  DevBuf<uint32_t> R[3];                // CRT residues [nb][m*m][d+1] per prime
  DevBuf<uint32_t> FA, FB, FC;          // [nb][m*m][nmax]
  DevBuf<uint32_t> Tt;                  // leaf transforms of one block [nb][K][m][m]
  DevBuf<unsigned long long> leafmask;  // [nb][K]
  DevBuf<uint32_t> sigma_inv;           // [nb][m]
  DevBuf<int64_t> delta;                // [nb][m]
  DevBuf<int> status;
  int64_t cs = 0;                      // residual coefficient stride of the leaves kernel (words)
  int fold4 = 0;
  bool mma = false;                    // tensor-core leaves kernel (b <= 16)
  // per recursion depth: MM, GG, MMM ([nb] each)
  std::vector<std::unique_ptr<DevBuf<uint32_t>>> bufs;
};

// A strided polynomial matrix of every generator of the batch: entry (i, j)
// of generator z starts at p + z * bs + i * rs + j * cs.
struct MatView {
  uint32_t* p;
  int64_t rs, cs, bs;
  PolyView polys(int cols, int rows) const { return PolyView{p, cols, rows * cols, rs, cs, bs}; }
};

// NTTs of the npb polynomials of each of the nb generators in src (zero
// padded to N) into a (dense, [nb * npb][N]).
// Launch shape of the shared-memory NTT kernels for span T over nblocks blocks.
struct NttShape {
  int logT, G, threads;
  unsigned grid;
  size_t smem;
};
NttShape ntt_shape(int64_t T, int64_t nblocks) {
  NttShape sh;
  sh.logT = 0;
  while ((1ll << sh.logT) < T) ++sh.logT;
  sh.G = T >= kNttGroup ? 1 : (int)(kNttGroup / T);
  sh.threads = (int)std::min<int64_t>(512, std::max<int64_t>(32, sh.G * T / 2));
  sh.grid = (unsigned)((nblocks + sh.G - 1) / sh.G);
  sh.smem = (size_t)(sh.G * T + T) * 4;
  return sh;
}

int ntt_forward(Pm& P, const NttPrime& Q, uint32_t* a, int64_t N, PolyView src, int64_t src_len) {
  const int64_t npoly = (int64_t)P.nb * src.npb;
  const int64_t T = std::min<int64_t>(N, kNttBlock);
  if (N <= kNttBlock) {
    const NttShape sh = ntt_shape(T, npoly);
    ntt_fwd_smem_kernel<<<sh.grid, sh.threads, sh.smem, P.s>>>(a, N, sh.logT, npoly, src, src_len, Q.fwd(), Q.q);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  pad_copy_kernel<<<grid_for(npoly * N), 256, 0, P.s>>>(a, N, npoly, src, src_len, Q.q);
  RR_CUDA(cudaGetLastError());
  for (int64_t len = N; len > kNttBlock; len >>= 1) {
    ntt_fwd_stage_kernel<<<grid_for(npoly * N / 2), 256, 0, P.s>>>(a, N, npoly, len, Q.fwd(), Q.q);
    RR_CUDA(cudaGetLastError());
  }
  const PolyView none{nullptr, 1, 1, 0, 0, 0};
  const NttShape sh = ntt_shape(T, npoly * (N / T));
  ntt_fwd_smem_kernel<<<sh.grid, sh.threads, sh.smem, P.s>>>(a, N, sh.logT, npoly * (N / T), none, 0, Q.fwd(), Q.q);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// Inverse NTTs of a ([nb * npb][N]); coefficients [lo, lo + cnt), scaled by
// N^{-1}, go to dst.
int ntt_inverse(Pm& P, const NttPrime& Q, uint32_t* a, int64_t N, PolyView dst, int64_t lo, int64_t cnt) {
  const int64_t npoly = (int64_t)P.nb * dst.npb;
  const int64_t T = std::min<int64_t>(N, kNttBlock);
  const uint32_t ninv = host_invmod((uint32_t)(N % Q.q), Q.q);
  const uint32_t ninv_s = (uint32_t)(((uint64_t)ninv << 32) / Q.q);
  if (N <= kNttBlock) {
    const NttShape sh = ntt_shape(T, npoly);
    ntt_inv_smem_kernel<<<sh.grid, sh.threads, sh.smem, P.s>>>(a, N, sh.logT, npoly, dst, lo, cnt, ninv, ninv_s,
                                                               Q.inv(), Q.q);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  const PolyView none{nullptr, 1, 1, 0, 0, 0};
  const NttShape sh = ntt_shape(T, npoly * (N / T));
  ntt_inv_smem_kernel<<<sh.grid, sh.threads, sh.smem, P.s>>>(a, N, sh.logT, npoly * (N / T), none, 0, 0, 0, 0,
                                                             Q.inv(), Q.q);
  RR_CUDA(cudaGetLastError());
  for (int64_t len = 2 * kNttBlock; len <= N; len <<= 1) {
    ntt_inv_stage_kernel<<<grid_for(npoly * N / 2), 256, 0, P.s>>>(a, N, npoly, len, Q.inv(), Q.q);
    RR_CUDA(cudaGetLastError());
  }
  extract_scale_kernel<<<grid_for(npoly * cnt), 256, 0, P.s>>>(a, N, npoly, dst, lo, cnt, ninv, ninv_s, Q.q);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// One NTT product modulo the transform prime Q: coefficients [lo, lo + cnt)
// of A * B into dst.
int ntt_product(Pm& P, const NttPrime& Q, MatView A, int mA, int r, int64_t la, MatView B, int k, int64_t lb,
                int64_t N, PolyView dst, int64_t lo, int64_t cnt) {
  RR_TRY(ntt_forward(P, Q, P.FA.ptr, N, A.polys(r, mA), la));
  RR_TRY(ntt_forward(P, Q, P.FB.ptr, N, B.polys(k, r), lb));
  if (mA % 4 == 0 && k % 4 == 0)
    pointwise_kernel<<<grid_for((int64_t)P.nb * (mA / 4) * (k / 4) * N), 256, 0, P.s>>>(
        P.FA.ptr, P.FB.ptr, P.FC.ptr, mA, r, k, N, P.nb, Q.fold4 ? 3 : 1, Q.M);
  else
    pointwise1_kernel<<<grid_for((int64_t)P.nb * mA * k * N), 256, 0, P.s>>>(P.FA.ptr, P.FB.ptr, P.FC.ptr, mA, r, k, N,
                                                                              P.nb, Q.M);
  RR_CUDA(cudaGetLastError());
  return ntt_inverse(P, Q, P.FC.ptr, N, dst, lo, cnt);
}

CrtParams crt_params(const Pm& P) {
  CrtParams C;
  C.k = (int)P.nps.size();
  for (int i = 0; i < 3; ++i) {
    C.q[i] = i < C.k ? P.nps[i]->q : 1u;
    C.Mq[i] = i < C.k ? P.nps[i]->M : ModP{};
  }
  const uint32_t q0 = C.q[0], q1 = C.q[1];
  C.c01 = host_invmod(q0 % q1, q1);
  C.c02 = C.k == 3 ? host_invmod(q0 % C.q[2], C.q[2]) : 0;
  C.c12 = C.k == 3 ? host_invmod(q1 % C.q[2], C.q[2]) : 0;
  C.q0p = q0 % P.p;
  C.q01p = (uint32_t)((uint64_t)(q0 % P.p) * (q1 % P.p) % P.p);
  C.Mp = P.M;
  return C;
}

// dst[i][j][0..cnt) = coefficients [lo, lo+cnt) of A * B for every generator
// of the batch, where A is mA x r with la coefficients and B is r x k with lb
// coefficients.
int poly_mat_mul(Pm& P, MatView A, int mA, int r, int64_t la, MatView B, int k, int64_t lb, MatView dst, int64_t lo,
                 int64_t cnt) {
  int64_t N = 1;
  while (N < la + lb - 1) N <<= 1;
  if (!P.use_ntt) {
    schoolbook_kernel<<<grid_for((int64_t)P.nb * mA * k * cnt), 256, 0, P.s>>>(
        A.p, mA, r, la, A.rs, A.cs, A.bs, B.p, k, lb, B.rs, B.cs, B.bs, dst.p, dst.rs, dst.cs, dst.bs, lo, cnt, P.nb,
        P.M);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  if (N > P.nmax) return fail(RR_EINVAL, "internal: NTT length %lld exceeds table %lld", (long long)N, (long long)P.nmax);
  if (!P.crt) return ntt_product(P, *P.nps[0], A, mA, r, la, B, k, lb, N, dst.polys(k, mA), lo, cnt);
  // residues per transform prime, dense [nb][mA * k][cnt], then CRT into dst
  const int64_t per = (int64_t)mA * k * cnt;
  for (size_t i = 0; i < P.nps.size(); ++i) {
    const PolyView Rv{P.R[i].ptr, k, mA * k, (int64_t)k * cnt, cnt, per};
    RR_TRY(ntt_product(P, *P.nps[i], A, mA, r, la, B, k, lb, N, Rv, lo, cnt));
  }
  const int64_t npoly = (int64_t)P.nb * mA * k;
  crt_kernel<<<grid_for(npoly * cnt), 256, 0, P.s>>>(P.R[0].ptr, P.R[1].ptr, P.nps.size() > 2 ? P.R[2].ptr : nullptr,
                                                     npoly, cnt, dst.polys(k, mA), crt_params(P));
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

int run_base(Pm& P, MatView G, int nleaves, MatView Mout) {
  LeafParams L;
  L.G = G.p;
  L.g_rs = G.rs;
  L.g_cs = G.cs;
  L.g_bs = G.bs;
  L.m = P.m;
  L.n = P.n;
  L.K = nleaves;
  L.cs = P.cs;
  L.delta = P.delta.ptr;
  L.Tt = P.Tt.ptr;
  L.mask = P.leafmask.ptr;
  L.sigma_inv = P.sigma_inv.ptr;
  L.M = P.M;
  L.status = P.status.ptr;
  const unsigned nb = (unsigned)P.nb;
  if (P.mma) {
    pm_leaves_mma_kernel<<<nb, kLeafThreads, leaves_mma_smem_bytes(P.m, P.n, nleaves), P.s>>>(L);
  } else if (P.n % 4 == 0) {
    const size_t smem = leaves_smem_bytes(P.m, P.n, nleaves, P.cs);
    if (P.fold4) pm_leaves_kernel<4, 4><<<nb, kLeafThreads, smem, P.s>>>(L);
    else pm_leaves_kernel<4, 2><<<nb, kLeafThreads, smem, P.s>>>(L);
  } else {
    const size_t smem = leaves_smem_bytes(P.m, P.n, nleaves, P.cs);
    if (P.fold4) pm_leaves_kernel<1, 4><<<nb, kLeafThreads, smem, P.s>>>(L);
    else pm_leaves_kernel<1, 2><<<nb, kLeafThreads, smem, P.s>>>(L);
  }
  RR_CUDA(cudaGetLastError());
  // the leaves kernel indexes its transforms with the block's own K; the
  // block basis reads them with the same K
  const dim3 grid((unsigned)P.m, nb);
  if (P.mma) {
    pm_block_basis_mma_kernel<<<grid, 256, block_basis_mma_smem_bytes(nleaves), P.s>>>(
        P.Tt.ptr, P.leafmask.ptr, P.sigma_inv.ptr, P.m, nleaves, Mout.p, Mout.rs, Mout.cs, Mout.bs, P.M);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  const size_t bsm = block_basis_smem_bytes(P.m, nleaves);
  if (P.fold4)
    pm_block_basis_kernel<4><<<grid, 256, bsm, P.s>>>(P.Tt.ptr, P.leafmask.ptr, P.sigma_inv.ptr, P.m, nleaves, Mout.p,
                                                      Mout.rs, Mout.cs, Mout.bs, P.M);
  else
    pm_block_basis_kernel<2><<<grid, 256, bsm, P.s>>>(P.Tt.ptr, P.leafmask.ptr, P.sigma_inv.ptr, P.m, nleaves, Mout.p,
                                                      Mout.rs, Mout.cs, Mout.bs, P.M);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// Residual coefficient stride of the leaves kernel: m * n rounded to 16-byte
// words plus 4, so that neighbouring coefficients start in different banks.
int64_t leaf_coeff_stride(int m, int n) { return (((int64_t)m * n + 3) & ~(int64_t)3) + 4; }

// Largest block of leaves (a power of two <= 64 for m <= 16, <= 32 otherwise,
// and <= d) whose double-buffered residual fits in shared memory.
int pick_block_leaves(int m, int n, int64_t d, bool mma, size_t* smem) {
  const int kmax = m <= 16 ? 64 : 32;
  int K = (int)std::min<int64_t>(d, kmax);
  const int64_t cs = leaf_coeff_stride(m, n);
  auto bytes = [&](int k) { return mma ? leaves_mma_smem_bytes(m, n, k) : leaves_smem_bytes(m, n, k, cs); };
  while (K > 1 && bytes(K) > kBaseSmemBudget) K /= 2;
  *smem = bytes(K);
  return K;
}

int set_leaves_smem_limit(size_t bytes, size_t basis_bytes) {
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  RR_CUDA(cudaFuncSetAttribute(pm_leaves_kernel<4, 4>, attr, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_leaves_kernel<4, 2>, attr, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_leaves_kernel<1, 4>, attr, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_leaves_kernel<1, 2>, attr, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_leaves_mma_kernel, attr, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_block_basis_kernel<4>, attr, (int)basis_bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_block_basis_kernel<2>, attr, (int)basis_bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_block_basis_mma_kernel, attr, (int)block_basis_mma_smem_bytes(64)));
  return RR_OK;
}

int set_base_smem_limit(size_t bytes) {
  RR_CUDA(cudaFuncSetAttribute(pm_base_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_base_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return RR_OK;
}

// _PM_Basis (src/sigma_basis.rs:190-219) on G (m x n, coefficients [0, d]
// used) for every generator of the batch; Mo receives m x m x (d+1).
int pm_rec(Pm& P, MatView G, int64_t d, int depth, MatView Mo) {
  if (d <= P.K) return run_base(P, G, (int)d, Mo);
  const int m = P.m, n = P.n;
  const int64_t h = d / 2;
  const int64_t hl = h + 1;
  const MatView MM{P.bufs[3 * depth + 0]->ptr, (int64_t)m * hl, hl, (int64_t)m * m * hl};   // m x m x (h+1)
  const MatView GG{P.bufs[3 * depth + 1]->ptr, (int64_t)n * hl, hl, (int64_t)m * n * hl};   // m x n x (h+1)
  const MatView MMM{P.bufs[3 * depth + 2]->ptr, (int64_t)m * hl, hl, (int64_t)m * m * hl};  // m x m x (h+1)
  RR_TRY(pm_rec(P, G, h, depth + 1, MM));
  // GG = (MM * G)[h .. d]   (poly_mat_mul_red_adaptive(MM, G, p, 0, d+1) + shift_trunc_in(h, h))
  RR_TRY(poly_mat_mul(P, MM, m, m, hl, G, n, d + 1, GG, h, hl));
  RR_TRY(pm_rec(P, GG, h, depth + 1, MMM));
  // M = MMM * MM
  return poly_mat_mul(P, MMM, m, m, hl, MM, m, hl, Mo, 0, d + 1);
}

}  // namespace

// Device bytes the batched generator holds per generator of degree d and width b.
size_t pm_workspace_bytes(int b, int64_t d) {
  const size_t m = 2 * (size_t)b, n = (size_t)b;
  int64_t nmax = 1;
  while (nmax < d + d / 2 + 1) nmax <<= 1;
  size_t bytes = 3 * m * m * (size_t)nmax * 4;               // NTT workspace
  for (int64_t dd = d; dd > 1; dd /= 2) bytes += (2 * m * m + m * n) * (size_t)(dd / 2 + 1) * 4;  // per depth
  bytes += (m * n + m * m) * (size_t)(d + 1) * 4 + (size_t)b * (b + 1) / 2 * (size_t)(d + 1) * 4;  // G, Mo, seq
  bytes += 64 * m * m * 4;                                    // leaf transforms
  bytes += 3 * m * m * (size_t)(d + 1) * 4;                   // CRT residues (primes without a suitable NTT)
  return bytes;
}

// PM-basis of nb generators with the same b, d and p, solved in lockstep: one
// leaf-kernel CTA per generator, one launch per NTT / product step for all.
int pm_basis_batch_device(rr_ctx* ctx, int nb, const uint32_t* const* seqs, const int64_t* seq_strides, int b,
                          int64_t d, uint32_t p, uint32_t* const* Mh, int64_t* const* deltah) {
  if (nb < 1) return RR_OK;
  Pm P;
  P.ctx = ctx;
  P.s = ctx->stream;
  P.nb = nb;
  P.m = 2 * b;
  P.n = b;
  P.p = p;
  P.M = make_modp(p);
  size_t leaves_smem = 0;
  P.mma = ctx->pm_tensor_cores && P.m <= kMmaRows && P.n <= kMmaCols;
  P.K = pick_block_leaves(P.m, P.n, d, P.mma, &leaves_smem);
  P.cs = leaf_coeff_stride(P.m, P.n);
  P.fold4 = fold4_ok(p, P.M);
  const int m = P.m, n = P.n;
  // NTT table for the largest product: length nextpow2(3d/2 + 1) = 2d (d >= 2)
  int64_t nmax = 1;
  while (nmax < d + d / 2 + 1) nmax <<= 1;
  nmax = std::max<int64_t>(nmax, 2);
  P.nmax = nmax;
  // NTT products: modulo p itself when p - 1 is divisible by the transform
  // length, else exact integer products by CRT over two or three NTT primes
  // (whose product must exceed inner dimension x length x (p-1)^2)
  P.use_ntt = d > P.K;
  if (P.use_ntt) {
    std::vector<uint32_t> qs;
    if ((uint64_t)(p - 1) % (uint64_t)nmax == 0) {
      qs.push_back(p);
    } else {
      P.crt = true;
      const long double bound = (long double)m * (long double)(d + 1) * (long double)(p - 1) * (long double)(p - 1);
      long double prod = 1;
      for (int i = 0; i < 3 && prod <= bound; ++i) {
        if ((uint64_t)(kCrtPrimes[i] - 1) % (uint64_t)nmax != 0)
          return fail(RR_EUNSUPPORTED, "d = %lld: NTT length %lld beyond the CRT primes", (long long)d, (long long)nmax);
        qs.push_back(kCrtPrimes[i]);
        prod *= kCrtPrimes[i];
      }
      if (prod <= bound) return fail(RR_EUNSUPPORTED, "d = %lld too large for a three-prime CRT at p = %u", (long long)d, p);
      if (qs.size() < 2) qs.push_back(kCrtPrimes[1]);  // Garner needs two residues
    }
    std::vector<uint32_t> t(nmax / 2), ts(nmax / 2), ti(nmax / 2), tis(nmax / 2);
    for (uint32_t q : qs) {
      std::unique_ptr<NttPrime> Q(new NttPrime());
      Q->q = q;
      Q->M = make_modp(q);
      Q->fold4 = fold4_ok(q, Q->M);
      Q->nmax = nmax;
      const uint32_t g = find_generator(q);
      const uint32_t w = host_powmod(g, (q - 1) / (uint64_t)nmax, q);
      const uint32_t wi = host_invmod(w, q);
      uint64_t x = 1, y = 1;
      for (int64_t j = 0; j < nmax / 2; ++j) {
        t[j] = (uint32_t)x;
        ti[j] = (uint32_t)y;
        ts[j] = (uint32_t)((x << 32) / q);
        tis[j] = (uint32_t)((y << 32) / q);
        x = x * w % q;
        y = y * wi % q;
      }
      RR_TRY(Q->tw.alloc_async(nmax / 2, P.s));
      RR_TRY(Q->tws.alloc_async(nmax / 2, P.s));
      RR_TRY(Q->twi.alloc_async(nmax / 2, P.s));
      RR_TRY(Q->twis.alloc_async(nmax / 2, P.s));
      RR_CUDA(cudaMemcpyAsync(Q->tw.ptr, t.data(), t.size() * 4, cudaMemcpyHostToDevice, P.s));
      RR_CUDA(cudaMemcpyAsync(Q->tws.ptr, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice, P.s));
      RR_CUDA(cudaMemcpyAsync(Q->twi.ptr, ti.data(), ti.size() * 4, cudaMemcpyHostToDevice, P.s));
      RR_CUDA(cudaMemcpyAsync(Q->twis.ptr, tis.data(), tis.size() * 4, cudaMemcpyHostToDevice, P.s));
      RR_CUDA(cudaStreamSynchronize(P.s));  // the host tables are reused for the next prime
      P.nps.push_back(std::move(Q));
    }
    RR_TRY(P.FA.alloc_async((size_t)nb * m * m * nmax, P.s));
    RR_TRY(P.FB.alloc_async((size_t)nb * m * m * nmax, P.s));
    RR_TRY(P.FC.alloc_async((size_t)nb * m * m * nmax, P.s));
    if (P.crt)
      for (size_t i = 0; i < P.nps.size(); ++i) RR_TRY(P.R[i].alloc_async((size_t)nb * m * m * (d + 1), P.s));
  }
  // per-depth buffers
  {
    int depth = 0;
    for (int64_t dd = d; dd > P.K; dd /= 2, ++depth) {
      const int64_t hl = dd / 2 + 1;
      for (int q = 0; q < 3; ++q) {
        P.bufs.emplace_back(new DevBuf<uint32_t>());
        RR_TRY(P.bufs.back()->alloc_async((size_t)nb * m * (q == 1 ? n : m) * hl, P.s));
      }
    }
  }
  RR_TRY(P.delta.alloc_async((size_t)nb * m, P.s));
  RR_TRY(P.status.alloc_async(1, P.s));
  RR_TRY(P.Tt.alloc_async((size_t)nb * P.K * m * m, P.s));
  RR_TRY(P.leafmask.alloc_async((size_t)nb * P.K, P.s));
  RR_TRY(P.sigma_inv.alloc_async((size_t)nb * m, P.s));
  RR_CUDA(cudaMemsetAsync(P.delta.ptr, 0, (size_t)nb * m * sizeof(int64_t), P.s));
  RR_CUDA(cudaMemsetAsync(P.status.ptr, 0, sizeof(int), P.s));
  // the limits are per kernel, shared by every caller in the process (the
  // batched engine runs generators on several threads): always the budget,
  // never this call's size, so a concurrent smaller call cannot lower them
  if (leaves_smem > kBaseSmemBudget) return fail(RR_EUNSUPPORTED, "leaf block needs %zu bytes of shared memory", leaves_smem);
  RR_TRY(set_leaves_smem_limit(kBaseSmemBudget, block_basis_smem_bytes(64, 64)));
  // G = [S; I], coefficients [0, d], one after the other
  DevBuf<uint32_t> dseq, G;
  const int np = b * (b + 1) / 2;
  const int64_t glen = d + 1;
  RR_TRY(dseq.alloc_async((size_t)nb * np * glen, P.s));
  RR_TRY(G.alloc_async((size_t)nb * m * n * glen, P.s));
  for (int z = 0; z < nb; ++z) {
    uint32_t* dz = dseq.ptr + (size_t)z * np * glen;
    RR_CUDA(cudaMemcpy2DAsync(dz, glen * 4, seqs[z], seq_strides[z] * 4, glen * 4, np, cudaMemcpyHostToDevice, P.s));
    build_G_kernel<<<grid_for((int64_t)m * n * glen), 256, 0, P.s>>>(dz, glen, b, glen, G.ptr + (size_t)z * m * n * glen,
                                                                     p);
    RR_CUDA(cudaGetLastError());
  }
  DevBuf<uint32_t> Mo;
  RR_TRY(Mo.alloc_async((size_t)nb * m * m * (d + 1), P.s));
  const MatView Gv{G.ptr, (int64_t)n * glen, glen, (int64_t)m * n * glen};
  const MatView Mv{Mo.ptr, (int64_t)m * (d + 1), d + 1, (int64_t)m * m * (d + 1)};
  RR_TRY(pm_rec(P, Gv, d, 0, Mv));
  int status = 0;
  for (int z = 0; z < nb; ++z) {
    RR_CUDA(cudaMemcpyAsync(Mh[z], Mo.ptr + (size_t)z * m * m * (d + 1), (size_t)m * m * (d + 1) * 4,
                            cudaMemcpyDeviceToHost, P.s));
    RR_CUDA(cudaMemcpyAsync(deltah[z], P.delta.ptr + (size_t)z * m, m * sizeof(int64_t), cudaMemcpyDeviceToHost, P.s));
  }
  RR_CUDA(cudaMemcpyAsync(&status, P.status.ptr, sizeof(int), cudaMemcpyDeviceToHost, P.s));
  RR_CUDA(cudaStreamSynchronize(P.s));
  if (status == 3) return fail(RR_ETIMEOUT, "PM-basis leaf kernel: a hand-off between its warp groups gave up");
  if (status) return fail(RR_ECUDA, "PM-basis device status %d (zero row scale)", status);
  return RR_OK;
}

int pm_basis_device(rr_ctx* ctx, const uint32_t* seq, int64_t seq_stride, int b, int64_t nlen, int64_t d, uint32_t p,
                    uint32_t* Mh, int64_t* deltah) {
  (void)nlen;
  return pm_basis_batch_device(ctx, 1, &seq, &seq_stride, b, d, p, &Mh, &deltah);
}

// ---------------------------------------------------------------- no-allocation variant
// rr_pm_basis_short_noalloc builds G (build_G_kernel) and runs one block of
// leaves in one CTA of pm_base_kernel -- the original single-kernel block,
// kept for this entry point; rr_pm_basis now runs the leaves and the block
// basis as two kernels.  tests/test_zz_no_alloc.py checks both against each
// other and against the oracle.  Its scratch -- the matrix G, the base
// kernel's double-buffered basis and the status word -- comes from the
// file-scope array below instead of an allocation.
// Limits: b <= 16 and d (rounded up to a power of two) <= 32.
namespace {
constexpr int kNoallocMaxB = 16;
constexpr int kNoallocMaxD = 32;
constexpr size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaGOff = 0;
constexpr size_t kNaGBytes = round256((size_t)2 * kNoallocMaxB * kNoallocMaxB * (kNoallocMaxD + 1) * 4);
constexpr size_t kNaMbufOff = kNaGOff + kNaGBytes;
constexpr size_t kNaMbufBytes =
    round256((size_t)2 * (kNoallocMaxD + 1) * (2 * kNoallocMaxB) * (2 * kNoallocMaxB) * 4);
constexpr size_t kNaStatusOff = kNaMbufOff + kNaMbufBytes;
constexpr size_t kNoallocScratchBytes = kNaStatusOff + 256;  // 338,176 bytes
constexpr int kNoallocMaxDevices = 64;

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kNoallocMaxDevices] = {};
}  // namespace

// Held by every GPU that loads this library, until the process exits.
static __device__ __align__(256) unsigned char g_pm_noalloc_scratch[kNoallocScratchBytes];

// Device address of the scratch array on the current device, looked up once
// per device (host code must not use the symbol itself as an address).  The
// same first call per device raises pm_base_kernel's shared-memory limit to
// the largest size this entry point launches, so no later call changes a
// kernel attribute.
static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  RR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(RR_EUNSUPPORTED, "device %d beyond %d", dev, kNoallocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    RR_CUDA(cudaGetSymbolAddress(&p, g_pm_noalloc_scratch));
    RR_TRY(set_base_smem_limit(base_smem_bytes(2 * kNoallocMaxB, kNoallocMaxB, kNoallocMaxD, false)));
    g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_addr[dev];
  return RR_OK;
}

}  // namespace rr

extern "C" int rr_pm_basis_short_noalloc(const uint32_t* d_seq, int64_t seq_stride, int32_t b, int64_t nlen, int64_t d,
                                         uint32_t p, uint32_t* d_M, int64_t* d_delta, void* stream) {
  using namespace rr;
  if (!d_seq || !d_M || !d_delta) return fail(RR_EINVAL, "NULL argument");
  RR_TRY(rr_prime_check(p));
  if (b < 1 || b > kNoallocMaxB)
    return fail(RR_EINVAL, "b = %d outside the no-allocation limit 1 <= b <= %d", b, kNoallocMaxB);
  if (d < 1) return fail(RR_EINVAL, "d = %lld must be >= 1", (long long)d);
  int64_t dd = 1;
  while (dd < d) dd *= 2;
  if (dd > kNoallocMaxD)
    return fail(RR_EINVAL, "d = %lld (rounded to %lld) exceeds the no-allocation limit d <= %d; use rr_pm_basis",
                (long long)d, (long long)dd, kNoallocMaxD);
  if (dd >= nlen) return fail(RR_EINVAL, "sequence too short: d = %lld, nlen = %lld", (long long)dd, (long long)nlen);
  if (seq_stride < nlen) return fail(RR_EINVAL, "seq_stride < nlen");
  unsigned char* base = nullptr;
  RR_TRY(noalloc_scratch(&base));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int m = 2 * b, n = b;
  const int64_t glen = dd + 1;
  uint32_t* G = reinterpret_cast<uint32_t*>(base + kNaGOff);
  uint32_t* Mbuf = reinterpret_cast<uint32_t*>(base + kNaMbufOff);
  int* status = reinterpret_cast<int*>(base + kNaStatusOff);
  // delta starts at zero (src/sigma_basis.rs:48); the status word is cleared per call
  RR_CUDA(cudaMemsetAsync(d_delta, 0, (size_t)m * sizeof(int64_t), s));
  RR_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
  build_G_kernel<<<grid_for((int64_t)m * n * glen), 256, 0, s>>>(d_seq, seq_stride, b, glen, G, p);
  RR_CUDA(cudaGetLastError());
  BaseParams B;
  B.G = G;
  B.g_rs = (int64_t)n * glen;
  B.g_cs = glen;
  B.m = m;
  B.n = n;
  B.nleaves = (int)dd;
  B.delta = d_delta;
  B.Mout = d_M;
  B.out_rs = (int64_t)m * glen;
  B.out_cs = glen;
  B.Mbuf = Mbuf;
  B.m_smem = 0;  // the basis stays in the scratch array
  B.M = make_modp(p);
  B.status = status;
  const size_t bytes = base_smem_bytes(m, n, (int)dd, false);  // within the limit set at the first call
  if (n % 4 == 0) pm_base_kernel<4><<<1, kBaseThreads, bytes, s>>>(B);
  else pm_base_kernel<1><<<1, kBaseThreads, bytes, s>>>(B);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}
