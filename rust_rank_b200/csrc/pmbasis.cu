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

// ---------------------------------------------------------------- NTT kernels
// Forward DIF stage with butterfly span `len` (len > kNttBlock) in global memory.
__global__ void ntt_fwd_stage_kernel(uint32_t* a, int64_t N, int64_t npoly, int64_t len, Twiddles tw, uint32_t p) {
  const int64_t half = len / 2;
  const int64_t per = N / 2;
  const int64_t total = npoly * per;
  const int64_t tstep = tw.nmax / len;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t poly = t / per, b = t % per;
    const int64_t j = b % half;
    uint32_t* x = a + poly * N + (b / half) * len + j;
    const uint32_t u = x[0], v = x[half];
    x[0] = addmod(u, v, p);
    x[half] = mul_shoup(submod(u, v, p), tw.w[j * tstep], tw.ws[j * tstep], p);
  }
}

// Inverse DIT stage with span len (len > kNttBlock) in global memory.
__global__ void ntt_inv_stage_kernel(uint32_t* a, int64_t N, int64_t npoly, int64_t len, Twiddles tw, uint32_t p) {
  const int64_t half = len / 2;
  const int64_t per = N / 2;
  const int64_t total = npoly * per;
  const int64_t tstep = tw.nmax / len;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t poly = t / per, b = t % per;
    const int64_t j = b % half;
    uint32_t* x = a + poly * N + (b / half) * len + j;
    const uint32_t u = x[0];
    const uint32_t v = mul_shoup(x[half], tw.w[j * tstep], tw.ws[j * tstep], p);
    x[0] = addmod(u, v, p);
    x[half] = submod(u, v, p);
  }
}

// Forward transform of the last stages (span <= T = min(N, kNttBlock)) of each
// block of T elements in shared memory.  When src != nullptr the block is
// first loaded from src (poly q: src[(q / src_cols) * src_rs + (q % src_cols) * src_cs + t],
// t < src_len, zero padded) -- only valid when N <= kNttBlock.
__global__ void __launch_bounds__(512) ntt_fwd_smem_kernel(uint32_t* a, int64_t N, int T, const uint32_t* src,
                                                           int src_cols, int64_t src_rs, int64_t src_cs,
                                                           int64_t src_len, Twiddles tw, uint32_t p) {
  __shared__ uint32_t s[kNttBlock];
  const int64_t blocks_per_poly = N / T;
  const int64_t poly = blockIdx.x / blocks_per_poly;
  const int64_t off = (blockIdx.x % blocks_per_poly) * T;
  uint32_t* x = a + poly * N + off;
  if (src) {
    const uint32_t* sp = src + (poly / src_cols) * src_rs + (poly % src_cols) * src_cs;
    for (int t = threadIdx.x; t < T; t += blockDim.x) s[t] = (t < src_len) ? sp[t] : 0u;
  } else {
    for (int t = threadIdx.x; t < T; t += blockDim.x) s[t] = x[t];
  }
  __syncthreads();
  for (int len = T; len >= 2; len >>= 1) {
    const int half = len / 2;
    const int64_t tstep = tw.nmax / len;
    for (int b = threadIdx.x; b < T / 2; b += blockDim.x) {
      const int j = b % half;
      const int i0 = (b / half) * len + j;
      const uint32_t u = s[i0], v = s[i0 + half];
      s[i0] = addmod(u, v, p);
      s[i0 + half] = mul_shoup(submod(u, v, p), tw.w[j * tstep], tw.ws[j * tstep], p);
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < T; t += blockDim.x) x[t] = s[t];
}

// Inverse transform of the first stages (span <= T) in shared memory.  When
// dst != nullptr (only valid when N <= T) the result is scaled by N^{-1} and
// coefficients [lo, lo + cnt) are written to dst[(q / dst_cols) * dst_rs + (q % dst_cols) * dst_cs + t].
__global__ void __launch_bounds__(512) ntt_inv_smem_kernel(uint32_t* a, int64_t N, int T, uint32_t* dst, int dst_cols,
                                                           int64_t dst_rs, int64_t dst_cs, int64_t lo, int64_t cnt,
                                                           uint32_t ninv, uint32_t ninv_s, Twiddles tw, uint32_t p) {
  __shared__ uint32_t s[kNttBlock];
  const int64_t blocks_per_poly = N / T;
  const int64_t poly = blockIdx.x / blocks_per_poly;
  const int64_t off = (blockIdx.x % blocks_per_poly) * T;
  uint32_t* x = a + poly * N + off;
  for (int t = threadIdx.x; t < T; t += blockDim.x) s[t] = x[t];
  __syncthreads();
  for (int len = 2; len <= T; len <<= 1) {
    const int half = len / 2;
    const int64_t tstep = tw.nmax / len;
    for (int b = threadIdx.x; b < T / 2; b += blockDim.x) {
      const int j = b % half;
      const int i0 = (b / half) * len + j;
      const uint32_t u = s[i0];
      const uint32_t v = mul_shoup(s[i0 + half], tw.w[j * tstep], tw.ws[j * tstep], p);
      s[i0] = addmod(u, v, p);
      s[i0 + half] = submod(u, v, p);
    }
    __syncthreads();
  }
  if (dst) {
    uint32_t* dp = dst + (poly / dst_cols) * dst_rs + (poly % dst_cols) * dst_cs;
    for (int64_t t = threadIdx.x; t < cnt; t += blockDim.x) dp[t] = mul_shoup(s[lo + t], ninv, ninv_s, p);
  } else {
    for (int t = threadIdx.x; t < T; t += blockDim.x) x[t] = s[t];
  }
}

// Copy poly q of a strided source into a dense N-length slot with zero padding.
__global__ void pad_copy_kernel(uint32_t* a, int64_t N, int64_t npoly, const uint32_t* src, int src_cols, int64_t src_rs,
                                int64_t src_cs, int64_t src_len) {
  const int64_t total = npoly * N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / N, k = t % N;
    a[t] = (k < src_len) ? src[(q / src_cols) * src_rs + (q % src_cols) * src_cs + k] : 0u;
  }
}

__global__ void extract_scale_kernel(const uint32_t* a, int64_t N, int64_t npoly, uint32_t* dst, int dst_cols,
                                     int64_t dst_rs, int64_t dst_cs, int64_t lo, int64_t cnt, uint32_t ninv,
                                     uint32_t ninv_s, uint32_t p) {
  const int64_t total = npoly * cnt;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = t / cnt, k = t % cnt;
    dst[(q / dst_cols) * dst_rs + (q % dst_cols) * dst_cs + k] = mul_shoup(a[q * N + lo + k], ninv, ninv_s, p);
  }
}

// Pointwise stage: C[i][j][f] = sum_r A[i][r][f] * B[r][j][f]  (all N-length).
__global__ void pointwise_kernel(const uint32_t* __restrict__ A, const uint32_t* __restrict__ Bm, uint32_t* __restrict__ C,
                                 int m, int r, int k, int64_t N, ModP M) {
  const int64_t total = (int64_t)m * k * N;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = t % N;
    const int64_t ij = t / N;
    const int i = (int)(ij / k), j = (int)(ij % k);
    const uint32_t* a = A + (int64_t)i * r * N + f;
    const uint32_t* b = Bm + (int64_t)j * N + f;
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
                                  const uint32_t* Bm, int k, int64_t lb, int64_t b_rs, int64_t b_cs, uint32_t* dst,
                                  int64_t d_rs, int64_t d_cs, int64_t lo, int64_t cnt, ModP M) {
  const int64_t total = (int64_t)mA * k * cnt;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = lo + t % cnt;
    const int64_t ij = t / cnt;
    const int i = (int)(ij / k), j = (int)(ij % k);
    uint64_t acc = 0;
    int parity = 0;
    for (int s = 0; s < r; ++s) {
      const uint32_t* a = A + (int64_t)i * a_rs + (int64_t)s * a_cs;
      const uint32_t* b = Bm + (int64_t)s * b_rs + (int64_t)j * b_cs;
      const int64_t u0 = c - (lb - 1) > 0 ? c - (lb - 1) : 0;
      const int64_t u1 = c < la - 1 ? c : la - 1;
      for (int64_t u = u0; u <= u1; ++u) {
        acc = mad_wide(a[u], b[c - u], acc);
        if (++parity == 2) { acc = fold(acc, M); parity = 0; }
      }
    }
    dst[(int64_t)i * d_rs + (int64_t)j * d_cs + (c - lo)] = reduce(acc, M);
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
  for (int i = tid; i < m; i += nt) P.delta[i] = sdelta[i];
  __syncthreads();
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

struct Pm {
  rr_ctx* ctx = nullptr;
  cudaStream_t s = nullptr;
  int m = 0, n = 0;
  uint32_t p = 0;
  ModP M{};
  int K = 0;
  bool use_ntt = false;
  int64_t nmax = 0;
  DevBuf<uint32_t> tw, tws, twi, twis;
  DevBuf<uint32_t> FA, FB, FC;
  DevBuf<uint32_t> Mbuf;
  DevBuf<int64_t> delta;
  DevBuf<int> status;
  size_t base_smem = 0;
  // per recursion depth: MM, GG, MMM
  std::vector<std::unique_ptr<DevBuf<uint32_t>>> bufs;
  Twiddles fwd() const { return Twiddles{tw.ptr, tws.ptr, nmax}; }
  Twiddles inv() const { return Twiddles{twi.ptr, twis.ptr, nmax}; }
};

int ntt_forward(Pm& P, uint32_t* a, int64_t N, int64_t npoly, const uint32_t* src, int src_cols, int64_t src_rs,
                int64_t src_cs, int64_t src_len) {
  const int T = (int)std::min<int64_t>(N, kNttBlock);
  const int threads = std::min(512, std::max(32, T / 2));
  if (N <= kNttBlock) {
    ntt_fwd_smem_kernel<<<(unsigned)npoly, threads, 0, P.s>>>(a, N, T, src, src_cols, src_rs, src_cs, src_len, P.fwd(), P.p);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  pad_copy_kernel<<<grid_for(npoly * N), 256, 0, P.s>>>(a, N, npoly, src, src_cols, src_rs, src_cs, src_len);
  RR_CUDA(cudaGetLastError());
  for (int64_t len = N; len > kNttBlock; len >>= 1) {
    ntt_fwd_stage_kernel<<<grid_for(npoly * N / 2), 256, 0, P.s>>>(a, N, npoly, len, P.fwd(), P.p);
    RR_CUDA(cudaGetLastError());
  }
  ntt_fwd_smem_kernel<<<(unsigned)(npoly * (N / T)), threads, 0, P.s>>>(a, N, T, nullptr, 1, 0, 0, 0, P.fwd(), P.p);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

int ntt_inverse(Pm& P, uint32_t* a, int64_t N, int64_t npoly, uint32_t* dst, int dst_cols, int64_t dst_rs, int64_t dst_cs,
                int64_t lo, int64_t cnt) {
  const int T = (int)std::min<int64_t>(N, kNttBlock);
  const int threads = std::min(512, std::max(32, T / 2));
  const uint32_t ninv = host_invmod((uint32_t)(N % P.p), P.p);
  const uint32_t ninv_s = (uint32_t)(((uint64_t)ninv << 32) / P.p);
  if (N <= kNttBlock) {
    ntt_inv_smem_kernel<<<(unsigned)npoly, threads, 0, P.s>>>(a, N, T, dst, dst_cols, dst_rs, dst_cs, lo, cnt, ninv, ninv_s,
                                                             P.inv(), P.p);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  ntt_inv_smem_kernel<<<(unsigned)(npoly * (N / T)), threads, 0, P.s>>>(a, N, T, nullptr, 1, 0, 0, 0, 0, 0, 0, P.inv(), P.p);
  RR_CUDA(cudaGetLastError());
  for (int64_t len = 2 * kNttBlock; len <= N; len <<= 1) {
    ntt_inv_stage_kernel<<<grid_for(npoly * N / 2), 256, 0, P.s>>>(a, N, npoly, len, P.inv(), P.p);
    RR_CUDA(cudaGetLastError());
  }
  extract_scale_kernel<<<grid_for(npoly * cnt), 256, 0, P.s>>>(a, N, npoly, dst, dst_cols, dst_rs, dst_cs, lo, cnt, ninv,
                                                              ninv_s, P.p);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// dst[i][j][0..cnt) = coefficients [lo, lo+cnt) of A * B, where
// A is mA x r with la coefficients (strides a_rs, a_cs) and B is r x k with
// lb coefficients (strides b_rs, b_cs); dst has strides d_rs, d_cs.
int poly_mat_mul(Pm& P, const uint32_t* A, int mA, int r, int64_t la, int64_t a_rs, int64_t a_cs, const uint32_t* B,
                 int k, int64_t lb, int64_t b_rs, int64_t b_cs, uint32_t* dst, int64_t d_rs, int64_t d_cs, int64_t lo,
                 int64_t cnt) {
  int64_t N = 1;
  while (N < la + lb - 1) N <<= 1;
  if (!P.use_ntt) {
    schoolbook_kernel<<<grid_for((int64_t)mA * k * cnt), 256, 0, P.s>>>(A, mA, r, la, a_rs, a_cs, B, k, lb, b_rs, b_cs,
                                                                        dst, d_rs, d_cs, lo, cnt, P.M);
    RR_CUDA(cudaGetLastError());
    return RR_OK;
  }
  if (N > P.nmax) return fail(RR_EINVAL, "internal: NTT length %lld exceeds table %lld", (long long)N, (long long)P.nmax);
  RR_TRY(ntt_forward(P, P.FA.ptr, N, (int64_t)mA * r, A, r, a_rs, a_cs, la));
  RR_TRY(ntt_forward(P, P.FB.ptr, N, (int64_t)r * k, B, k, b_rs, b_cs, lb));
  pointwise_kernel<<<grid_for((int64_t)mA * k * N), 256, 0, P.s>>>(P.FA.ptr, P.FB.ptr, P.FC.ptr, mA, r, k, N, P.M);
  RR_CUDA(cudaGetLastError());
  return ntt_inverse(P, P.FC.ptr, N, (int64_t)mA * k, dst, k, d_rs, d_cs, lo, cnt);
}

int run_base(Pm& P, const uint32_t* G, int64_t g_rs, int64_t g_cs, int nleaves, uint32_t* Mout, int64_t o_rs,
             int64_t o_cs) {
  BaseParams B;
  B.G = G;
  B.g_rs = g_rs;
  B.g_cs = g_cs;
  B.m = P.m;
  B.n = P.n;
  B.nleaves = nleaves;
  B.delta = P.delta.ptr;
  B.Mout = Mout;
  B.out_rs = o_rs;
  B.out_cs = o_cs;
  B.Mbuf = P.Mbuf.ptr;
  B.m_smem = 1;
  B.M = P.M;
  B.status = P.status.ptr;
  if (P.n % 4 == 0) pm_base_kernel<4><<<1, kBaseThreads, P.base_smem, P.s>>>(B);
  else pm_base_kernel<1><<<1, kBaseThreads, P.base_smem, P.s>>>(B);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// Largest block of leaves (a power of two <= 32 and <= d) whose residual and
// basis fit in shared memory.
int pick_block_leaves(int m, int n, int64_t d, size_t* smem) {
  int K = (int)std::min<int64_t>(d, 32);
  while (K > 1 && base_smem_bytes(m, n, K, true) > kBaseSmemBudget) K /= 2;
  *smem = base_smem_bytes(m, n, K, true);
  return K;
}

int set_base_smem_limit(size_t bytes) {
  RR_CUDA(cudaFuncSetAttribute(pm_base_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  RR_CUDA(cudaFuncSetAttribute(pm_base_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return RR_OK;
}

// _PM_Basis (src/sigma_basis.rs:190-219) on G (m x n, strides g_rs/g_cs,
// coefficients [0, d] used); M_out receives m x m x (d+1) (strides o_rs/o_cs).
int pm_rec(Pm& P, const uint32_t* G, int64_t g_rs, int64_t g_cs, int64_t d, int depth, uint32_t* Mo, int64_t o_rs,
           int64_t o_cs) {
  if (d <= P.K) return run_base(P, G, g_rs, g_cs, (int)d, Mo, o_rs, o_cs);
  const int m = P.m, n = P.n;
  const int64_t h = d / 2;
  uint32_t* MM = P.bufs[3 * depth + 0]->ptr;   // m x m x (h+1)
  uint32_t* GG = P.bufs[3 * depth + 1]->ptr;   // m x n x (h+1)
  uint32_t* MMM = P.bufs[3 * depth + 2]->ptr;  // m x m x (h+1)
  const int64_t hl = h + 1;
  RR_TRY(pm_rec(P, G, g_rs, g_cs, h, depth + 1, MM, (int64_t)m * hl, hl));
  // GG = (MM * G)[h .. d]   (poly_mat_mul_red_adaptive(MM, G, p, 0, d+1) + shift_trunc_in(h, h))
  RR_TRY(poly_mat_mul(P, MM, m, m, hl, (int64_t)m * hl, hl, G, n, d + 1, g_rs, g_cs, GG, (int64_t)n * hl, hl, h, hl));
  RR_TRY(pm_rec(P, GG, (int64_t)n * hl, hl, h, depth + 1, MMM, (int64_t)m * hl, hl));
  // M = MMM * MM
  return poly_mat_mul(P, MMM, m, m, hl, (int64_t)m * hl, hl, MM, m, hl, (int64_t)m * hl, hl, Mo, o_rs, o_cs, 0, d + 1);
}

}  // namespace

int pm_basis_device(rr_ctx* ctx, const uint32_t* seq, int64_t seq_stride, int b, int64_t nlen, int64_t d, uint32_t p,
                    uint32_t* Mh, int64_t* deltah) {
  Pm P;
  P.ctx = ctx;
  P.s = ctx->stream;
  P.m = 2 * b;
  P.n = b;
  P.p = p;
  P.M = make_modp(p);
  P.K = pick_block_leaves(P.m, P.n, d, &P.base_smem);
  const int m = P.m, n = P.n;
  // NTT table for the largest product: length nextpow2(3d/2 + 1) = 2d (d >= 2)
  int64_t nmax = 1;
  while (nmax < d + d / 2 + 1) nmax <<= 1;
  nmax = std::max<int64_t>(nmax, 2);
  P.nmax = nmax;
  // NTT products need p - 1 divisible by the transform length; other primes
  // use the direct product (quadratic in the degree)
  P.use_ntt = d > P.K && (uint64_t)(p - 1) % (uint64_t)nmax == 0;
  if (P.use_ntt) {
    const uint32_t g = find_generator(p);
    const uint32_t w = host_powmod(g, (p - 1) / (uint64_t)nmax, p);
    const uint32_t wi = host_invmod(w, p);
    std::vector<uint32_t> t(nmax / 2), ts(nmax / 2), ti(nmax / 2), tis(nmax / 2);
    uint64_t x = 1, y = 1;
    for (int64_t j = 0; j < nmax / 2; ++j) {
      t[j] = (uint32_t)x;
      ti[j] = (uint32_t)y;
      ts[j] = (uint32_t)((x << 32) / p);
      tis[j] = (uint32_t)((y << 32) / p);
      x = x * w % p;
      y = y * wi % p;
    }
    RR_TRY(P.tw.alloc_async(nmax / 2, P.s));
    RR_TRY(P.tws.alloc_async(nmax / 2, P.s));
    RR_TRY(P.twi.alloc_async(nmax / 2, P.s));
    RR_TRY(P.twis.alloc_async(nmax / 2, P.s));
    RR_CUDA(cudaMemcpyAsync(P.tw.ptr, t.data(), t.size() * 4, cudaMemcpyHostToDevice, P.s));
    RR_CUDA(cudaMemcpyAsync(P.tws.ptr, ts.data(), ts.size() * 4, cudaMemcpyHostToDevice, P.s));
    RR_CUDA(cudaMemcpyAsync(P.twi.ptr, ti.data(), ti.size() * 4, cudaMemcpyHostToDevice, P.s));
    RR_CUDA(cudaMemcpyAsync(P.twis.ptr, tis.data(), tis.size() * 4, cudaMemcpyHostToDevice, P.s));
    RR_TRY(P.FA.alloc_async((size_t)m * m * nmax, P.s));
    RR_TRY(P.FB.alloc_async((size_t)m * m * nmax, P.s));
    RR_TRY(P.FC.alloc_async((size_t)m * m * nmax, P.s));
    RR_CUDA(cudaStreamSynchronize(P.s));
  }
  // per-depth buffers
  {
    int depth = 0;
    for (int64_t dd = d; dd > P.K; dd /= 2, ++depth) {
      const int64_t hl = dd / 2 + 1;
      for (int q = 0; q < 3; ++q) {
        P.bufs.emplace_back(new DevBuf<uint32_t>());
        RR_TRY(P.bufs.back()->alloc_async((size_t)m * (q == 1 ? n : m) * hl, P.s));
      }
    }
  }
  RR_TRY(P.delta.alloc_async(m, P.s));
  RR_TRY(P.status.alloc_async(1, P.s));
  RR_CUDA(cudaMemsetAsync(P.delta.ptr, 0, m * sizeof(int64_t), P.s));
  RR_CUDA(cudaMemsetAsync(P.status.ptr, 0, sizeof(int), P.s));
  RR_TRY(set_base_smem_limit(P.base_smem));
  // G = [S; I], coefficients [0, d]
  DevBuf<uint32_t> dseq, G;
  const int np = b * (b + 1) / 2;
  const int64_t glen = d + 1;
  RR_TRY(dseq.alloc_async((size_t)np * glen, P.s));
  RR_CUDA(cudaMemcpy2DAsync(dseq.ptr, glen * 4, seq, seq_stride * 4, glen * 4, np, cudaMemcpyHostToDevice, P.s));
  RR_TRY(G.alloc_async((size_t)m * n * glen, P.s));
  build_G_kernel<<<grid_for((int64_t)m * n * glen), 256, 0, P.s>>>(dseq.ptr, glen, b, glen, G.ptr, p);
  RR_CUDA(cudaGetLastError());
  DevBuf<uint32_t> Mo;
  RR_TRY(Mo.alloc_async((size_t)m * m * (d + 1), P.s));
  RR_TRY(pm_rec(P, G.ptr, (int64_t)n * glen, glen, d, 0, Mo.ptr, (int64_t)m * (d + 1), d + 1));
  int status = 0;
  RR_CUDA(cudaMemcpyAsync(Mh, Mo.ptr, Mo.bytes(), cudaMemcpyDeviceToHost, P.s));
  RR_CUDA(cudaMemcpyAsync(deltah, P.delta.ptr, m * sizeof(int64_t), cudaMemcpyDeviceToHost, P.s));
  RR_CUDA(cudaMemcpyAsync(&status, P.status.ptr, sizeof(int), cudaMemcpyDeviceToHost, P.s));
  RR_CUDA(cudaStreamSynchronize(P.s));
  if (status) return fail(RR_ECUDA, "PM-basis device status %d (zero row scale)", status);
  return RR_OK;
}

// ---------------------------------------------------------------- no-allocation variant
// rr_pm_basis_short_noalloc runs the same two kernels as rr_pm_basis does for a
// short sequence (build_G_kernel, then one pm_base_kernel block), but takes its
// scratch -- the matrix G, the base kernel's double-buffered basis and the
// status word -- from the file-scope array below instead of allocating it.
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
// per device (host code must not use the symbol itself as an address).
static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  RR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(RR_EUNSUPPORTED, "device %d beyond %d", dev, kNoallocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    RR_CUDA(cudaGetSymbolAddress(&p, g_pm_noalloc_scratch));
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
  const size_t bytes = base_smem_bytes(m, n, (int)dd, false);
  RR_TRY(set_base_smem_limit(bytes));
  if (n % 4 == 0) pm_base_kernel<4><<<1, kBaseThreads, bytes, s>>>(B);
  else pm_base_kernel<1><<<1, kBaseThreads, bytes, s>>>(B);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}
