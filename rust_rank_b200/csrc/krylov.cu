// krylov.cu -- the fused Krylov step of the block-Wiedemann engine.
//
// One application of B = D_c A^T D_r A D_c (src/main.rs:522-526) to the block
// w_k (b vectors) produces the two sequence terms of src/main.rs:138-156:
//
//   S_{2k+1} = w_k^T B w_k = z^T D_r z,   z = A x,   x = D_c w_k
//   S_{2k+2} = w_{k+1}^T w_{k+1},         w_{k+1} = D_c A^T (D_r z)
//
// (both equal the reference's dot products mod p exactly).  The state kept on
// the device is x_k = D_c w_k, so A is used with its raw entries and the
// diagonal preconditioners are applied in the epilogues:
//
//   pass 1 (rows of A):   z = A x;  U = D_r z;  Gram_odd  += z (x) U
//   pass 2 (rows of A^T): t = A^T U; w' = D_c t; x' = D_c w';  Gram_even += w' (x) w'
//
// The block is stored interleaved, X[row][B] uint32 (B = 4..32 lanes); a
// thread owns 8 lanes (4 when B = 4) and gathers them with 128-bit loads, so a
// row of the block is one 16..128-byte segment.  CSR entries are packed
// (column, value) pairs read with one 64-bit load.  Each thread issues the
// loads of four entries before it multiplies, so eight (or four) gathers are in
// flight per thread.  Sums are accumulated lazily in 64 bits with a fold every
// 2 or 4 products and finished with a Montgomery reduction; the factor R^{-1}
// it leaves is absorbed into the preconditioner scales (d R^2 mod p, d R mod p)
// and, for the odd term, into one final multiplication by R.
//
// The Gram terms are reduced per CTA in shared memory, then across CTAs with
// 64-bit atomics; the last CTA to finish writes the finished term and resets
// the accumulators, so no separate reduction kernel and no host round trip is
// needed.
//
// Rows are renumbered by decreasing degree.  Rows longer than kHeavyDegree are
// cut into chunks of at most kChunkNnz entries that are processed
// warp-per-chunk and merged with 64-bit atomics; the pass kernel then applies
// the epilogue to them like to any other row.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <type_traits>

#include "krylov_params.h"

namespace rr {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
static_assert(kWarps == kPassWarps, "host-side run tables assume this many warps per CTA");

// Threads of a warp split into RPW row slots of TPR threads; a thread owns
// LPT lanes of its row's block, as NV 128-bit words interleaved with the other
// threads of the slot: word v of thread `sub` is word v * TPR + sub of the row
// (lanes 4 (v TPR + sub) .. + 3).  So one warp load instruction reads TPR
// adjacent 16-byte words per row -- whole 32-byte sectors for B >= 8 -- and a
// gathered row costs the L1 the minimum of B / 8 sector accesses.
template <int B>
constexpr int kDefaultLpt = (B >= 16) ? 8 : 4;

template <int B, int L = kDefaultLpt<B>>
struct Shape {
  static constexpr int LPT = L;                   // lanes of the block per thread
  static constexpr int NV = LPT / 4;              // 128-bit words per thread per row
  static constexpr int TPR = B / LPT;             // threads per row
  static constexpr int RPW = 32 / TPR;            // rows per warp batch (slots)
  // block lane of this thread's lane l
  static __device__ __forceinline__ int lane_of(int sub, int l) { return 4 * ((l >> 2) * TPR + sub) + (l & 3); }
  // 128-bit word index within a row of this thread's word v
  static __device__ __forceinline__ int word_of(int sub, int v) { return v * TPR + sub; }
};

__device__ __forceinline__ void pair_of(int q, int B, int& i, int& j) {
  // q enumerates (i <= j) row-major: offset(i) = i*B - i*(i-1)/2
  i = 0;
  int off = 0;
  while (q >= off + (B - i)) {
    off += B - i;
    ++i;
  }
  j = i + (q - off);
}

// acc[l] += sum over entries k = beg, beg+stride, ... < end of val * X[col][lane l]
// for this thread's LPT lanes (lane block `sub`).  Four entries per step, all
// loads issued before the multiplies; acc is folded after every FE products,
// so it leaves folded (< p * 2^32).
template <int B, int FE, int L = kDefaultLpt<B>>
__device__ __forceinline__ void mac_step(const uint2 (&e)[4], const uint4 (&g)[4][Shape<B, L>::NV], const ModP& M,
                                         uint64_t (&acc)[Shape<B, L>::LPT]) {
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const uint32_t val = e[u].y;
#pragma unroll
    for (int v = 0; v < Shape<B, L>::NV; ++v) {
      acc[4 * v + 0] = mad_wide(val, g[u][v].x, acc[4 * v + 0]);
      acc[4 * v + 1] = mad_wide(val, g[u][v].y, acc[4 * v + 1]);
      acc[4 * v + 2] = mad_wide(val, g[u][v].z, acc[4 * v + 2]);
      acc[4 * v + 3] = mad_wide(val, g[u][v].w, acc[4 * v + 3]);
    }
    if ((u % FE) == FE - 1) {
#pragma unroll
      for (int l = 0; l < Shape<B, L>::LPT; ++l) acc[l] = fold(acc[l], M);
    }
  }
}

// Full steps of four entries run without predicates, with the entries of the
// next step loaded while the current step's gathers are in flight; the last,
// partial step clamps its index into the row and multiplies by zero instead
// of branching (the clamped gather re-reads a row already in cache).
// Gathers of the block: through the read-only path, or (COH, inside the
// persistent batched kernel, where the block is rewritten between grid
// barriers) from L2 with ordinary coherent loads.
template <bool COH>
__device__ __forceinline__ uint4 ld_block(const uint4* p) {
  if (COH) return __ldcg(p);
  return __ldg(p);
}

template <int B, int FE, bool COH = false, int L = kDefaultLpt<B>>
__device__ __forceinline__ void gather_sum(const uint2* __restrict__ cv, uint32_t beg, uint32_t end, uint32_t stride,
                                           const uint4* __restrict__ X, int sub, const ModP& M,
                                           uint64_t (&acc)[Shape<B, L>::LPT]) {
  constexpr int NV = Shape<B, L>::NV;
  constexpr int RW = B / 4;  // 128-bit words per block row
  const uint4* Xs = X + sub;  // word v of the row at Xs + v * TPR
  uint32_t k = beg;
  const uint32_t step = 4 * stride;
  if (k + 3 * stride < end) {
    uint2 e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = __ldg(cv + k + u * stride);
    for (;;) {
      uint4 g[4][NV];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < NV; ++v) g[u][v] = ld_block<COH>(Xs + (size_t)e[u].x * RW + v * Shape<B, L>::TPR);
      k += step;
      const bool more = k + 3 * stride < end;
      uint2 en[4];
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u) en[u] = __ldg(cv + k + u * stride);
      }
      mac_step<B, FE, L>(e, g, M, acc);
      if (!more) break;
#pragma unroll
      for (int u = 0; u < 4; ++u) e[u] = en[u];
    }
  }
  if (k < end) {
    uint2 e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t kk = k + u * stride;
      e[u] = __ldg(cv + (kk < end ? kk : k));
      if (kk >= end) e[u].y = 0u;
    }
    uint4 g[4][NV];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < NV; ++v) g[u][v] = ld_block<COH>(Xs + (size_t)e[u].x * RW + v * Shape<B, L>::TPR);
    mac_step<B, FE, L>(e, g, M, acc);
  }
}

// The same sum with eight entries per step (two groups of four in flight per
// thread): with 4 lanes per thread a whole 64- or 128-byte block row is one
// warp load instruction (one L1 wavefront per gathered row instead of two),
// and the eight loads keep as many bytes in flight as four steps of 8 lanes.
template <int B, int FE, int L>
__device__ __forceinline__ void gather_sum8(const uint2* __restrict__ cv, uint32_t beg, uint32_t end, uint32_t stride,
                                            const uint4* __restrict__ X, int sub, const ModP& M,
                                            uint64_t (&acc)[Shape<B, L>::LPT]) {
  constexpr int NV = Shape<B, L>::NV, TPR = Shape<B, L>::TPR;
  constexpr int RW = B / 4;
  const uint4* Xs = X + sub;
  uint32_t k = beg;
  if (k + 7 * stride < end) {
    uint2 e0[4], e1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      e0[u] = __ldg(cv + k + u * stride);
      e1[u] = __ldg(cv + k + (u + 4) * stride);
    }
    for (;;) {
      uint4 g0[4][NV], g1[4][NV];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          g0[u][v] = __ldg(Xs + (size_t)e0[u].x * RW + v * TPR);
          g1[u][v] = __ldg(Xs + (size_t)e1[u].x * RW + v * TPR);
        }
      k += 8 * stride;
      const bool more = k + 7 * stride < end;
      uint2 n0[4], n1[4];
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          n0[u] = __ldg(cv + k + u * stride);
          n1[u] = __ldg(cv + k + (u + 4) * stride);
        }
      }
      mac_step<B, FE, L>(e0, g0, M, acc);
      mac_step<B, FE, L>(e1, g1, M, acc);
      if (!more) break;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        e0[u] = n0[u];
        e1[u] = n1[u];
      }
    }
  }
  while (k < end) {  // at most two steps of four, the last one clamped
    uint2 e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t kk = k + u * stride;
      e[u] = __ldg(cv + (kk < end ? kk : k));
      if (kk >= end) e[u].y = 0u;
    }
    uint4 g[4][NV];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < NV; ++v) g[u][v] = __ldg(Xs + (size_t)e[u].x * RW + v * TPR);
    mac_step<B, FE, L>(e, g, M, acc);
    k += 4 * stride;
  }
}

__device__ __forceinline__ int pair_index(int i, int j, int B) { return i * B - i * (i - 1) / 2 + (j - i); }

// Programmatic dependent launch: the single-matrix kernels are launched so
// that the next kernel of an application may be scheduled while the previous
// one finishes.  griddep_wait() blocks until the previous kernel has completed
// and its writes are visible (it returns at once for a normal launch), so every
// such kernel calls it before reading what its predecessor wrote;
// griddep_launch() tells the scheduler a CTA has no more main-loop work.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ---------------------------------------------------------------- Gram terms
// Both accumulators sum G[i][j] = sum over rows of gz[i] * gu[j] (i <= j) for
// the rows a warp processes, then add their residues into the CTA's red[].

// CUDA cores (B = 4): the batch is staged in shared memory and every lane
// accumulates a few (i, j) pairs over the staged rows.
template <int B, int FE, int L = kDefaultLpt<B>>
struct GramCore {
  static constexpr int LPT = Shape<B, L>::LPT, RPW = Shape<B, L>::RPW;
  static constexpr int NP = B * (B + 1) / 2, PPL = (NP + 31) / 32;
  static constexpr int kWords = 2 * RPW * B;  // shared words per warp
  uint32_t* zs;  // [RPW][B]
  uint32_t* us;
  uint32_t pij[PPL];
  unsigned long long acc[PPL];

  __device__ __forceinline__ void init(uint32_t* w, int lane) {
    zs = w;
    us = w + RPW * B;
#pragma unroll
    for (int t = 0; t < PPL; ++t) {
      const int q = lane + 32 * t;
      int i = 0, j = 0;
      if (q < NP) pair_of(q, B, i, j);
      pij[t] = ((uint32_t)i << 8) | (uint32_t)j;
      acc[t] = 0;
    }
  }
  __device__ __forceinline__ void add(const uint32_t (&gz)[LPT], const uint32_t (&gu)[LPT], int slot, int sub,
                                      int lane, const ModP& M, const uint32_t (&)[3]) {
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      zs[slot * B + Shape<B, L>::lane_of(sub, l)] = gz[l];
      us[slot * B + Shape<B, L>::lane_of(sub, l)] = gu[l];
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < PPL; ++t) {
      if (lane + 32 * t < NP) {
        const int i = pij[t] >> 8, j = pij[t] & 0xff;
        unsigned long long a = acc[t];
#pragma unroll
        for (int rr = 0; rr < RPW; ++rr) {
          a = mad_wide(zs[rr * B + i], us[rr * B + j], a);
          if ((rr % FE) == FE - 1) a = fold(a, M);
        }
        acc[t] = a;
      }
    }
    __syncwarp();
  }
  __device__ __forceinline__ void finish(int, int, int, const ModP&, const uint32_t (&)[3]) {}
  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int t = 0; t < PPL; ++t) acc[t] = 0;
  }
  __device__ __forceinline__ void emit(unsigned long long* red, int lane, const ModP& M) {
#pragma unroll
    for (int t = 0; t < PPL; ++t) {
      const int q = lane + 32 * t;
      if (q < NP) atomicAdd(&red[q], (unsigned long long)reduce(acc[t], M));
    }
  }
};

// D += A * B with A 16x32 u8 (row-major fragments), B 32x8 u8, D 16x8 s32.
__device__ __forceinline__ void mma_u8(int (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Tensor cores (B >= 8): exact integer Gram by byte limbs.  Residues are
// < 2^31, so z = sum_a z_a 256^a with bytes z_a, and
//   Z^T U = sum_{a,c} 256^{a+c} Z_a^T U_c.
// A warp stages 32 rows (one K tile) as byte planes P[limb][lane][row] in
// shared memory -- each row's four limbs are spread over four rows' words with
// a 4x4 byte transpose across lanes (two shuffles and two byte permutes) --
// then issues 16 m16n8k32 u8 MMAs per 16x8 output tile.  Per K tile a limb
// pair's product is < 32 * 255^2 < 2^21, so the shift classes s = a + c stay
// exact in int32; classes 0..3 are recombined exactly in 64 bits (< 2^48) and
// classes 4..6 are added with their weights 2^{8s} mod p.
template <int B, int FE, int L = kDefaultLpt<B>>
struct GramMma {
  static constexpr int LPT = Shape<B, L>::LPT, TPR = Shape<B, L>::TPR, RPW = Shape<B, L>::RPW;
  static constexpr int TB = 32 / RPW;           // batches per K tile
  static constexpr int BM = B < 16 ? 16 : B;    // rows of the M dimension (zero padded)
  static constexpr int MT = BM / 16, NT = B / 8;
  static constexpr int RS = 9;                  // words per (limb, lane) plane row: 32 bytes + 4 pad
  static constexpr int kPlane = 4 * BM * RS;    // words per plane set
  static constexpr int kWords = 2 * kPlane;     // shared words per warp
  uint32_t* pz;
  uint32_t* pu;
  unsigned long long acc[MT][NT][4];
  int bt;

  __device__ __forceinline__ void init(uint32_t* w, int lane) {
    pz = w;
    pu = w + kPlane;
    for (int q = lane; q < kWords; q += 32) w[q] = 0;  // zero padding rows stay zero
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[mt][nt][v] = 0;
    bt = 0;
    __syncwarp();
  }

  // 4x4 byte transpose among the lanes holding rows 4q..4q+3 (lane distance
  // TPR): afterwards byte k of the word of the lane with row 4q+rho is limb
  // rho of the value of row 4q+k.
  __device__ __forceinline__ static uint32_t transpose4(uint32_t w, int rho) {
    uint32_t p = __shfl_xor_sync(0xffffffffu, w, TPR);
    w = (rho & 1) ? __byte_perm(p, w, 0x7351) : __byte_perm(w, p, 0x6240);
    p = __shfl_xor_sync(0xffffffffu, w, 2 * TPR);
    return (rho & 2) ? __byte_perm(p, w, 0x7632) : __byte_perm(w, p, 0x5410);
  }

  __device__ __forceinline__ void stage(const uint32_t (&gz)[LPT], const uint32_t (&gu)[LPT], int slot, int sub) {
    const int rho = slot & 3;
    const int word = (bt * RPW + (slot & ~3)) >> 2;  // 4-row group inside the K tile
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int i = Shape<B, L>::lane_of(sub, l);
      pz[(rho * BM + i) * RS + word] = transpose4(gz[l], rho);
      pu[(rho * BM + i) * RS + word] = transpose4(gu[l], rho);
    }
  }

  __device__ __forceinline__ void flush(int lane, const ModP& M, const uint32_t (&W)[3]) {
    __syncwarp();
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      uint32_t A[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const uint32_t* r0 = pz + (a * BM + mt * 16 + g) * RS;
        const uint32_t* r1 = r0 + 8 * RS;
        A[a][0] = r0[t];
        A[a][1] = r1[t];
        A[a][2] = r0[t + 4];
        A[a][3] = r1[t + 4];
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        if (mt * 16 > nt * 8 + 7) continue;  // tile entirely below the diagonal
        uint32_t Bf[4][2];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t* r = pu + (c * BM + nt * 8 + g) * RS;
          Bf[c][0] = r[t];
          Bf[c][1] = r[t + 4];
        }
        uint64_t lo[4] = {0, 0, 0, 0};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          int C[4] = {0, 0, 0, 0};
#pragma unroll
          for (int a = 0; a <= s; ++a) mma_u8(C, A[a], Bf[s - a][0], Bf[s - a][1]);
#pragma unroll
          for (int v = 0; v < 4; ++v) lo[v] += (uint64_t)(uint32_t)C[v] << (8 * s);
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[mt][nt][v] = fold(acc[mt][nt][v] + lo[v], M);
#pragma unroll
        for (int s = 4; s < 7; ++s) {
          int C[4] = {0, 0, 0, 0};
#pragma unroll
          for (int a = s - 3; a < 4; ++a) mma_u8(C, A[a], Bf[s - a][0], Bf[s - a][1]);
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[mt][nt][v] = mad_wide((uint32_t)C[v], W[s - 4], acc[mt][nt][v]);
        }
      }
    }
    __syncwarp();
  }

  __device__ __forceinline__ void add(const uint32_t (&gz)[LPT], const uint32_t (&gu)[LPT], int slot, int sub,
                                      int lane, const ModP& M, const uint32_t (&W)[3]) {
    stage(gz, gu, slot, sub);
    if (++bt == TB) {
      flush(lane, M, W);
      bt = 0;
    }
  }

  __device__ __forceinline__ void reset() {
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[mt][nt][v] = 0;
    bt = 0;
  }

  __device__ __forceinline__ void finish(int slot, int sub, int lane, const ModP& M, const uint32_t (&W)[3]) {
    if (bt == 0) return;
    uint32_t z[LPT];
#pragma unroll
    for (int l = 0; l < LPT; ++l) z[l] = 0;
    while (bt < TB) {  // zero the rows of the batches the tile did not get
      stage(z, z, slot, sub);
      ++bt;
    }
    flush(lane, M, W);
    bt = 0;
  }

  __device__ __forceinline__ void emit(unsigned long long* red, int lane, const ModP& M) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int i = mt * 16 + g + (v >= 2 ? 8 : 0);
          const int j = nt * 8 + 2 * t + (v & 1);
          if (i <= j && j < B) atomicAdd(&red[pair_index(i, j, B)], (unsigned long long)reduce(acc[mt][nt][v], M));
        }
  }
};

// Batched mode: where the Gram partials of segment sg go (its own slot for
// this launch's term, or the segment's shared accumulator); NP = padded pairs.
__device__ __forceinline__ unsigned long long* seg_target(const PassParams& P, unsigned long long* acc, int sg, int NP) {
  if (P.gram_all != nullptr) return P.gram_all + P.seg_G_off[sg] + P.term * (int64_t)NP;
  return acc + (size_t)sg * NP;
}

// One pass over the rows of A (MODE odd), of A^T (even) or the initial
// scaling (init), by the whole CTA: gram_smem is the per-warp Gram staging,
// red[NP] the CTA's Gram reduction, is_last a shared flag.
template <int B, int MODE, int FE, bool COH, bool GRAM = true, int L = kDefaultLpt<B>>
__device__ __forceinline__ void pass_body(const PassParams& P, uint32_t* gram_smem, unsigned long long* red,
                                          bool& is_last) {
  using S = Shape<B, L>;
  constexpr int LPT = S::LPT, NV = S::NV, TPR = S::TPR, RPW = S::RPW;
  constexpr int NP = B * (B + 1) / 2;  // pairs in padded space
  constexpr bool kMma = B >= 8;
  using Gram = typename std::conditional<kMma, GramMma<B, FE, L>, GramCore<B, FE, L>>::type;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane % TPR;
  const int slot = lane / TPR;
  const ModP M = P.M;
  const uint32_t W[3] = {P.w4, P.w5, P.w6};

  for (int q = threadIdx.x; q < NP; q += kThreads) red[q] = 0;
  Gram gram;
  const bool emit = GRAM && (P.S_out != nullptr || P.term_ctr != nullptr);
  if (emit) gram.init(gram_smem + (size_t)warp * Gram::kWords, lane);
  __syncthreads();  // red[] zeroed before a warp may emit into it

  const int64_t nbatch = (P.rows + RPW - 1) / RPW;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  const bool segmented = P.batch_seg != nullptr;
  // one matrix: grid-stride over the degree-sorted batches; batched: contiguous
  // runs, so that a warp changes matrix (and flushes its Gram terms) rarely
  int64_t b_first = gw, b_stop = nbatch, b_step = nw;
  if (segmented) {
    if (P.runs != nullptr) {  // runs of equal work (nonzeros + rows), built on the host
      b_first = P.runs[gw];
      b_stop = P.runs[gw + 1];
    } else {
      const int64_t total = nbatch - P.batch_begin;
      const int64_t q = (total + nw - 1) / nw;
      b_first = P.batch_begin + gw * q;
      b_stop = b_first + q < nbatch ? b_first + q : nbatch;
    }
    b_step = 1;
  }
  int cur_seg = -1;
  // batched: the CTA's first matrix is reduced in shared memory (red), any
  // other matrix a warp meets goes straight to the accumulators
  int seg0 = -1;
  unsigned long long* const acc = P.gram_acc + (size_t)(blockIdx.x % P.replicas) * P.gram_stride;
  if (segmented) {
    const int64_t lo = P.runs != nullptr ? (int64_t)P.runs[(int64_t)blockIdx.x * kWarps]
                                         : P.batch_begin + (int64_t)blockIdx.x * kWarps *
                                                               ((nbatch - P.batch_begin + nw - 1) / nw);
    if (lo < nbatch) seg0 = P.batch_seg[lo];
  }

  for (int64_t batch = b_first; batch < b_stop; batch += b_step) {
    if (segmented && emit) {
      const int sg = P.batch_seg[batch];
      if (sg != cur_seg) {
        if (cur_seg >= 0) {
          gram.finish(slot, sub, lane, M, W);
          gram.emit(cur_seg == seg0 ? red : seg_target(P, acc, cur_seg, NP), lane, M);
          gram.reset();
        }
        cur_seg = sg;
      }
    }
    const int64_t r = batch * RPW + slot;
    if (P.tail_begin > 0 && batch * RPW >= P.tail_begin) {
      // a batch of rows without entries: zero output, nothing to the Gram term
      if (r < P.rows) {
#pragma unroll
        for (int v = 0; v < NV; ++v) P.Y[r * (B / 4) + S::word_of(sub, v)] = make_uint4(0, 0, 0, 0);
      }
      continue;
    }
    uint32_t gz[LPT], gu[LPT];
    if (r < P.rows) {
      uint32_t t[LPT];
      if (MODE == kModeInit) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const uint4 w = ld_block<COH>(P.X + r * (B / 4) + S::word_of(sub, v));
          t[4 * v + 0] = w.x; t[4 * v + 1] = w.y; t[4 * v + 2] = w.z; t[4 * v + 3] = w.w;
        }
      } else {
        uint64_t acc[LPT];
#pragma unroll
        for (int l = 0; l < LPT; ++l) acc[l] = 0;
        if (r < P.heavy_rows) {
          unsigned long long* h = P.heavy_acc + (size_t)r * B;
#pragma unroll
          for (int l = 0; l < LPT; ++l) {
            acc[l] = fold(h[S::lane_of(sub, l)], M);
            h[S::lane_of(sub, l)] = 0;
          }
        } else {
          gather_sum<B, FE, COH, L>(P.cv, P.rowptr[r], P.rowptr[r + 1], 1u, P.X, sub, M, acc);
        }
#pragma unroll
        for (int l = 0; l < LPT; ++l) t[l] = redc(acc[l], M);  // t = (row sum) R^{-1}
      }
      const uint32_t s1 = P.scale[r];
      uint32_t o[LPT];
      if (MODE == kModeOdd) {
        // z R^{-1} = t; U = d_r z = redc(t * d_r R^2)
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
          gz[l] = t[l];
          gu[l] = redc((uint64_t)t[l] * s1, M);
          o[l] = gu[l];
        }
      } else if (MODE == kModeEven) {
        // w' = d_c t_true = redc(t * d_c R^2); x' = d_c w' = redc(w' * d_c R)
        const uint32_t s2 = P.scale2[r];
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
          gz[l] = redc((uint64_t)t[l] * s1, M);
          gu[l] = gz[l];
          o[l] = redc((uint64_t)gz[l] * s2, M);
        }
      } else {
        // init: w given; x = d_c w = redc(w * d_c R)
#pragma unroll
        for (int l = 0; l < LPT; ++l) {
          gz[l] = t[l];
          gu[l] = t[l];
          o[l] = redc((uint64_t)t[l] * s1, M);
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v)
        P.Y[r * (B / 4) + S::word_of(sub, v)] = make_uint4(o[4 * v], o[4 * v + 1], o[4 * v + 2], o[4 * v + 3]);
    } else {
#pragma unroll
      for (int l = 0; l < LPT; ++l) { gz[l] = 0; gu[l] = 0; }
    }
    if (emit) gram.add(gz, gu, slot, sub, lane, M, W);
  }
  if (!segmented) griddep_launch();

  if (!emit) return;
  gram.finish(slot, sub, lane, M, W);
  __syncthreads();  // red[] is zeroed before any warp emits into it
  if (segmented) {
    if (cur_seg >= 0) gram.emit(cur_seg == seg0 ? red : seg_target(P, acc, cur_seg, NP), lane, M);
    __syncthreads();
    if (seg0 >= 0) {
      unsigned long long* t0 = seg_target(P, acc, seg0, NP);
      for (int q = threadIdx.x; q < NP; q += kThreads) atomicAdd(&t0[q], red[q]);
    }
    if (P.gram_all != nullptr) return;  // finished later, once per group
  } else {
    gram.emit(red, lane, M);
    __syncthreads();
    for (int q = threadIdx.x; q < NP; q += kThreads) atomicAdd(&acc[q], red[q]);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = (atomicAdd(P.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // the last CTA: write the finished terms (real pairs only) and reset
  const int b = P.b_real;
  const int npr = b * (b + 1) / 2;
  if (segmented) {
    // every other CTA's atomics are visible (fence + counter), so plain L2
    // loads suffice; four in flight per thread
    const int nseg = P.seg_end - P.seg_begin;
    const int64_t total = (int64_t)nseg * npr;
    for (int64_t e0 = threadIdx.x; e0 < total; e0 += 4 * kThreads) {
      unsigned long long v[4];
      unsigned long long* g[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t e = e0 + (int64_t)u * kThreads;
        g[u] = nullptr;
        if (e < total) {
          const int s = P.seg_begin + (int)(e / npr), q = (int)(e % npr);
          int i, j;
          pair_of(q, b, i, j);
          g[u] = P.gram_acc + (size_t)s * NP + pair_index(i, j, B);
          v[u] = 0;
          for (int r = 0; r < P.replicas; ++r) v[u] += __ldcg(g[u] + (size_t)r * P.gram_stride);
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int64_t e = e0 + (int64_t)u * kThreads;
        if (g[u] != nullptr) {
          const int s = P.seg_begin + (int)(e / npr), q = (int)(e % npr);
          P.S_all[P.seg_S_off[s] + P.term * npr + q] = mulmod(reduce(v[u], M), P.gram_mul, M);
          for (int r = 0; r < P.replicas; ++r) __stcg(g[u] + (size_t)r * P.gram_stride, 0ull);
        }
      }
    }
  } else {
    uint32_t* S_out = P.S_out;
    if (P.term_ctr != nullptr) S_out = *P.S_ptr + (size_t)__ldcg(P.term_ctr) * npr;
    for (int q = threadIdx.x; q < npr; q += kThreads) {
      int i, j;
      pair_of(q, b, i, j);
      const int qb = pair_index(i, j, B);
      unsigned long long v = 0;
      for (int r = 0; r < P.replicas; ++r) v += __ldcg(P.gram_acc + (size_t)r * P.gram_stride + qb);
      S_out[q] = mulmod(reduce(v, M), P.gram_mul, M);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NP * P.replicas; q += kThreads)
      __stcg(P.gram_acc + (size_t)(q / NP) * P.gram_stride + q % NP, 0ull);
    if (P.term_ctr != nullptr && threadIdx.x == 0) *P.term_ctr += 1u;  // read above by thread 0 only after the barrier
  }
  if (threadIdx.x == 0) atomicExch(P.counter, 0u);
}

// Four CTAs (32 warps) per SM: the walk is latency bound, so occupancy is
// worth a few spilled registers (measured on the 2M x 1.5M Zipf matrix).  At
// B = 32 the Gram accumulators alone take 48 registers, and two CTAs per SM
// with 128 registers run the same matrix 1.2x faster than four with spills.
//
// Resident CTAs per SM the register budget is set for: 5 for the lean pass at
// width 16 (48 registers; one more CTA of latency hiding measured 1.3 % faster
// than 4 with 62 registers), 2 for fused passes at width 32, else 4.
template <int B, bool GRAM>
constexpr int kPassMinBlocks = (B >= 32 && GRAM) ? 2 : ((!GRAM && B == 16) ? 5 : 4);

template <int B, int MODE, int FE, bool GRAM = true, int L = kDefaultLpt<B>>
__global__ void __launch_bounds__(kThreads, kPassMinBlocks<B, GRAM>) pass_kernel(PassParams P) {
  extern __shared__ __align__(16) uint32_t gram_smem[];
  __shared__ unsigned long long red[B * (B + 1) / 2];
  __shared__ bool is_last;
  griddep_wait();
  pass_body<B, MODE, FE, false, GRAM, L>(P, gram_smem, red, is_last);
}

// Lanes per thread of the single-matrix odd and even passes: 4 (a whole
// 16-lane row in one warp load instruction, one L1 line look-up per gathered
// row) at padded width 16, the pass kernels' default otherwise.
template <int B>
constexpr int kLeanLpt = (B == 16) ? 4 : kDefaultLpt<B>;

// Which single-matrix passes compute their Gram terms themselves (u8-limb
// mma.sync on the block rows still in registers) and which run without them,
// followed by a tcgen05 Gram pass (gram_tc_kernel) that reads the written
// block once more.  Measured per pass on the 2M x 1.5M Zipf matrix: at width
// 16 the odd pass is faster split (0.251 ms against 0.269 fused), the even
// pass fused (0.146 against 0.173); at width 32 both are faster split (0.93
// ms per application against 1.29 fused).
template <int B>
constexpr bool kFusedOdd = (B <= 8);
template <int B>
constexpr bool kFusedEven = (B <= 16);

// ---------------------------------------------------------------- Gram pass on tcgen05
// The Gram term of a block (kModeGram: gz = x * scale, gu = gram_sym ? gz : x
// per row) on the 5th-generation tensor cores, for padded widths 16 and 32.
//
// Exact integers by byte limbs: with gz = sum_a 256^a Z_a and gu = sum_c 256^c
// U_c (bytes), G[i][j] = sum_{a,c} 256^{a+c} (Z_a^T U_c)[i][j].  One UMMA
// D[M x N] += A[M x K] B[N x K]^T (kind::i8, unsigned bytes, s32 accumulators
// in TMEM) computes all 16 limb pairs at once: A row (a, i) holds limb a of
// lane i of the tile's rows (K = rows), B row (c, j) limb c of gu; M = 128
// (4 B rows, zero-padded to 128 for B = 16), N = 4 B.  A CTA stages 128-row
// tiles into shared memory in the canonical K-major layout without swizzle
// (8-row x 16-byte core matrices; K-adjacent cores 128 bytes apart, 8-row
// groups 256 bytes apart); one thread issues the four K = 32 MMAs of a tile.
// A per-row limb product is < 2^16, so the int32 accumulators are read out
// every kTcDrain tiles (tcgen05.ld), limb pairs weighted by 2^{8(a+c)} mod p,
// and the CTA's sums join the same replicated 64-bit accumulators and
// last-CTA finish as the pass kernels.  Every wait on an mbarrier gives up
// after 2 s and sets *status.
constexpr int kTcDrain = 64;        // tiles between drains of the int32 accumulators
constexpr uint64_t kTcWaitLimitNs = 2000000000ull;  // 2 s of %globaltimer

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no swizzle: start >> 4, LBO = 128 B (K-direction core stride),
// SBO = 256 B (8-row group stride), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) |
         (1ull << 46);
}

// Operand rows within a limb: lane i = 4 g + c (g its 128-bit word, c the
// word's component) sits in row c * B/4 + g, so that the 32 stores of one
// warp instruction (8 words g x 4 row quads, fixed c) fall in 32 different
// banks at B = 32.  tc_lane maps a row back to its lane.
template <int B>
__device__ __forceinline__ constexpr int tc_lane(int r) {
  return 4 * (r % (B / 4)) + r / (B / 4);
}

// Byte offset of (row, k) in a staged operand of R rows x 128 K-bytes.
__device__ __forceinline__ uint32_t tc_off(int R, int row, int k) {
  return (uint32_t)((k >> 5) * (R / 8) * 256 + (row >> 3) * 256 + ((k & 31) >> 4) * 128 + (row & 7) * 16 + (k & 15));
}

__device__ __forceinline__ uint64_t tc_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  const uint64_t t0 = tc_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (tc_ns() - t0 > kTcWaitLimitNs) return false;
  }
}

// Warp roles of the Gram pass CTA (one CTA per SM):
//   warp 0     producer: lane 0 keeps a ring of RING raw tiles filled by 1-D
//              bulk copies (block rows and row scales of one tile each);
//   warp 1     MMA issuer: lane 0 issues the tile's K = 32 UMMAs into one of
//              two TMEM accumulators and commits them to the stage's mbarrier;
//   warps 2-5  epilogue: every kTcDrain tiles they read the finished
//              accumulator (tcgen05.ld; warp w owns TMEM lanes 32 (w % 4)),
//              weight the limb pairs and free it, while the MMAs go on in the
//              other accumulator;
//   warps 6-   transposers, NG groups of TW warps, group g taking tiles
//              j = g mod NG: scale the rows, split them into byte limbs and
//              store them in operand stage j mod OPS.
// Hand-offs are mbarriers only (no CTA-wide barrier inside the loop): raw
// slot full (bulk-copy bytes) / empty (TW arrivals), operand stage full (TW
// arrivals) / empty (MMA commit), accumulator full (commit) / empty (4
// arrivals).  Every wait gives up after 2 s or once another role gave up.
template <int B>
struct TcShape {
  static constexpr int TILE = 128;                           // rows (K bytes) per tile
  static constexpr int MR = 4 * B;                           // real A rows (limb, lane)
  static constexpr int M = 128;                              // UMMA M (zero rows above MR)
  static constexpr int N = 4 * B;                            // UMMA N
  static constexpr int A_BYTES = M * TILE;
  static constexpr int B_BYTES = N * TILE;
  static constexpr int STAGE = A_BYTES + B_BYTES;            // one operand stage
  static constexpr int OPS = 4;                              // operand stages
  static constexpr int RAW_Y = TILE * B * 4;                 // a tile's block rows
  static constexpr int RAW_BYTES = RAW_Y + TILE * 4;         // plus its row scales
  static constexpr int RING = 4;                             // raw tiles in flight
  static constexpr int GROUPS = B / 4;                       // 128-bit words per row
  static constexpr int TASKS = (TILE / 4) * GROUPS;          // 4 rows x 4 lanes each
  static constexpr int TW = TASKS / 32;                      // transposer warps per tile
  static constexpr int NG = B >= 32 ? 2 : 4;                 // tiles transposed at once
  static constexpr int XW0 = 6;                              // first transposer warp
  static constexpr int WARPS = XW0 + NG * TW;
  static constexpr int THREADS = 32 * WARPS;
  static constexpr int COLS = 2 * N <= 128 ? 128 : 256;      // two accumulators
  static constexpr uint32_t IDESC = (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
  static_assert(TASKS % 32 == 0 && OPS % NG == 0 && RING % NG == 0, "tile shape");
};

template <int B>
constexpr size_t gram_tc_smem_bytes() {
  return (size_t)TcShape<B>::OPS * TcShape<B>::STAGE + (size_t)TcShape<B>::RING * TcShape<B>::RAW_BYTES;
}
// dynamic + static (the CTA sums, barriers) within the 227 KB a CTA may hold
static_assert(gram_tc_smem_bytes<16>() + 16 * 16 * 8 + 1024 <= 232448, "Gram stages too large");
static_assert(gram_tc_smem_bytes<32>() + 32 * 32 * 8 + 1024 <= 232448, "Gram stages too large");

__device__ __forceinline__ void byte_transpose4(const uint32_t (&v)[4], uint32_t (&w)[4]) {
  // w[a] = bytes a of v[0..3]: limb a of four consecutive rows
  const uint32_t t0 = __byte_perm(v[0], v[1], 0x5140), t1 = __byte_perm(v[2], v[3], 0x5140);
  const uint32_t t2 = __byte_perm(v[0], v[1], 0x7362), t3 = __byte_perm(v[2], v[3], 0x7362);
  w[0] = __byte_perm(t0, t1, 0x5410);
  w[1] = __byte_perm(t0, t1, 0x7632);
  w[2] = __byte_perm(t2, t3, 0x5410);
  w[3] = __byte_perm(t2, t3, 0x7632);
}

// y * s * 2^-32 mod p without the final correction: a value in [0, 2p) < 2^32
// congruent to the Montgomery product.  The Gram pass only needs the value
// mod p (its limb products are exact for any 32-bit operand and its sums are
// reduced mod p), so the comparison and subtraction are left out.
__device__ __forceinline__ uint32_t redc_lazy(uint32_t y, uint32_t s, const ModP& M) {
  uint32_t lo = 0, hi = 0;
  mac_cc(y, s, lo, hi);
  mac_cc(lo * M.pinv, M.p, lo, hi);  // lo becomes 0; y s + q p < 2 p 2^32
  return hi;
}

// A bounded wait that also ends when another role of the CTA gave up.
__device__ __forceinline__ bool mbar_wait_or(uint32_t addr, uint32_t parity, const volatile int* abort) {
  const uint64_t t0 = tc_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (*abort) return false;
    if (tc_ns() - t0 > kTcWaitLimitNs) return false;
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Thread 0 of the producer: the raw rows (and scales) of `tile` into ring
// slot `dst` by two 1-D bulk copies completing on `mbar` (rows past the end
// are not copied; the scale copy is rounded up to 16 bytes, which the scale
// arrays are padded for).
template <int B>
__device__ __forceinline__ void tc_fetch(const PassParams& P, int64_t tile, unsigned char* dst, uint64_t* mbar) {
  using T = TcShape<B>;
  const int64_t r0 = tile * T::TILE;
  const int rows = (int)(P.rows - r0 < T::TILE ? P.rows - r0 : T::TILE);
  const uint32_t ybytes = (uint32_t)rows * B * 4;
  const uint32_t sbytes = (uint32_t)((rows * 4 + 15) & ~15);
  const uint32_t mb = smem_u32(mbar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(ybytes + sbytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<const uint32_t*>(P.X) + r0 * B), "r"(ybytes), "r"(mb)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst + T::RAW_Y)),
               "l"(P.scale + r0), "r"(sbytes), "r"(mb)
               : "memory");
}

template <int B>
__global__ void __launch_bounds__(TcShape<B>::THREADS, 1) gram_tc_kernel(PassParams P, int* status) {
  using T = TcShape<B>;
  constexpr int NP = B * (B + 1) / 2;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t raw_full[T::RING], raw_empty[T::RING];
  __shared__ __align__(8) uint64_t op_full[T::OPS], op_empty[T::OPS];
  __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2], fin;
  __shared__ uint32_t tmem_base_s;
  __shared__ unsigned long long red[B * B];
  __shared__ bool is_last;
  __shared__ volatile int s_fail;
  __shared__ int64_t s_issued;
  unsigned char* const raw0 = tc_smem + T::OPS * T::STAGE;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const ModP M = P.M;

  // zero the operand stages once (the A rows above 4B stay zero), the CTA sums, the barriers
  for (int e = tid; e < T::OPS * T::STAGE / 16; e += T::THREADS)
    reinterpret_cast<uint4*>(tc_smem)[e] = make_uint4(0, 0, 0, 0);
  for (int e = tid; e < B * B; e += T::THREADS) red[e] = 0;
  if (tid == 0) {
    s_fail = 0;
    s_issued = 0;
    auto init = [](uint64_t* bar, int count) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    };
    for (int i = 0; i < T::RING; ++i) {
      init(&raw_full[i], 1);
      init(&raw_empty[i], T::TW);
    }
    for (int i = 0; i < T::OPS; ++i) {
      init(&op_full[i], T::TW);
      init(&op_empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      init(&acc_full[i], 1);
      init(&acc_empty[i], 4);
    }
    init(&fin, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(T::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the zeroed stages, for the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  griddep_wait();  // the block this pass reads was written by the previous kernel

  const int64_t ntiles = (P.rows + T::TILE - 1) / T::TILE;
  const int64_t mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;  // tiles of this CTA
  auto give_up = [&]() {
    s_fail = 1;
    atomicExch(status, 1);
  };

  // epilogue state: thread (warp w in 2..5, lane l) owns A row m = 32 (w % 4)
  // + l = (a, i) and keeps sum_c 256^{a+c} D[m][(c, j)] mod p per lane j
  uint32_t part[B];
#pragma unroll
  for (int j = 0; j < B; ++j) part[j] = 0;
  const int quad = warp & 3;
  const int m_row = 32 * quad + lane;
  const bool reader = warp >= 2 && warp < 6 && m_row < T::MR;

  if (warp == 0) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      for (int64_t j = 0; j < mine; ++j) {
        const int slot = (int)(j % T::RING);
        if (j >= T::RING && !mbar_wait_or(smem_u32(&raw_empty[slot]), (uint32_t)((j / T::RING - 1) & 1), &s_fail)) {
          give_up();
          break;
        }
        tc_fetch<B>(P, blockIdx.x + j * gridDim.x, raw0 + slot * T::RAW_BYTES, &raw_full[slot]);
        s_issued = j + 1;
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      for (int64_t j = 0; j < mine; ++j) {
        const int s = (int)(j % T::OPS);
        const int64_t grp = j / kTcDrain;
        const int a = (int)(grp & 1);
        const bool first = j % kTcDrain == 0;
        if (first && grp >= 2 && !mbar_wait_or(smem_u32(&acc_empty[a]), (uint32_t)((grp / 2 - 1) & 1), &s_fail)) {
          give_up();
          break;
        }
        if (!mbar_wait_or(smem_u32(&op_full[s]), (uint32_t)((j / T::OPS) & 1), &s_fail)) {
          give_up();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(tc_smem + s * T::STAGE), b0 = a0 + T::A_BYTES;
#pragma unroll
        for (int kb = 0; kb < T::TILE / 32; ++kb) {
          const uint64_t da = umma_desc(a0 + kb * (T::M / 8) * 256);
          const uint64_t db = umma_desc(b0 + kb * (T::N / 8) * 256);
          const uint32_t accum = (!first || kb > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
              :
              : "r"(tmem + (uint32_t)(a * T::N)), "l"(da), "l"(db), "r"(T::IDESC), "r"(accum), "r"(0u), "r"(0u),
                "r"(0u), "r"(0u)
              : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&op_empty[s]))
                     : "memory");
        if (j % kTcDrain == kTcDrain - 1 || j == mine - 1)
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&acc_full[a]))
                       : "memory");
      }
    }
  } else if (warp < T::XW0) {
    // ------------------------------------------------------------ epilogue
    uint32_t wgt[4];  // 2^{8(a + c)} mod p for c = 0..3, a = this row's limb
    {
      uint64_t w = 1;
      for (int e = 0; e < (reader ? m_row / B : 0); ++e) w = w * 256 % M.p;
      for (int c = 0; c < 4; ++c) {
        wgt[c] = (uint32_t)w;
        w = w * 256 % M.p;
      }
    }
    const int64_t ngrp = (mine + kTcDrain - 1) / kTcDrain;
    for (int64_t G = 0; G < ngrp; ++G) {
      const int a = (int)(G & 1);
      if (!mbar_wait_or(smem_u32(&acc_full[a]), (uint32_t)((G / 2) & 1), &s_fail)) {
        give_up();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int c0 = 0; c0 < T::N; c0 += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)(a * T::N + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (reader) {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int n = c0 + q, c = n / B, j = tc_lane<B>(n % B);
            part[j] = addmod(part[j], mulmod(v[q], wgt[c], M), M.p);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[a]);
    }
  } else {
    // ------------------------------------------------------------ transposers
    const int xw = warp - T::XW0, g = xw / T::TW;
    const int task = (xw % T::TW) * 32 + lane;
    const int gw = task % T::GROUPS, qd = task / T::GROUPS;  // word gw of rows 4 qd .. 4 qd + 3
    for (int64_t j = g; j < mine; j += T::NG) {
      const int slot = (int)(j % T::RING), s = (int)(j % T::OPS);
      if (!mbar_wait_or(smem_u32(&raw_full[slot]), (uint32_t)((j / T::RING) & 1), &s_fail)) {
        give_up();
        break;
      }
      if (j >= T::OPS && !mbar_wait_or(smem_u32(&op_empty[s]), (uint32_t)((j / T::OPS - 1) & 1), &s_fail)) {
        give_up();
        break;
      }
      const unsigned char* raw = raw0 + slot * T::RAW_BYTES;
      const uint32_t* scl = reinterpret_cast<const uint32_t*>(raw + T::RAW_Y);
      unsigned char* const bufA = tc_smem + s * T::STAGE;
      unsigned char* const bufB = bufA + T::A_BYTES;
      const int64_t r0 = (blockIdx.x + j * gridDim.x) * T::TILE;
      uint4 y[4];
      uint32_t sc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int rr = 4 * qd + q;
        const bool in = r0 + rr < P.rows;
        y[q] = in ? *reinterpret_cast<const uint4*>(raw + ((size_t)rr * B + 4 * gw) * 4) : make_uint4(0, 0, 0, 0);
        sc[q] = in ? scl[rr] : 0u;
      }
#pragma unroll
      for (int c4 = 0; c4 < 4; ++c4) {  // lane 4 gw + c4
        uint32_t z[4], u[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint32_t yv = c4 == 0 ? y[q].x : c4 == 1 ? y[q].y : c4 == 2 ? y[q].z : y[q].w;
          z[q] = redc_lazy(yv, sc[q], M);
          u[q] = P.gram_sym ? z[q] : yv;
        }
        uint32_t wz[4], wu[4];
        byte_transpose4(z, wz);
        byte_transpose4(u, wu);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          *reinterpret_cast<uint32_t*>(bufA + tc_off(T::M, a * B + c4 * T::GROUPS + gw, 4 * qd)) = wz[a];
          *reinterpret_cast<uint32_t*>(bufB + tc_off(T::N, a * B + c4 * T::GROUPS + gw, 4 * qd)) = wu[a];
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // stores visible to the tensor cores
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&op_full[s]);
        mbar_arrive(&raw_empty[slot]);
      }
    }
  }
  griddep_launch();
  __syncthreads();
  if (s_fail) {  // let what was committed or fetched finish before the memory goes away
    if (tid == 32) {
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&fin))
                   : "memory");
      mbar_wait(smem_u32(&fin), 0);
    }
    if (tid == 0) {  // the last RING fetches issued, one per slot
      const int64_t hi = s_issued;
      for (int64_t j = hi > T::RING ? hi - T::RING : 0; j < hi; ++j)
        mbar_wait(smem_u32(&raw_full[(int)(j % T::RING)]), (uint32_t)((j / T::RING) & 1));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::COLS) : "memory");
  }
  // CTA sums: G[i][j] += part (4 limb rows a per (i, j))
  if (reader) {
    const int i = tc_lane<B>(m_row % B);
#pragma unroll
    for (int jj = 0; jj < B; ++jj) atomicAdd(&red[i * B + jj], (unsigned long long)part[jj]);
  }
  __syncthreads();
  unsigned long long* const acc = P.gram_acc + (size_t)(blockIdx.x % P.replicas) * P.gram_stride;
  for (int q = tid; q < NP; q += T::THREADS) {
    int i, jj;
    pair_of(q, B, i, jj);
    atomicAdd(&acc[q], (unsigned long long)reduce(red[i * B + jj], M));
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) is_last = (atomicAdd(P.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // the last CTA: the finished term (real pairs), then reset
  const int b = P.b_real;
  const int npr = b * (b + 1) / 2;
  uint32_t* S_out = *P.S_ptr + (size_t)__ldcg(P.term_ctr) * npr;
  for (int q = tid; q < npr; q += T::THREADS) {
    int i, jj;
    pair_of(q, b, i, jj);
    const int qb = pair_index(i, jj, B);
    unsigned long long v = 0;
    for (int r = 0; r < P.replicas; ++r) v += __ldcg(P.gram_acc + (size_t)r * P.gram_stride + qb);
    S_out[q] = mulmod(reduce(v, M), P.gram_mul, M);
  }
  __syncthreads();
  for (int q = tid; q < NP * P.replicas; q += T::THREADS)
    __stcg(P.gram_acc + (size_t)(q / NP) * P.gram_stride + q % NP, 0ull);
  if (tid == 0) {
    *P.term_ctr += 1u;
    atomicExch(P.counter, 0u);
  }
}

// ---------------------------------------------------------------- persistent batched loop
// Grid-wide barrier of a cooperative launch: thread 0 of each CTA arrives on
// bar[0]; the last arrival resets it and advances the generation bar[1]; the
// others wait for the generation to move, at most limit_ns of wall time
// (%globaltimer), after which they set *error and every CTA returns false at
// this or the next barrier.  `expected` is the number of CTAs that arrive.
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool grid_barrier(unsigned int* bar, int* error, uint64_t limit_ns, unsigned int expected) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned int* gen = bar + 1;
    const unsigned int g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == expected - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = global_ns();
      while (*gen == g) {
        if (*(volatile int*)error) { ok = 0; break; }
        if (global_ns() - t0 > limit_ns) {
          atomicExch(error, 1);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    s_ok = ok && *(volatile int*)error == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// Applications [t_begin, t_end) of B for a batch phase in one launch: pass
// over the stacked rows of A, grid barrier, pass over the rows of A^T, grid
// barrier.  The blocks are read with coherent loads (they change between
// barriers); the Gram partials go to the per-(matrix, term) slots.
template <int B, int FE, int L>
__global__ void __launch_bounds__(kThreads, (B >= 32 ? 2 : 4)) persistent_kernel(PersistParams Q) {
  extern __shared__ __align__(16) uint32_t gram_smem[];
  __shared__ unsigned long long red[B * (B + 1) / 2];
  __shared__ bool is_last;
  int cur = Q.cur0;
  for (int64_t t = Q.t_begin; t < Q.t_end; ++t) {
    PassParams P = Q.odd;
    P.X = Q.X[cur];
    P.Y = Q.U;
    P.term = 2 * t + 1;
    pass_body<B, kModeOdd, FE, true, true, L>(P, gram_smem, red, is_last);
    if (!grid_barrier(Q.bar, Q.error, Q.limit_ns, gridDim.x)) return;
    P = Q.even;
    P.X = Q.U;
    P.Y = Q.X[cur ^ 1];
    P.term = 2 * t + 2;
    pass_body<B, kModeEven, FE, true, true, L>(P, gram_smem, red, is_last);
    if (!grid_barrier(Q.bar, Q.error, Q.limit_ns, gridDim.x)) return;
    cur ^= 1;
  }
}

// A cooperative launch whose CTAs pass `rounds` grid barriers that wait for
// `expected` arrivals (expected > gridDim.x: a barrier nothing completes).
__global__ void barrier_check_kernel(unsigned int* bar, int* error, uint64_t limit_ns, unsigned int expected,
                                     int rounds) {
  for (int r = 0; r < rounds; ++r)
    if (!grid_barrier(bar, error, limit_ns, expected)) return;
}

// Long rows: one warp per chunk of at most kChunkNnz entries, warps taking the
// next chunk from a dispenser (an atomic ticket), so that the kernel ends
// within about one chunk's time of its last warp.  Lanes form RPW slots of TPR
// threads; slot s takes entries beg+s, beg+s+RPW, ...  The slot sums (exact
// residues) are combined with shuffles and added to heavy_acc with 64-bit
// atomics.  At widths 16 and 32 a thread holds 4 lanes and sums eight entries
// per step (gather_sum8): a whole gathered row per load instruction, as many
// bytes in flight as 8 lanes and four entries.
template <int B>
constexpr int kChunkLpt = (B >= 16) ? 4 : kDefaultLpt<B>;

template <int B, int FE, int L = kChunkLpt<B>>
__global__ void __launch_bounds__(kThreads, 3) chunk_kernel(ChunkParams P) {
  using S = Shape<B, L>;
  constexpr int LPT = S::LPT, TPR = S::TPR, RPW = S::RPW;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int slot = lane / TPR;
  const ModP M = P.M;
  griddep_wait();
  for (;;) {
    unsigned int ticket = 0;
    if (lane == 0) ticket = atomicAdd(P.next, 1u);
    const int64_t ch = __shfl_sync(0xffffffffu, ticket, 0);
    if (ch >= P.nchunks) {
      // the last warp of the launch to run out of chunks (all tickets are
      // taken by then) rewinds the dispenser for the next launch
      if (lane == 0 && atomicAdd(P.next + 1, 1u) == gridDim.x * (unsigned)kWarps - 1u) {
        P.next[0] = 0u;
        P.next[1] = 0u;
      }
      break;
    }
    const uint32_t beg = P.chunk_begin[ch], end = P.chunk_end[ch];
    const uint32_t row = P.chunk_row[ch];
    uint64_t acc[LPT];
#pragma unroll
    for (int l = 0; l < LPT; ++l) acc[l] = 0;
    if constexpr (L == 4 && B >= 16)
      gather_sum8<B, FE, L>(P.cv, beg + slot, end, (uint32_t)RPW, P.X, sub, M, acc);
    else
      gather_sum<B, FE, false, L>(P.cv, beg + slot, end, (uint32_t)RPW, P.X, sub, M, acc);
    uint32_t y[LPT];
#pragma unroll
    for (int l = 0; l < LPT; ++l) y[l] = reduce(acc[l], M);
#pragma unroll
    for (int off = TPR; off < 32; off <<= 1) {
#pragma unroll
      for (int l = 0; l < LPT; ++l) y[l] = addmod(y[l], __shfl_xor_sync(0xffffffffu, y[l], off), M.p);
    }
    if (slot == 0) {
      unsigned long long* h = P.heavy_acc + (size_t)row * B;
#pragma unroll
      for (int l = 0; l < LPT; ++l) atomicAdd(&h[S::lane_of(sub, l)], (unsigned long long)y[l]);
    }
  }
  griddep_launch();
}

// x[c'][l] = (l < b) ? V[l][colperm[c']] : 0   (V vector-major, original order)
__global__ void scatter_block_kernel(const uint32_t* __restrict__ V, const int32_t* __restrict__ colperm,
                                     int64_t n, int b, int B, uint32_t* __restrict__ out) {
  const int64_t total = n * B;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / B;
    const int l = (int)(i % B);
    out[i] = l < b ? V[(size_t)l * n + colperm[c]] : 0u;
  }
}

// curv[l][colperm[c']] = x[c'][l] * dcinv[c']
__global__ void gather_curv_kernel(const uint32_t* __restrict__ x, const uint32_t* __restrict__ dcinv,
                                   const int32_t* __restrict__ colperm, int64_t n, int b, int B, ModP M,
                                   uint32_t* __restrict__ curv) {
  const int64_t total = n * b;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / b;
    const int l = (int)(i % b);
    curv[(size_t)l * n + colperm[c]] = mulmod(x[c * B + l], dcinv[c], M);
  }
}

// Slot-per-term Gram sums of segments [seg_begin, seg_end) -> sequence terms
// (real pairs; odd terms were accumulated from z R^{-1} and take a factor R).
__global__ void batch_finalize_kernel(const unsigned long long* __restrict__ gram_all,
                                      const int64_t* __restrict__ seg_G_off, uint32_t* __restrict__ S_all,
                                      const int64_t* __restrict__ seg_S_off, const int64_t* __restrict__ seg_terms,
                                      int seg_begin, int b, int B, uint32_t r1, ModP M) {
  const int s = seg_begin + (int)blockIdx.y;
  const int npr = b * (b + 1) / 2, NP = B * (B + 1) / 2;
  const int64_t total = seg_terms[s] * npr;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = e / npr;
    const int q = (int)(e - t * npr);
    int i, j;
    pair_of(q, b, i, j);
    const unsigned long long v = gram_all[seg_G_off[s] + t * NP + pair_index(i, j, B)];
    const uint32_t r = reduce(v, M);
    S_all[seg_S_off[s] + t * npr + q] = (t & 1) ? mulmod(r, r1, M) : r;
  }
}

int launch_batch_finalize(cudaStream_t s, const unsigned long long* gram_all, const int64_t* d_seg_G_off,
                          uint32_t* S_all, const int64_t* d_seg_S_off, const int64_t* d_seg_terms, int seg_begin,
                          int seg_end, int64_t max_terms, int b, int B, const ModP& M) {
  if (seg_end <= seg_begin) return RR_OK;
  const int64_t work = max_terms * (b * (b + 1) / 2);
  const dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 1024)), (unsigned)(seg_end - seg_begin));
  batch_finalize_kernel<<<grid, 256, 0, s>>>(gram_all, d_seg_G_off, S_all, d_seg_S_off, d_seg_terms, seg_begin, b, B,
                                             M.r1, M);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// ---------------------------------------------------------------- launchers
// dynamic shared memory of the pass kernel: the per-warp Gram staging area
template <int B>
constexpr size_t pass_smem_bytes() {
  return (size_t)kWarps * 4 * (B >= 8 ? GramMma<B, 4>::kWords : GramCore<B, 4>::kWords);
}

// CTAs for a pass over `rows` rows: the resident maximum, but no more CTAs
// than there are warp batches for (idle CTAs would still add their Gram
// partials and lengthen the pass on small matrices).
template <int B>
static int pass_grid(const rr_krylov* kr, int64_t rows) {
  const int64_t nbatch = (rows + Shape<B>::RPW - 1) / Shape<B>::RPW;
  const int64_t need = (nbatch + kWarps - 1) / kWarps;
  return (int)std::max<int64_t>(1, std::min<int64_t>(kr->grid_pass, need));
}

template <int B>
static int pass_grid_lean(const rr_krylov* kr, int64_t rows) {
  constexpr int RPW = Shape<B, kLeanLpt<B>>::RPW;
  const int64_t nbatch = (rows + RPW - 1) / RPW;
  const int64_t need = (nbatch + kWarps - 1) / kWarps;
  return (int)std::max<int64_t>(1, std::min<int64_t>(kr->grid_lean, need));
}

// Kernel launches of the single-matrix path, through cudaLaunchKernelEx.
template <class... Args>
static int launch_ex(const rr_krylov* kr, void (*fn)(Args...), dim3 grid, dim3 block, size_t smem,
                          cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  // the kernel may be scheduled while its predecessor on the stream finishes;
  // it waits for it (griddep_wait) before reading the predecessor's output
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)kr;
  RR_CUDA(cudaLaunchKernelEx(&cfg, fn, args...));
  return RR_OK;
}

// Single-matrix launches: a fused pass (kFusedOdd / kFusedEven) adds its Gram
// term itself; a lean pass runs without it (no staging, no tensor-core flush,
// so fewer registers and no shared memory) and is followed by a tcgen05 Gram
// pass over the block it wrote (kModeGram).  The initial pass computes S_0
// itself.
template <int B, int FE>
static int launch_pass_BF(rr_krylov* kr, const PassParams& P, int mode, dim3 grid, cudaStream_t s) {
  const dim3 block(kThreads);
  const size_t sm = pass_smem_bytes<B>();
  switch (mode) {
    case kModeInit: return launch_ex(kr, pass_kernel<B, kModeInit, FE, true>, grid, block, sm, s, P);
    case kModeOdd:
      if constexpr (kFusedOdd<B>) return launch_ex(kr, pass_kernel<B, kModeOdd, FE, true>, grid, block, sm, s, P);
      else return launch_ex(kr, pass_kernel<B, kModeOdd, FE, false, kLeanLpt<B>>, grid, block, 0, s, P);
    case kModeEven:
      if constexpr (kFusedEven<B>) return launch_ex(kr, pass_kernel<B, kModeEven, FE, true>, grid, block, sm, s, P);
      else return launch_ex(kr, pass_kernel<B, kModeEven, FE, false, kLeanLpt<B>>, grid, block, 0, s, P);
  }
  return fail(RR_EINVAL, "pass mode %d has no pass kernel at width %d", mode, B);
}

// Gram passes (widths 16 and 32) run on tcgen05 (gram_tc_kernel).
template <int B>
static int launch_gram_tc(rr_krylov* kr, const PassParams& P, cudaStream_t s) {
  const int64_t ntiles = (P.rows + TcShape<B>::TILE - 1) / TcShape<B>::TILE;
  const dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)kr->mat->ctx->num_sms)));
  return launch_ex(kr, gram_tc_kernel<B>, grid, dim3(TcShape<B>::THREADS), gram_tc_smem_bytes<B>(), s, P,
                        kr->d_status.ptr);
}

template <int B>
static int launch_pass_B(rr_krylov* kr, const PassParams& P, int mode) {
  if constexpr (B >= 16) {
    if (mode == kModeGram) {
      cudaStream_t s = kr->launch_stream ? kr->launch_stream : kr->mat->ctx->stream;
      return launch_gram_tc<B>(kr, P, s);
    }
  }
  const bool lean = (mode == kModeOdd && !kFusedOdd<B>) || (mode == kModeEven && !kFusedEven<B>);
  const dim3 grid(lean ? pass_grid_lean<B>(kr, P.rows) : pass_grid<B>(kr, P.rows));
  cudaStream_t s = kr->launch_stream ? kr->launch_stream : kr->mat->ctx->stream;
  return kr->fold4 ? launch_pass_BF<B, 4>(kr, P, mode, grid, s) : launch_pass_BF<B, 2>(kr, P, mode, grid, s);
}

template <int B, int FE>
static int set_pass_smem() {
  const int sm = (int)pass_smem_bytes<B>();
  RR_CUDA(cudaFuncSetAttribute(pass_kernel<B, kModeInit, FE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  RR_CUDA(cudaFuncSetAttribute(pass_kernel<B, kModeOdd, FE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  RR_CUDA(cudaFuncSetAttribute(pass_kernel<B, kModeEven, FE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  return RR_OK;
}

static int launch_pass(rr_krylov* kr, const PassParams& P, int mode) {
  kr->launches += 1;
  switch (kr->B) {
    case 4: return launch_pass_B<4>(kr, P, mode);
    case 8: return launch_pass_B<8>(kr, P, mode);
    case 16: return launch_pass_B<16>(kr, P, mode);
    case 32: return launch_pass_B<32>(kr, P, mode);
  }
  return fail(RR_EINVAL, "unsupported padded block width %d", kr->B);
}

template <int B>
static int launch_chunk_B(rr_krylov* kr, const ChunkParams& P) {
  const dim3 grid((unsigned)std::max<int64_t>(1, std::min<int64_t>(kr->grid_chunk, (P.nchunks + kWarps - 1) / kWarps))),
      block(kThreads);
  cudaStream_t s = kr->launch_stream ? kr->launch_stream : kr->mat->ctx->stream;
  if (kr->fold4) return launch_ex(kr, chunk_kernel<B, 4>, grid, block, 0, s, P);
  return launch_ex(kr, chunk_kernel<B, 2>, grid, block, 0, s, P);
}

static int launch_chunk(rr_krylov* kr, const ChunkParams& P) {
  kr->launches += 1;
  switch (kr->B) {
    case 4: return launch_chunk_B<4>(kr, P);
    case 8: return launch_chunk_B<8>(kr, P);
    case 16: return launch_chunk_B<16>(kr, P);
    case 32: return launch_chunk_B<32>(kr, P);
  }
  return fail(RR_EINVAL, "unsupported padded block width %d", kr->B);
}

template <int B>
static int occupancy_B(rr_krylov* kr, int* pass_blocks, int* chunk_blocks, int* lean_blocks) {
  const size_t sm = pass_smem_bytes<B>();
  if (kr->fold4) {
    RR_TRY((set_pass_smem<B, 4>()));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(pass_blocks, pass_kernel<B, kModeOdd, 4>, kThreads, sm));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunk_blocks, chunk_kernel<B, 4>, kThreads, 0));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(lean_blocks, pass_kernel<B, kModeOdd, 4, false, kLeanLpt<B>>,
                                                          kThreads, 0));
  } else {
    RR_TRY((set_pass_smem<B, 2>()));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(pass_blocks, pass_kernel<B, kModeOdd, 2>, kThreads, sm));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunk_blocks, chunk_kernel<B, 2>, kThreads, 0));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(lean_blocks, pass_kernel<B, kModeOdd, 2, false, kLeanLpt<B>>,
                                                          kThreads, 0));
  }
  return RR_OK;
}

template <int B>
static int launch_pass_raw_B(cudaStream_t s, int fold4, int grid, const PassParams& P, int mode) {
  const size_t sm = pass_smem_bytes<B>();
  const dim3 g(grid), block(kThreads);
  if (fold4) {
    if (mode == kModeInit) pass_kernel<B, kModeInit, 4><<<g, block, sm, s>>>(P);
    else if (mode == kModeOdd) pass_kernel<B, kModeOdd, 4><<<g, block, sm, s>>>(P);
    else pass_kernel<B, kModeEven, 4><<<g, block, sm, s>>>(P);
  } else {
    if (mode == kModeInit) pass_kernel<B, kModeInit, 2><<<g, block, sm, s>>>(P);
    else if (mode == kModeOdd) pass_kernel<B, kModeOdd, 2><<<g, block, sm, s>>>(P);
    else pass_kernel<B, kModeEven, 2><<<g, block, sm, s>>>(P);
  }
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

int launch_pass_raw(cudaStream_t s, int B, int fold4, int grid, const PassParams& P, int mode) {
  switch (B) {
    case 4: return launch_pass_raw_B<4>(s, fold4, grid, P, mode);
    case 8: return launch_pass_raw_B<8>(s, fold4, grid, P, mode);
    case 16: return launch_pass_raw_B<16>(s, fold4, grid, P, mode);
    case 32: return launch_pass_raw_B<32>(s, fold4, grid, P, mode);
  }
  return fail(RR_EINVAL, "unsupported padded block width %d", B);
}

template <int B, int L>
static int launch_persistent_BL(cudaStream_t s, int fold4, int grid, PersistParams& Q) {
  const size_t sm = pass_smem_bytes<B>();
  void* args[] = {&Q};
  // the shared-memory limit was raised by persistent_blocks_per_sm at set-up
  const void* fn = fold4 ? (const void*)persistent_kernel<B, 4, L> : (const void*)persistent_kernel<B, 2, L>;
  RR_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, sm, s));
  return RR_OK;
}

template <int B, int L>
static int persistent_blocks_BL(int fold4, int* blocks) {
  const size_t sm = pass_smem_bytes<B>();
  if (fold4) {
    RR_CUDA(cudaFuncSetAttribute(persistent_kernel<B, 4, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, persistent_kernel<B, 4, L>, kThreads, sm));
  } else {
    RR_CUDA(cudaFuncSetAttribute(persistent_kernel<B, 2, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, persistent_kernel<B, 2, L>, kThreads, sm));
  }
  return RR_OK;
}

// Lanes per thread the persistent kernel is built for at padded width B.
int persistent_lane_options(int B, int* opts) {
  if (B == 4) {
    opts[0] = 4;
    return 1;
  }
  opts[0] = 4;
  opts[1] = 8;
  return 2;
}

int launch_persistent_raw(cudaStream_t s, int B, int fold4, int grid, int lpt, PersistParams& Q) {
  switch (B * 100 + lpt) {
    case 404: return launch_persistent_BL<4, 4>(s, fold4, grid, Q);
    case 804: return launch_persistent_BL<8, 4>(s, fold4, grid, Q);
    case 808: return launch_persistent_BL<8, 8>(s, fold4, grid, Q);
    case 1604: return launch_persistent_BL<16, 4>(s, fold4, grid, Q);
    case 1608: return launch_persistent_BL<16, 8>(s, fold4, grid, Q);
    case 3204: return launch_persistent_BL<32, 4>(s, fold4, grid, Q);
    case 3208: return launch_persistent_BL<32, 8>(s, fold4, grid, Q);
  }
  return fail(RR_EINVAL, "no persistent kernel for width %d and %d lanes per thread", B, lpt);
}

int persistent_blocks_per_sm(int B, int fold4, int lpt, int* blocks) {
  switch (B * 100 + lpt) {
    case 404: return persistent_blocks_BL<4, 4>(fold4, blocks);
    case 804: return persistent_blocks_BL<8, 4>(fold4, blocks);
    case 808: return persistent_blocks_BL<8, 8>(fold4, blocks);
    case 1604: return persistent_blocks_BL<16, 4>(fold4, blocks);
    case 1608: return persistent_blocks_BL<16, 8>(fold4, blocks);
    case 3204: return persistent_blocks_BL<32, 4>(fold4, blocks);
    case 3208: return persistent_blocks_BL<32, 8>(fold4, blocks);
  }
  return fail(RR_EINVAL, "no persistent kernel for width %d and %d lanes per thread", B, lpt);
}

int launch_barrier_check(cudaStream_t s, int grid, unsigned int* bar, int* error, uint64_t limit_ns,
                         unsigned int expected, int rounds) {
  void* args[] = {&bar, &error, &limit_ns, &expected, &rounds};
  RR_CUDA(cudaLaunchCooperativeKernel((const void*)barrier_check_kernel, dim3(grid), dim3(kThreads), args, 0, s));
  return RR_OK;
}

template <int B>
static int pass_blocks_B(int fold4, int* blocks) {
  const size_t sm = pass_smem_bytes<B>();
  if (fold4) {
    RR_TRY((set_pass_smem<B, 4>()));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, pass_kernel<B, kModeEven, 4>, kThreads, sm));
  } else {
    RR_TRY((set_pass_smem<B, 2>()));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, pass_kernel<B, kModeEven, 2>, kThreads, sm));
  }
  return RR_OK;
}

int pass_blocks_per_sm(int B, int fold4, int* blocks) {
  switch (B) {
    case 4: return pass_blocks_B<4>(fold4, blocks);
    case 8: return pass_blocks_B<8>(fold4, blocks);
    case 16: return pass_blocks_B<16>(fold4, blocks);
    case 32: return pass_blocks_B<32>(fold4, blocks);
  }
  return fail(RR_EINVAL, "unsupported padded block width %d", B);
}

int rows_per_batch(int B, int lpt) {
  if (lpt <= 0) lpt = B >= 16 ? 8 : 4;
  return 32 * lpt / B;  // 32 / threads per row
}

int krylov_occupancy(rr_krylov* kr) {
  if (kr->B == 16)
    RR_CUDA(cudaFuncSetAttribute(gram_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gram_tc_smem_bytes<16>()));
  if (kr->B == 32)
    RR_CUDA(cudaFuncSetAttribute(gram_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)gram_tc_smem_bytes<32>()));
  int pb = 1, cb = 1, lb = 1;
  switch (kr->B) {
    case 4: RR_TRY(occupancy_B<4>(kr, &pb, &cb, &lb)); break;
    case 8: RR_TRY(occupancy_B<8>(kr, &pb, &cb, &lb)); break;
    case 16: RR_TRY(occupancy_B<16>(kr, &pb, &cb, &lb)); break;
    case 32: RR_TRY(occupancy_B<32>(kr, &pb, &cb, &lb)); break;
    default: return fail(RR_EINVAL, "unsupported padded block width %d", kr->B);
  }
  const int sms = kr->mat->ctx->num_sms;
  kr->grid_pass = std::max(1, pb) * sms;
  kr->grid_chunk = std::max(1, cb) * sms;
  kr->grid_lean = std::max(1, lb) * sms;
  return RR_OK;
}

static PassParams base_params(rr_krylov* kr) {
  PassParams P;
  std::memset(&P, 0, sizeof(P));
  P.heavy_acc = kr->heavy_acc.ptr;
  P.gram_acc = kr->gram_acc.ptr;
  P.gram_stride = kr->B * (kr->B + 1) / 2;
  P.replicas = kGramReplicas;
  P.counter = kr->counter.ptr;
  P.gram_mul = 1;
  P.w4 = kr->M.c32;
  P.w5 = (uint32_t)((uint64_t)kr->M.c32 * 256 % kr->M.p);
  P.w6 = (uint32_t)((uint64_t)P.w5 * 256 % kr->M.p);
  P.b_real = kr->b;
  P.M = kr->M;
  return P;
}

int krylov_launch_init(rr_krylov* kr, const uint32_t* d_w, bool emit_s0) {
  const int np = kr->b * (kr->b + 1) / 2;
  PassParams P = base_params(kr);
  P.rows = kr->mat->n;
  P.heavy_rows = 0;
  P.X = reinterpret_cast<const uint4*>(d_w);
  P.Y = reinterpret_cast<uint4*>(kr->X[kr->cur].ptr);
  P.scale = kr->dc_r.ptr;
  // S_0 goes to slot len - base; the caller publishes it (len += 1) later
  P.S_out = emit_s0 ? kr->S.ptr + (size_t)(kr->len - kr->base) * np : nullptr;
  return launch_pass(kr, P, kModeInit);
}

static int run_chunks(rr_krylov* kr, const DevCsr& A, const uint32_t* X) {
  if (A.nchunks == 0) return RR_OK;
  ChunkParams C;
  C.cv = A.cv.ptr;
  C.chunk_row = A.chunk_row.ptr;
  C.chunk_begin = A.chunk_begin.ptr;
  C.chunk_end = A.chunk_end.ptr;
  C.nchunks = A.nchunks;
  C.X = reinterpret_cast<const uint4*>(X);
  C.heavy_acc = kr->heavy_acc.ptr;
  C.next = kr->chunk_next.ptr;  // [ticket, warps done], zero between launches
  C.M = kr->M;
  return launch_chunk(kr, C);
}

// ev (optional): four events recorded before pass 1, after pass 1, after the
// chunks of pass 2 and after pass 2.
int krylov_launch_application(rr_krylov* kr, cudaEvent_t* ev) {
  rr_matrix* mat = kr->mat;
  cudaStream_t s = kr->launch_stream ? kr->launch_stream : mat->ctx->stream;
  uint32_t* x = kr->X[kr->cur].ptr;
  uint32_t* xn = kr->X[kr->cur ^ 1].ptr;
  if (ev) RR_CUDA(cudaEventRecord(ev[0], s));
  // pass 1: rows of A
  RR_TRY(run_chunks(kr, mat->A, x));
  PassParams P = base_params(kr);
  P.rowptr = mat->A.rowptr.ptr;
  P.cv = mat->A.cv.ptr;
  P.rows = mat->A.rows;
  P.heavy_rows = mat->A.heavy_rows;
  P.tail_begin = mat->A.live_rows;
  P.X = reinterpret_cast<const uint4*>(x);
  P.Y = reinterpret_cast<uint4*>(kr->U.ptr);
  P.scale = kr->dr_m.ptr;
  // kFusedOdd / kFusedEven: passes that add their own Gram terms
  const bool fused_odd = kr->B <= 8, fused_even = kr->B <= 16;
  if (fused_odd) {
    P.gram_mul = kr->M.r1;  // the odd pass sums z R^{-1} (x) U
    P.term_ctr = kr->d_term.ptr;
    P.S_ptr = kr->d_sptr.ptr;
  }
  RR_TRY(launch_pass(kr, P, kModeOdd));
  // odd term: sum over rows of z (x) U with z = U d_r^{-1}
  if (!fused_odd) {
    PassParams G = base_params(kr);
    G.rows = mat->A.live_rows > 0 ? mat->A.live_rows : mat->A.rows;  // zero rows add nothing
    G.X = reinterpret_cast<const uint4*>(kr->U.ptr);
    G.scale = kr->drinv_r.ptr;
    G.gram_sym = 0;
    G.term_ctr = kr->d_term.ptr;
    G.S_ptr = kr->d_sptr.ptr;
    RR_TRY(launch_pass(kr, G, kModeGram));
  }
  if (ev) RR_CUDA(cudaEventRecord(ev[1], s));
  // pass 2: rows of A^T
  RR_TRY(run_chunks(kr, mat->At, kr->U.ptr));
  if (ev) RR_CUDA(cudaEventRecord(ev[2], s));
  P.rowptr = mat->At.rowptr.ptr;
  P.cv = mat->At.cv.ptr;
  P.rows = mat->At.rows;
  P.heavy_rows = mat->At.heavy_rows;
  P.tail_begin = mat->At.live_rows;
  P.X = reinterpret_cast<const uint4*>(kr->U.ptr);
  P.Y = reinterpret_cast<uint4*>(xn);
  P.scale = kr->dc_m.ptr;
  P.scale2 = kr->dc_r.ptr;
  P.gram_mul = 1;
  if (fused_even) {
    P.term_ctr = kr->d_term.ptr;
    P.S_ptr = kr->d_sptr.ptr;
  }
  RR_TRY(launch_pass(kr, P, kModeEven));
  // even term: sum over rows of w' (x) w' with w' = x' d_c^{-1}
  if (!fused_even) {
    PassParams G = base_params(kr);
    G.rows = mat->At.live_rows > 0 ? mat->At.live_rows : mat->At.rows;  // zero rows add nothing
    G.X = reinterpret_cast<const uint4*>(xn);
    G.scale = kr->dcinv_r.ptr;
    G.gram_sym = 1;
    G.term_ctr = kr->d_term.ptr;
    G.S_ptr = kr->d_sptr.ptr;
    RR_TRY(launch_pass(kr, G, kModeGram));
  }
  if (ev) RR_CUDA(cudaEventRecord(ev[3], s));
  kr->len += 2;
  kr->cur ^= 1;
  return RR_OK;
}

int krylov_launch_get_curv(rr_krylov* kr, uint32_t* d_out) {
  const int64_t n = kr->mat->n;
  const int threads = 256;
  const int64_t want = (n * kr->b + threads - 1) / threads;
  const int blocks = (int)std::min<int64_t>(want, 65535);
  gather_curv_kernel<<<std::max(blocks, 1), threads, 0, kr->mat->ctx->stream>>>(
      kr->X[kr->cur].ptr, kr->dcinv.ptr, kr->mat->d_colperm.ptr, n, kr->b, kr->B, kr->M, d_out);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// The preconditioners in device order and in the forms the epilogues use:
// d_r R^2, d_c R^2, d_c R and d_c^{-1} (mod p; the inverse by Fermat, p prime).
__device__ __forceinline__ uint32_t inverse_mod(uint32_t a, const ModP& M) {  // a^(p-2), p prime
  uint32_t r = 1;
  for (uint32_t e = M.p - 2; e; e >>= 1) {
    if (e & 1) r = mulmod(r, a, M);
    a = mulmod(a, a, M);
  }
  return r;
}

__global__ void precond_kernel(const uint32_t* __restrict__ rp, const uint32_t* __restrict__ cp,
                               const int32_t* __restrict__ rowperm, const int32_t* __restrict__ colperm, int64_t m,
                               int64_t n, uint32_t R1, uint32_t R2, ModP M, uint32_t* __restrict__ dr_m,
                               uint32_t* __restrict__ drinv_r, uint32_t* __restrict__ dc_m, uint32_t* __restrict__ dc_r,
                               uint32_t* __restrict__ dcinv, uint32_t* __restrict__ dcinv_r) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m + n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < m) {
      const uint32_t r = rp[rowperm[i]];
      dr_m[i] = mulmod(r, R2, M);
      drinv_r[i] = mulmod(inverse_mod(r, M), R1, M);
    } else {
      const int64_t j = i - m;
      const uint32_t c = cp[colperm[j]];
      dc_m[j] = mulmod(c, R2, M);
      dc_r[j] = mulmod(c, R1, M);
      const uint32_t ci = inverse_mod(c, M);
      dcinv[j] = ci;
      dcinv_r[j] = mulmod(ci, R1, M);
    }
  }
}

int launch_precond(rr_krylov* kr, const uint32_t* d_rp, const uint32_t* d_cp, const int32_t* d_rowperm) {
  const int64_t m = kr->mat->m, n = kr->mat->n;
  const uint64_t p = kr->M.p, R1 = kr->M.r1, R2 = R1 * R1 % p;
  const int threads = 256;
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((m + n + threads - 1) / threads, 4 * 148 * 8));
  precond_kernel<<<blocks, threads, 0, kr->mat->ctx->stream>>>(d_rp, d_cp, d_rowperm, kr->mat->d_colperm.ptr, m, n,
                                                               (uint32_t)R1, (uint32_t)R2, kr->M, kr->dr_m.ptr,
                                                               kr->drinv_r.ptr, kr->dc_m.ptr, kr->dc_r.ptr,
                                                               kr->dcinv.ptr, kr->dcinv_r.ptr);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

int launch_scatter_block(rr_krylov* kr, const uint32_t* d_V, uint32_t* d_out) {
  const int64_t n = kr->mat->n;
  const int threads = 256;
  const int64_t want = (n * kr->B + threads - 1) / threads;
  const int blocks = (int)std::min<int64_t>(want, 65535);
  scatter_block_kernel<<<std::max(blocks, 1), threads, 0, kr->mat->ctx->stream>>>(d_V, kr->mat->d_colperm.ptr, n,
                                                                                  kr->b, kr->B, d_out);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

}  // namespace rr
