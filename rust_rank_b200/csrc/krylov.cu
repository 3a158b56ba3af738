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
// The block is stored interleaved, X[row][B] uint32 (B = 4..32 lanes), so a
// gathered row is one 16..128-byte segment read by B/4 threads with 128-bit
// loads.  Sums are accumulated lazily in 64 bits with a fold every 2 or 4
// products (rr_modp.cuh).  The Gram terms are reduced per CTA in shared
// memory, then across CTAs with 64-bit atomics; the last CTA to finish writes
// the finished term and resets the accumulators, so no separate reduction
// kernel and no host round trip is needed.
//
// Rows are renumbered by decreasing degree.  Rows longer than kHeavyDegree
// (Zipf-heavy columns of A^T) are cut into chunks of kChunkNnz entries that
// are processed warp-per-chunk and merged with 64-bit atomics; the pass
// kernel then applies the epilogue to them like to any other row.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "rr_internal.h"

namespace rr {

enum PassMode { kModeInit = 0, kModeOdd = 1, kModeEven = 2 };

struct PassParams {
  const uint32_t* rowptr;
  const int32_t* col;
  const uint32_t* val;
  int64_t rows;
  int64_t heavy_rows;
  const uint4* X;           // gathered block [cols][B/4]   (kModeInit: w [rows][B/4])
  uint4* Y;                 // output block   [rows][B/4]
  const uint32_t* scale;    // per-row diagonal: d_r (odd), d_c (even, init)
  unsigned long long* heavy_acc;  // [heavy_rows][B]
  unsigned long long* gram_acc;   // [B(B+1)/2]
  unsigned int* counter;
  uint32_t* S_out;          // finished term, real pairs; nullptr = do not emit
  int b_real;
  ModP M;
};

struct ChunkParams {
  const int32_t* col;
  const uint32_t* val;
  const uint32_t* chunk_row;
  const uint32_t* chunk_begin;
  const uint32_t* chunk_end;
  int64_t nchunks;
  const uint4* X;
  unsigned long long* heavy_acc;
  ModP M;
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

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

template <int B, int MODE, int FE>
__global__ void __launch_bounds__(kThreads) pass_kernel(PassParams P) {
  constexpr int TPR = B / 4;          // threads per row (one uint4 each)
  constexpr int RPW = 32 / TPR;       // rows per warp batch
  constexpr int NP = B * (B + 1) / 2; // pairs in padded space
  constexpr int PPL = (NP + 31) / 32; // pairs per lane

  __shared__ uint32_t zs[kWarps][RPW][B];
  __shared__ uint32_t us[kWarps][RPW][B];
  __shared__ unsigned long long red[NP];
  __shared__ bool is_last;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane % TPR;
  const int slot = lane / TPR;
  const ModP M = P.M;

  for (int q = threadIdx.x; q < NP; q += kThreads) red[q] = 0;

  int pi[PPL], pj[PPL];
#pragma unroll
  for (int t = 0; t < PPL; ++t) {
    const int q = lane + 32 * t;
    if (q < NP) pair_of(q, B, pi[t], pj[t]);
    else { pi[t] = 0; pj[t] = 0; }
  }
  unsigned long long gacc[PPL];
#pragma unroll
  for (int t = 0; t < PPL; ++t) gacc[t] = 0;

  const int64_t nbatch = (P.rows + RPW - 1) / RPW;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t nw = (int64_t)gridDim.x * kWarps;

  for (int64_t batch = gw; batch < nbatch; batch += nw) {
    const int64_t r = batch * RPW + slot;
    uint32_t y[4] = {0, 0, 0, 0};
    if (r < P.rows) {
      if (MODE == kModeInit) {
        const uint4 w = P.X[r * TPR + sub];
        y[0] = w.x; y[1] = w.y; y[2] = w.z; y[3] = w.w;
      } else if (r < P.heavy_rows) {
        unsigned long long* h = P.heavy_acc + (size_t)r * B + 4 * sub;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          y[l] = reduce(h[l], M);
          h[l] = 0;
        }
      } else {
        const uint32_t beg = P.rowptr[r], end = P.rowptr[r + 1];
        uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        uint32_t k = beg;
        for (; k + FE <= end; k += FE) {
#pragma unroll
          for (int u = 0; u < FE; ++u) {
            const int32_t c = __ldg(P.col + k + u);
            const uint32_t v = __ldg(P.val + k + u);
            const uint4 x = __ldg(P.X + (size_t)c * TPR + sub);
            a0 = mad_wide(v, x.x, a0);
            a1 = mad_wide(v, x.y, a1);
            a2 = mad_wide(v, x.z, a2);
            a3 = mad_wide(v, x.w, a3);
          }
          a0 = fold(a0, M); a1 = fold(a1, M); a2 = fold(a2, M); a3 = fold(a3, M);
        }
        for (; k < end; ++k) {
          const int32_t c = __ldg(P.col + k);
          const uint32_t v = __ldg(P.val + k);
          const uint4 x = __ldg(P.X + (size_t)c * TPR + sub);
          a0 = mad_wide(v, x.x, a0);
          a1 = mad_wide(v, x.y, a1);
          a2 = mad_wide(v, x.z, a2);
          a3 = mad_wide(v, x.w, a3);
        }
        y[0] = reduce(a0, M); y[1] = reduce(a1, M); y[2] = reduce(a2, M); y[3] = reduce(a3, M);
      }
    }
    // epilogue: scale, store, stage the Gram operands
    uint32_t gz[4], gu[4];
    if (r < P.rows) {
      const uint32_t s = P.scale[r];
      uint4 o;
      if (MODE == kModeOdd) {
        // z = y; U = d_r z
#pragma unroll
        for (int l = 0; l < 4; ++l) { gz[l] = y[l]; gu[l] = mulmod(y[l], s, M); }
        o = make_uint4(gu[0], gu[1], gu[2], gu[3]);
      } else if (MODE == kModeEven) {
        // w' = d_c t ; x' = d_c w'
        uint32_t xo[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          gz[l] = mulmod(y[l], s, M);
          gu[l] = gz[l];
          xo[l] = mulmod(gz[l], s, M);
        }
        o = make_uint4(xo[0], xo[1], xo[2], xo[3]);
      } else {
        // init: y = w; x = d_c w
        uint32_t xo[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) { gz[l] = y[l]; gu[l] = y[l]; xo[l] = mulmod(y[l], s, M); }
        o = make_uint4(xo[0], xo[1], xo[2], xo[3]);
      }
      P.Y[r * TPR + sub] = o;
    } else {
#pragma unroll
      for (int l = 0; l < 4; ++l) { gz[l] = 0; gu[l] = 0; }
    }
    if (P.S_out != nullptr) {
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        zs[warp][slot][4 * sub + l] = gz[l];
        us[warp][slot][4 * sub + l] = gu[l];
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < PPL; ++t) {
        if (lane + 32 * t < NP) {
          unsigned long long a = gacc[t];
#pragma unroll
          for (int rr = 0; rr < RPW; ++rr) {
            a = mad_wide(zs[warp][rr][pi[t]], us[warp][rr][pj[t]], a);
            if ((rr % FE) == FE - 1) a = fold(a, M);
          }
          gacc[t] = a;
        }
      }
      __syncwarp();
    }
  }

  if (P.S_out == nullptr) return;
  __syncthreads();
#pragma unroll
  for (int t = 0; t < PPL; ++t) {
    const int q = lane + 32 * t;
    if (q < NP) atomicAdd(&red[q], (unsigned long long)reduce(gacc[t], M));
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NP; q += kThreads) atomicAdd(&P.gram_acc[q], red[q]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = (atomicAdd(P.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // the last CTA: write the finished term (real pairs only) and reset
  const int b = P.b_real;
  const int npr = b * (b + 1) / 2;
  for (int q = threadIdx.x; q < npr; q += kThreads) {
    int i, j;
    pair_of(q, b, i, j);
    const int qb = i * B - i * (i - 1) / 2 + (j - i);
    P.S_out[q] = reduce(atomicAdd(&P.gram_acc[qb], 0ull), M);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < NP; q += kThreads) atomicExch(&P.gram_acc[q], 0ull);
  if (threadIdx.x == 0) atomicExch(P.counter, 0u);
}

// Heavy rows: one warp per chunk of kChunkNnz entries.  Lanes form RPW slots
// of TPR threads; slot s takes entries beg+s, beg+s+RPW, ...  The slot sums
// are combined with shuffles and added to heavy_acc with 64-bit atomics.
template <int B, int FE>
__global__ void __launch_bounds__(kThreads) chunk_kernel(ChunkParams P) {
  constexpr int TPR = B / 4;
  constexpr int RPW = 32 / TPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % TPR;
  const int slot = lane / TPR;
  const ModP M = P.M;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  for (int64_t ch = gw; ch < P.nchunks; ch += nw) {
    const uint32_t beg = P.chunk_begin[ch], end = P.chunk_end[ch];
    const uint32_t row = P.chunk_row[ch];
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    uint32_t k = beg + slot;
    for (; k + (FE - 1) * RPW < end; k += FE * RPW) {
#pragma unroll
      for (int u = 0; u < FE; ++u) {
        const uint32_t kk = k + u * RPW;
        const int32_t c = __ldg(P.col + kk);
        const uint32_t v = __ldg(P.val + kk);
        const uint4 x = __ldg(P.X + (size_t)c * TPR + sub);
        a0 = mad_wide(v, x.x, a0);
        a1 = mad_wide(v, x.y, a1);
        a2 = mad_wide(v, x.z, a2);
        a3 = mad_wide(v, x.w, a3);
      }
      a0 = fold(a0, M); a1 = fold(a1, M); a2 = fold(a2, M); a3 = fold(a3, M);
    }
    for (; k < end; k += RPW) {
      const int32_t c = __ldg(P.col + k);
      const uint32_t v = __ldg(P.val + k);
      const uint4 x = __ldg(P.X + (size_t)c * TPR + sub);
      a0 = mad_wide(v, x.x, a0);
      a1 = mad_wide(v, x.y, a1);
      a2 = mad_wide(v, x.z, a2);
      a3 = mad_wide(v, x.w, a3);
    }
    uint32_t y[4] = {reduce(a0, M), reduce(a1, M), reduce(a2, M), reduce(a3, M)};
#pragma unroll
    for (int off = TPR; off < 32; off <<= 1) {
#pragma unroll
      for (int l = 0; l < 4; ++l) y[l] = addmod(y[l], __shfl_xor_sync(0xffffffffu, y[l], off), M.p);
    }
    if (slot == 0) {
      unsigned long long* h = P.heavy_acc + (size_t)row * B + 4 * sub;
#pragma unroll
      for (int l = 0; l < 4; ++l) atomicAdd(&h[l], (unsigned long long)y[l]);
    }
  }
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

// ---------------------------------------------------------------- launchers
template <int B>
static int launch_pass_B(rr_krylov* kr, const PassParams& P, int mode) {
  const dim3 grid(kr->grid_pass), block(kThreads);
  cudaStream_t s = kr->mat->ctx->stream;
  if (kr->fold4) {
    if (mode == kModeInit) pass_kernel<B, kModeInit, 4><<<grid, block, 0, s>>>(P);
    else if (mode == kModeOdd) pass_kernel<B, kModeOdd, 4><<<grid, block, 0, s>>>(P);
    else pass_kernel<B, kModeEven, 4><<<grid, block, 0, s>>>(P);
  } else {
    if (mode == kModeInit) pass_kernel<B, kModeInit, 2><<<grid, block, 0, s>>>(P);
    else if (mode == kModeOdd) pass_kernel<B, kModeOdd, 2><<<grid, block, 0, s>>>(P);
    else pass_kernel<B, kModeEven, 2><<<grid, block, 0, s>>>(P);
  }
  RR_CUDA(cudaGetLastError());
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
  const dim3 grid(kr->grid_chunk), block(kThreads);
  cudaStream_t s = kr->mat->ctx->stream;
  if (kr->fold4) chunk_kernel<B, 4><<<grid, block, 0, s>>>(P);
  else chunk_kernel<B, 2><<<grid, block, 0, s>>>(P);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
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
static int occupancy_B(rr_krylov* kr, int* pass_blocks, int* chunk_blocks) {
  if (kr->fold4) {
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(pass_blocks, pass_kernel<B, kModeEven, 4>, kThreads, 0));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunk_blocks, chunk_kernel<B, 4>, kThreads, 0));
  } else {
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(pass_blocks, pass_kernel<B, kModeEven, 2>, kThreads, 0));
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunk_blocks, chunk_kernel<B, 2>, kThreads, 0));
  }
  return RR_OK;
}

int krylov_occupancy(rr_krylov* kr) {
  int pb = 1, cb = 1;
  switch (kr->B) {
    case 4: RR_TRY(occupancy_B<4>(kr, &pb, &cb)); break;
    case 8: RR_TRY(occupancy_B<8>(kr, &pb, &cb)); break;
    case 16: RR_TRY(occupancy_B<16>(kr, &pb, &cb)); break;
    case 32: RR_TRY(occupancy_B<32>(kr, &pb, &cb)); break;
    default: return fail(RR_EINVAL, "unsupported padded block width %d", kr->B);
  }
  const int sms = kr->mat->ctx->num_sms;
  kr->grid_pass = std::max(1, pb) * sms;
  kr->grid_chunk = std::max(1, cb) * sms;
  return RR_OK;
}

static PassParams base_params(rr_krylov* kr) {
  PassParams P;
  std::memset(&P, 0, sizeof(P));
  P.heavy_acc = kr->heavy_acc.ptr;
  P.gram_acc = kr->gram_acc.ptr;
  P.counter = kr->counter.ptr;
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
  P.scale = kr->dc.ptr;
  // S_0 goes to slot len - base; the caller publishes it (len += 1) later
  P.S_out = emit_s0 ? kr->S.ptr + (size_t)(kr->len - kr->base) * np : nullptr;
  return launch_pass(kr, P, kModeInit);
}

static int run_chunks(rr_krylov* kr, const DevCsr& A, const uint32_t* X) {
  if (A.nchunks == 0) return RR_OK;
  ChunkParams C;
  C.col = A.col.ptr;
  C.val = A.val.ptr;
  C.chunk_row = A.chunk_row.ptr;
  C.chunk_begin = A.chunk_begin.ptr;
  C.chunk_end = A.chunk_end.ptr;
  C.nchunks = A.nchunks;
  C.X = reinterpret_cast<const uint4*>(X);
  C.heavy_acc = kr->heavy_acc.ptr;
  C.M = kr->M;
  return launch_chunk(kr, C);
}

// ev (optional): four events recorded before pass 1, after pass 1, after the
// chunks of pass 2 and after pass 2.
int krylov_launch_application(rr_krylov* kr, cudaEvent_t* ev) {
  const int np = kr->b * (kr->b + 1) / 2;
  rr_matrix* mat = kr->mat;
  cudaStream_t s = mat->ctx->stream;
  uint32_t* x = kr->X[kr->cur].ptr;
  uint32_t* xn = kr->X[kr->cur ^ 1].ptr;
  if (ev) RR_CUDA(cudaEventRecord(ev[0], s));
  // pass 1: rows of A
  RR_TRY(run_chunks(kr, mat->A, x));
  PassParams P = base_params(kr);
  P.rowptr = mat->A.rowptr.ptr;
  P.col = mat->A.col.ptr;
  P.val = mat->A.val.ptr;
  P.rows = mat->A.rows;
  P.heavy_rows = mat->A.heavy_rows;
  P.X = reinterpret_cast<const uint4*>(x);
  P.Y = reinterpret_cast<uint4*>(kr->U.ptr);
  P.scale = kr->dr.ptr;
  P.S_out = kr->S.ptr + (size_t)(kr->len - kr->base) * np;
  RR_TRY(launch_pass(kr, P, kModeOdd));
  if (ev) RR_CUDA(cudaEventRecord(ev[1], s));
  // pass 2: rows of A^T
  RR_TRY(run_chunks(kr, mat->At, kr->U.ptr));
  if (ev) RR_CUDA(cudaEventRecord(ev[2], s));
  P.rowptr = mat->At.rowptr.ptr;
  P.col = mat->At.col.ptr;
  P.val = mat->At.val.ptr;
  P.rows = mat->At.rows;
  P.heavy_rows = mat->At.heavy_rows;
  P.X = reinterpret_cast<const uint4*>(kr->U.ptr);
  P.Y = reinterpret_cast<uint4*>(xn);
  P.scale = kr->dc.ptr;
  P.S_out = kr->S.ptr + (size_t)(kr->len + 1 - kr->base) * np;
  RR_TRY(launch_pass(kr, P, kModeEven));
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

// ---------------------------------------------------------------- matrix build
// Host preprocessing: degree-ordered renumbering of rows and columns, the
// transpose by counting sort (src/matrices.rs:734-778) and the chunk lists of
// heavy rows; then one upload.
namespace {

struct HostCsr {
  std::vector<uint32_t> ptr;
  std::vector<int32_t> col;
  std::vector<uint32_t> val;
  int64_t rows = 0, cols = 0;
};

std::vector<int32_t> degree_order(const std::vector<int64_t>& deg) {
  std::vector<int32_t> order(deg.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return deg[a] > deg[b]; });
  return order;
}

void transpose_host(const HostCsr& a, HostCsr& t) {
  t.rows = a.cols;
  t.cols = a.rows;
  t.ptr.assign(a.cols + 1, 0);
  for (int32_t c : a.col) t.ptr[c + 1]++;
  for (int64_t i = 0; i < a.cols; ++i) t.ptr[i + 1] += t.ptr[i];
  std::vector<uint32_t> next(t.ptr.begin(), t.ptr.end() - 1);
  t.col.resize(a.col.size());
  t.val.resize(a.val.size());
  for (int64_t r = 0; r < a.rows; ++r)
    for (uint32_t k = a.ptr[r]; k < a.ptr[r + 1]; ++k) {
      const uint32_t pos = next[a.col[k]]++;
      t.col[pos] = (int32_t)r;
      t.val[pos] = a.val[k];
    }
}

int upload_csr(const HostCsr& h, DevCsr& d, cudaStream_t s) {
  d.rows = h.rows;
  d.cols = h.cols;
  d.nnz = (int64_t)h.col.size();
  RR_TRY(d.rowptr.alloc(h.ptr.size()));
  RR_TRY(d.col.alloc(std::max<size_t>(h.col.size(), 1)));
  RR_TRY(d.val.alloc(std::max<size_t>(h.val.size(), 1)));
  RR_CUDA(cudaMemcpyAsync(d.rowptr.ptr, h.ptr.data(), h.ptr.size() * 4, cudaMemcpyHostToDevice, s));
  if (!h.col.empty()) {
    RR_CUDA(cudaMemcpyAsync(d.col.ptr, h.col.data(), h.col.size() * 4, cudaMemcpyHostToDevice, s));
    RR_CUDA(cudaMemcpyAsync(d.val.ptr, h.val.data(), h.val.size() * 4, cudaMemcpyHostToDevice, s));
  }
  // heavy rows form a prefix (rows are sorted by decreasing degree)
  int64_t heavy = 0;
  while (heavy < h.rows && (int64_t)(h.ptr[heavy + 1] - h.ptr[heavy]) > kHeavyDegree) ++heavy;
  d.heavy_rows = heavy;
  struct Chunk { uint32_t row, beg, end, key; };
  std::vector<Chunk> chunks;
  for (int64_t r = 0; r < heavy; ++r)
    for (uint32_t k = h.ptr[r]; k < h.ptr[r + 1]; k += (uint32_t)kChunkNnz) {
      const uint32_t e = std::min<uint32_t>(h.ptr[r + 1], k + (uint32_t)kChunkNnz);
      chunks.push_back({(uint32_t)r, k, e, (uint32_t)h.col[k]});
    }
  // chunks that gather the same region of the input block run together
  std::stable_sort(chunks.begin(), chunks.end(), [](const Chunk& a, const Chunk& b) { return a.key < b.key; });
  d.nchunks = (int64_t)chunks.size();
  if (d.nchunks) {
    std::vector<uint32_t> cr(d.nchunks), cb(d.nchunks), ce(d.nchunks);
    for (int64_t i = 0; i < d.nchunks; ++i) { cr[i] = chunks[i].row; cb[i] = chunks[i].beg; ce[i] = chunks[i].end; }
    RR_TRY(d.chunk_row.alloc(d.nchunks));
    RR_TRY(d.chunk_begin.alloc(d.nchunks));
    RR_TRY(d.chunk_end.alloc(d.nchunks));
    RR_CUDA(cudaMemcpyAsync(d.chunk_row.ptr, cr.data(), d.nchunks * 4, cudaMemcpyHostToDevice, s));
    RR_CUDA(cudaMemcpyAsync(d.chunk_begin.ptr, cb.data(), d.nchunks * 4, cudaMemcpyHostToDevice, s));
    RR_CUDA(cudaMemcpyAsync(d.chunk_end.ptr, ce.data(), d.nchunks * 4, cudaMemcpyHostToDevice, s));
    RR_CUDA(cudaStreamSynchronize(s));  // host vectors die at scope end
  }
  RR_CUDA(cudaStreamSynchronize(s));
  return RR_OK;
}

}  // namespace

int matrix_build(rr_ctx* ctx, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col, const uint32_t* val,
                 uint32_t p, rr_matrix* mat) {
  const int64_t nnz = rowptr[m];
  std::vector<int64_t> rdeg(m), cdeg(n, 0);
  for (int64_t r = 0; r < m; ++r) rdeg[r] = rowptr[r + 1] - rowptr[r];
  for (int64_t k = 0; k < nnz; ++k) cdeg[col[k]]++;
  mat->max_row_nnz = m ? *std::max_element(rdeg.begin(), rdeg.end()) : 0;
  mat->max_col_nnz = n ? *std::max_element(cdeg.begin(), cdeg.end()) : 0;
  mat->rowperm = degree_order(rdeg);
  mat->colperm = degree_order(cdeg);
  std::vector<int32_t> inv_col(n);
  for (int64_t c = 0; c < n; ++c) inv_col[mat->colperm[c]] = (int32_t)c;

  HostCsr A;
  A.rows = m;
  A.cols = n;
  A.ptr.resize(m + 1);
  A.col.resize(nnz);
  A.val.resize(nnz);
  A.ptr[0] = 0;
  std::vector<std::pair<int32_t, uint32_t>> tmp;
  for (int64_t rp = 0; rp < m; ++rp) {
    const int64_t r = mat->rowperm[rp];
    tmp.clear();
    for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k) tmp.push_back({inv_col[col[k]], val[k]});
    std::sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    uint32_t o = A.ptr[rp];
    for (auto& e : tmp) { A.col[o] = e.first; A.val[o] = e.second; ++o; }
    A.ptr[rp + 1] = o;
  }
  HostCsr At;
  transpose_host(A, At);
  cudaStream_t s = ctx->stream;
  RR_TRY(upload_csr(A, mat->A, s));
  RR_TRY(upload_csr(At, mat->At, s));
  RR_TRY(mat->d_colperm.alloc(std::max<int64_t>(n, 1)));
  RR_CUDA(cudaMemcpyAsync(mat->d_colperm.ptr, mat->colperm.data(), n * 4, cudaMemcpyHostToDevice, s));
  RR_CUDA(cudaStreamSynchronize(s));
  (void)p;
  return RR_OK;
}

}  // namespace rr
