// krylov_params.h -- launch parameters of the Krylov pass kernels (krylov.cu),
// shared with the batched engine (batch.cu).
#pragma once
#include "rr_internal.h"

namespace rr {

// kModeGram: no output block; the Gram term of the rows of X with
// gz = redc(x * scale) and gu = gram_sym ? gz : x (a Gram pass after a pass
// that did not compute its term).
enum PassMode { kModeInit = 0, kModeOdd = 1, kModeEven = 2, kModeGram = 3 };

struct PassParams {
  const uint32_t* rowptr;
  const uint2* cv;          // packed (column, value)
  int64_t rows;
  int64_t heavy_rows;
  // rows >= tail_begin have no entries (the end of the degree order): their
  // output rows are zero and they add nothing to the Gram term (0 = no tail)
  int64_t tail_begin;
  const uint4* X;           // gathered block [cols][B/4]   (kModeInit: w [rows][B/4])
  uint4* Y;                 // output block   [rows][B/4]
  const uint32_t* scale;    // odd: d_r R^2; even: d_c R^2; init: d_c R   (all mod p)
  const uint32_t* scale2;   // even: d_c R
  unsigned long long* heavy_acc;  // [heavy_rows][B]
  unsigned long long* gram_acc;   // [replicas][segments][B(B+1)/2]; CTA c adds into replica c % replicas
  int64_t gram_stride;            // words per replica (segments * B(B+1)/2)
  int replicas;                   // 1..kGramReplicas
  unsigned int* counter;
  uint32_t* S_out;          // finished term, real pairs; nullptr = do not emit (unless term_ctr)
  // Device-indexed output (replayable launches, e.g. in a CUDA graph): the
  // last CTA writes the term to (*S_ptr) + (*term_ctr) * pairs and advances
  // *term_ctr.  nullptr = S_out as given.
  unsigned int* term_ctr;
  uint32_t* const* S_ptr;
  // Batched, slot-per-term mode: the Gram partials of segment s for this
  // launch's term go to gram_all + seg_G_off[s] + term * NP with atomics and
  // nothing is finished in the kernel (batch_finalize_kernel does that once
  // per group of finished sequences).  nullptr = accumulators + last CTA.
  unsigned long long* gram_all;
  const int64_t* seg_G_off;
  uint32_t gram_mul;        // factor applied to the finished term
  uint32_t w4, w5, w6;      // 2^32, 2^40, 2^48 mod p (limb weights of the tensor-core Gram)
  int b_real;
  int gram_sym;             // kModeGram: both Gram factors scaled
  ModP M;
  // Batched mode (many matrices stacked block-diagonally, each padded to a
  // multiple of 32 rows): batch_seg[batch] is the matrix of a row batch.  Warps
  // then take contiguous runs of batches from batch_begin on, and Gram terms
  // go to gram_acc[seg][NP] and to S_all + seg_S_off[seg] + term * np.
  const int32_t* batch_seg; // nullptr: one matrix
  const int32_t* runs;      // batched: warp w takes batches [runs[w], runs[w+1]); nullptr = equal counts
  int64_t batch_begin;
  int32_t seg_begin, seg_end;
  uint32_t* S_all;
  const int64_t* seg_S_off;
  int64_t term;
};

struct ChunkParams {
  const uint2* cv;
  const uint32_t* chunk_row;
  const uint32_t* chunk_begin;
  const uint32_t* chunk_end;
  int64_t nchunks;
  const uint4* X;
  unsigned long long* heavy_acc;
  unsigned int* next;  // chunk dispenser [next ticket, warps done]: zero at launch, rewound by the last warp
  ModP M;
};

// The persistent batched loop (one cooperative launch per batch phase):
// applications [t_begin, t_end), odd pass (rows of A: X[cur] -> U) then even
// pass (rows of A^T: U -> X[cur ^ 1]) per application, separated by grid
// barriers that give up after limit_ns and set *error.
struct PersistParams {
  PassParams odd, even;     // everything but X, Y and term
  uint4* X[2];
  uint4* U;
  int cur0;
  int64_t t_begin, t_end;
  unsigned int* bar;        // [2]: arrivals, generation (zero before the first launch)
  int* error;
  uint64_t limit_ns;
};
// lpt: lanes of the block per thread (4 or 8; persistent_lane_options).
int launch_persistent_raw(cudaStream_t s, int B, int fold4, int grid, int lpt, PersistParams& Q);
// Largest co-resident CTAs per SM of the persistent kernel (sets its shared-memory limit).
int persistent_blocks_per_sm(int B, int fold4, int lpt, int* blocks);
// The lanes-per-thread variants of the persistent kernel at padded width B
// (into opts[2]); returns their count.
int persistent_lane_options(int B, int* opts);
// Cooperative launch of `grid` CTAs passing `rounds` barriers that wait for `expected` arrivals.
int launch_barrier_check(cudaStream_t s, int grid, unsigned int* bar, int* error, uint64_t limit_ns,
                         unsigned int expected, int rounds);

// Finish the slot-per-term Gram sums of segments [seg_begin, seg_end):
// S_all[seg_S_off[s] + t * pairs + q] = reduce(gram_all[seg_G_off[s] + t * NP + pair q]) * (t odd ? R : 1).
int launch_batch_finalize(cudaStream_t s, const unsigned long long* gram_all, const int64_t* d_seg_G_off,
                          uint32_t* S_all, const int64_t* d_seg_S_off, const int64_t* d_seg_terms, int seg_begin,
                          int seg_end, int64_t max_terms, int b, int B, const ModP& M);
// Launch one pass kernel for padded width B on stream s (grid = CTAs).
int launch_pass_raw(cudaStream_t s, int B, int fold4, int grid, const PassParams& P, int mode);
// CTAs per SM of the pass kernel for padded width B (also sets its shared-memory limit).
int pass_blocks_per_sm(int B, int fold4, int* blocks);
// Rows per warp batch for padded width B with lpt lanes per thread (0: the
// default shape of the pass kernels).
int rows_per_batch(int B, int lpt = 0);
// Warps per CTA of the pass kernel.
constexpr int kPassWarps = 8;
// Copies of the Gram accumulators: CTAs spread their 64-bit atomics over
// this many copies so that no L2 slice serialises all of them.
constexpr int kGramReplicas = 8;

}  // namespace rr
