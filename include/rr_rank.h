/* rr_rank.h -- C ABI of the B200 block-Wiedemann rank engine (librr_b200.so).
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point returns
 * an rr_status; on failure rr_last_error() gives a message for the calling
 * thread.  Handles are thread-compatible (one thread at a time per handle).
 * Host arrays passed in are copied; the caller keeps ownership.
 *
 * Reference call surface replaced (paths in wilthoma/rust_rank):
 *   src/vectorstream.rs:7-10      trait VectorStream { next, fill_status }
 *   src/vectorstream.rs:46,225    NormalVectorStream::new / SimdVectorStream2::new
 *   src/main.rs:88-216            main_loop_s_mt2 (sequence S_t = V^T B^t V)
 *   src/sigma_basis.rs:9-54       PM_Basis (minimal generator)
 *   src/sigma_basis.rs:71-152     analyze_pm_basis -> src/blockbmtest.rs:574-599
 *   src/wdm_files.rs:22-210       load_wdm_file_sym / save_wdm_file_sym
 *   src/matrices.rs:662-732       CsrMatrix::load_csr_matrix_from_sms
 */
#ifndef RR_RANK_H
#define RR_RANK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rr_status {
  RR_OK = 0,
  RR_EINVAL = 1,      /* bad argument (sizes, pointers, indices out of range) */
  RR_EPRIME = 2,      /* modulus not supported (must be a prime 2 < p < 2^31) */
  RR_ENOMEM = 3,      /* device or host allocation failed / admission refused */
  RR_ECUDA = 4,       /* CUDA runtime error */
  RR_ETIMEOUT = 5,    /* a bounded device-side wait gave up */
  RR_EIO = 6,         /* file could not be read / written / parsed */
  RR_ESTATE = 7,      /* call not valid in the handle's current state */
  RR_EUNSUPPORTED = 8 /* valid request outside what this build implements */
} rr_status;

typedef struct rr_ctx_s rr_ctx;       /* one device + one CUDA stream */
typedef struct rr_matrix_s rr_matrix; /* a sparse matrix resident on the device */
typedef struct rr_krylov_s rr_krylov; /* Krylov state of one block of vectors */
typedef struct rr_batch_s rr_batch;   /* many matrices stacked for one Krylov launch per pass */

const char* rr_status_string(int status);
/* Message of the last failed call on this thread ("" if none). */
const char* rr_last_error(void);
/* Library version string. */
const char* rr_version(void);

/* ---------------------------------------------------------------- context */
int rr_ctx_create(int device, rr_ctx** out);
int rr_ctx_destroy(rr_ctx* ctx);
/* The cudaStream_t (as void*) all work of this context is queued on. */
void* rr_ctx_stream(rr_ctx* ctx);
int rr_ctx_synchronize(rr_ctx* ctx);
/* PM-basis contractions of this context (the leaf residual updates and the
 * block-basis products): on the int8 tensor cores by byte limbs (enable = 1,
 * the default, for b <= 16) or on the CUDA cores with 64-bit sums (0).  The
 * generator is the same bit for bit; this selects the path, e.g. to compare
 * them.  No counterpart in the reference. */
int rr_ctx_set_pm_tensor_cores(rr_ctx* ctx, int32_t enable);

/* ---------------------------------------------------------------- checks */
/* RR_OK when p is a prime with 2 < p < 2^31, the range the engine computes
 * in exactly (the reference's overflow check, src/matrices.rs:861-870 and
 * src/main.rs:481-489, rejects most of these primes for its u32 path; this
 * engine does not accumulate lazily in 32 bits and has no such limit). */
int rr_prime_check(uint32_t p);

/* ---------------------------------------------------------------- matrix */
/* Upload an m x n CSR matrix over F_p.  rowptr[m+1] (int64, rowptr[0] = 0,
 * non-decreasing), col[nnz] in [0, n), val[nnz] in [0, p) -- the reference's
 * CsrMatrix<u32> after load (src/matrices.rs:53-64, 662-732).  The device
 * copy is reordered by degree and transposed once here
 * (src/matrices.rs:734-778).  Requires nnz < 2^32. */
int rr_matrix_create(rr_ctx* ctx, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                     const uint32_t* val, uint32_t p, rr_matrix** out);
int rr_matrix_destroy(rr_matrix* mat);
/* src/matrices.rs:842-860 max_nnzs. */
int rr_matrix_max_nnzs(const rr_matrix* mat, int64_t* max_row_nnz, int64_t* max_col_nnz);
int rr_matrix_shape(const rr_matrix* mat, int64_t* m, int64_t* n, int64_t* nnz);

/* ---------------------------------------------------------------- Krylov */
/* Start (or resume) the Krylov sequence of B = D_c A^T D_r A D_c
 * (src/main.rs:522-526) for a block of b vectors, 1 <= b <= 32.
 * row_precond[m], col_precond[n]: diagonal preconditioners in [1, p).
 * curv[b][n] (vector-major, like Vec<Vec<u32>>): the current block w_k
 * (= V when seq_len == 0).  seq_len: number of sequence terms already
 * computed (0 for a fresh start; 1 + 2k after k applications of B). */
int rr_krylov_create(rr_matrix* mat, int32_t b, const uint32_t* row_precond, const uint32_t* col_precond,
                     const uint32_t* curv, int64_t seq_len, rr_krylov** out);
int rr_krylov_destroy(rr_krylov* kr);

/* main_loop_s_mt2 (src/main.rs:88-216) fed by VectorStream::next
 * (src/vectorstream.rs:58-69): extend the sequence up to max_nlen terms
 * (a fresh start also emits S_0, so it ends at max_nlen + 1 terms; each
 * application of B adds two terms).  seq is a HOST array
 * [b(b+1)/2][seq_stride]; entries [current length, new length) are written,
 * pair ii enumerating (i <= j) row-major as in src/main.rs:113-127.
 * *new_len receives the new sequence length. */
int rr_krylov_advance(rr_krylov* kr, int64_t max_nlen, uint32_t* seq, int64_t seq_stride, int64_t* new_len);

/* rr_krylov_advance with the progress report of src/main.rs:57-85
 * (report_progress) and the timed checkpoint hook of src/main.rs:186-202: the
 * terms are computed in chunks of chunk_terms (<= 1: one chunk) and after each
 * chunk, whose terms are already in seq, fn(user, len, target_len, elapsed_s,
 * terms_per_s) is called (fn may be NULL); terms_per_s is the rate since the
 * previous report.  A non-zero return from fn stops after that chunk (the
 * caller saves its .wdm checkpoint and calls again to continue); *new_len is
 * the length reached. */
typedef int (*rr_progress_fn)(void* user, int64_t len, int64_t target_len, double elapsed_s, double terms_per_s);
int rr_krylov_advance_report(rr_krylov* kr, int64_t max_nlen, uint32_t* seq, int64_t seq_stride,
                             int64_t chunk_terms, rr_progress_fn fn, void* user, int64_t* new_len);
/* VectorStream::fill_status (src/vectorstream.rs:7-10): a one-line status of
 * the stream (terms queued, whether device work is in flight) into buf[cap]. */
int rr_krylov_fill_status(rr_krylov* kr, char* buf, int64_t cap);

/* Device-resident stepping for benchmarks and pipelines: queue n_apps
 * applications of B (2 terms each) on the context stream without any host
 * synchronisation.  Terms stay in the handle's device sequence buffer. */
int rr_krylov_step_device(rr_krylov* kr, int64_t n_apps);
/* Copy terms [from, to) of the device sequence buffer into the host array
 * seq[b(b+1)/2][seq_stride] (synchronises the context stream). */
int rr_krylov_fetch(rr_krylov* kr, int64_t from, int64_t to, uint32_t* seq, int64_t seq_stride);
/* Current sequence length (terms computed so far, including queued work). */
int rr_krylov_length(const rr_krylov* kr, int64_t* len);
/* The current block w_k as curv[b][n] (host, original column order). */
int rr_krylov_get_curv(rr_krylov* kr, uint32_t* curv);
/* Algorithmic bytes of one application of B (both SpMMs: CSR read once,
 * dense blocks read and written once), for bandwidth reporting. */
int rr_krylov_bytes_per_application(const rr_krylov* kr, double* bytes);
/* The same split by pass: [0] rows of A (8 nnz + 4 (m+1) + 4 b (n + m)),
 * [1] rows of A^T (8 nnz + 4 (n+1) + 4 b (m + n)). */
int rr_krylov_phase_bytes(const rr_krylov* kr, double* bytes2);
/* Like rr_krylov_step_device, but records CUDA events on the context stream
 * around each phase and returns the mean device time per application in ms:
 * ms3[0] pass over A (with its chunks), ms3[1] chunks of A^T, ms3[2] pass
 * over A^T (synchronises). */
int rr_krylov_profile(rr_krylov* kr, int64_t n_apps, double* ms3);
/* Number of kernels this handle has launched so far. */
int rr_krylov_launch_count(const rr_krylov* kr, int64_t* count);

/* ---------------------------------------------------------------- generator */
/* PM_Basis (src/sigma_basis.rs:9-54): minimal matrix generator of the
 * symmetric b x b sequence seq[b(b+1)/2][seq_stride] (nlen valid terms).
 * d is rounded up to a power of two and must be < nlen.  Outputs (host):
 * M[2b][2b][d+1] and delta[2b], identical to the reference's result computed
 * exactly mod p.  Products are NTT products mod p when p - 1 is divisible by
 * the transform length (p = 2013265921 = 15*2^27+1 up to d = 2^26), else
 * exact integer products over two or three NTT primes combined by CRT and
 * reduced mod p (src/poly_mat_mul.rs:240-256), up to d = 2^23. */
int rr_pm_basis(rr_ctx* ctx, const uint32_t* seq, int64_t seq_stride, int32_t b, int64_t nlen, int64_t d,
                uint32_t p, uint32_t* M, int64_t* delta);
/* No counterpart in the reference.  PM-basis of a short sequence for callers
 * that cannot allocate device memory: runtimes that hand all device memory to
 * their own pool allocator (a cudaMalloc from inside them would fail or
 * fragment the pool), and latency-critical loops where cudaMalloc's implicit
 * device synchronisation is not acceptable.  Same result as rr_pm_basis, but
 * every pointer is DEVICE memory owned by the caller: d_seq[b(b+1)/2][seq_stride]
 * (nlen valid terms), d_M[2b][2b][d'+1] and d_delta[2b] (d' = d rounded up to a
 * power of two).  Limits: 1 <= b <= 16 and d' <= 32 (RR_EINVAL beyond them).
 * The work is queued on `stream` (a cudaStream_t; NULL = legacy default) and
 * the call returns without waiting; outputs are ready when the stream gets
 * there.  A device-side failure cannot be returned by this asynchronous call:
 * it leaves every d_delta entry at INT64_MIN (exact arithmetic rules it out;
 * it would mean a fault in the library).  Scratch is one fixed 338,176-byte
 * __device__ array inside the library, present on every GPU that loads it
 * until the process exits; the first call on a device looks up its address
 * and sets a kernel attribute (make that first call before any stream
 * capture; after cudaDeviceReset the looked-up address is stale and the entry
 * point must not be called again in that process).  All calls share that
 * array and it keeps the last call's contents: calls whose work can overlap
 * on the GPU (different streams, different host threads) race and must be
 * serialised by the caller. */
int rr_pm_basis_short_noalloc(const uint32_t* d_seq, int64_t seq_stride, int32_t b, int64_t nlen, int64_t d,
                              uint32_t p, uint32_t* d_M, int64_t* d_delta, void* stream);
/* analyze_pm_basis + analyze_min_generators (src/sigma_basis.rs:71-152,
 * src/blockbmtest.rs:574-599): rank = b*(k-3) + rank(P[k-1]) + rank(P[0]).
 * M[2b][2b][len].  RR_ESTATE when k < 3 (no estimate). */
int rr_rank_from_basis(const uint32_t* M, const int64_t* delta, int32_t b, int64_t len, uint32_t p,
                       int64_t* rank);

/* is_generating_poly (src/blockbmtest.rs:445-461): *is_gen = 1 iff for every
 * l in [0, N - k) the matrix sum_{i<k} seq[l+i] * poly[i] is zero mod p.
 * poly [k][n][n], seq [N][n][n], row-major, entries in [0, p).  N < k is
 * RR_EINVAL (the reference's range 0..N-k has no meaning there).  Host code,
 * spread over the host's threads. */
int rr_is_generating_poly(const uint32_t* poly, int64_t k, const uint32_t* seq, int64_t N, int32_t n, uint32_t p,
                          int32_t* is_gen);

/* Scalar Berlekamp-Massey, the call surface of block_berlekamp_massey at
 * block width 1 (src/block_berlekamp_massey.rs:104-131, which hands seq[0] to
 * bubblemath 0.1.2's linear_recurrence::berlekamp_massey; that crate is not
 * part of the reference tree, so its output convention is not pinned here).
 * Returns Massey's connection polynomial of the shortest linear recurrence of
 * seq[0..n): conn[0] = 1, conn[0..L], sum_{i=0..L} conn[i] seq[j-i] = 0 mod p
 * for L <= j < n.  conn needs room for n + 1 entries.  Host code. */
int rr_berlekamp_massey(const uint32_t* seq, int64_t n, uint32_t p, uint32_t* conn, int64_t* L);

/* rr_pm_basis for `count` sequences with the same b, d and p, solved in
 * lockstep on the device (one launch per step of the recursion for all of
 * them); seqs[z] is [b(b+1)/2][seq_strides[z] >= nlen], M[z] and delta[z] as
 * for rr_pm_basis.  Each result equals rr_pm_basis on that sequence alone. */
int rr_pm_basis_batch(rr_ctx* ctx, int32_t count, const uint32_t* const* seqs, const int64_t* seq_strides, int32_t b,
                      int64_t nlen, int64_t d, uint32_t p, uint32_t* const* M, int64_t* const* delta);

/* Whole pipeline (src/main.rs:463-606): sequence length rule of
 * src/main.rs:497-504 when max_nlen == 0, Krylov sequence, PM-basis with
 * d = largest power of two <= length, rank readout. */
int rr_rank(rr_matrix* mat, int32_t b, const uint32_t* row_precond, const uint32_t* col_precond,
            const uint32_t* V, int64_t max_nlen, int64_t* rank);

/* ---------------------------------------------------------------- batches */
/* Many matrices (one per degree of a graph complex; the reference runs them
 * one main.rs invocation each, commands.txt) ranked together.  Matrix i is
 * m[i] x n[i] CSR (rowptr[i][m[i]+1], col[i], val[i] reduced mod p) with its
 * preconditioners and V[i] ([b][n[i]]).  Every matrix gets the sequence
 * length rule of src/main.rs:497-504 and the same sequence, generator and
 * rank as rr_rank on it alone.  The batch is copied at create time. */
int rr_batch_create(rr_ctx* ctx, int32_t nmat, const int64_t* m, const int64_t* n, const int64_t* const* rowptr,
                    const int32_t* const* col, const uint32_t* const* val, uint32_t p, int32_t b,
                    const uint32_t* const* row_precond, const uint32_t* const* col_precond,
                    const uint32_t* const* V, rr_batch** out);
int rr_batch_destroy(rr_batch* batch);
/* All Krylov sequences: S_0 for every matrix, then one persistent
 * cooperative launch per phase (the applications between two sequence ends)
 * that runs both passes of every application with grid-wide barriers between
 * them, all captured into one CUDA graph.  RR_ETIMEOUT when a barrier wait
 * gave up (2 s).  Once per batch. */
int rr_batch_krylov(rr_batch* batch);
/* Sequence of matrix i: *len = its length; seq [b(b+1)/2][seq_stride >= len]
 * (src/main.rs:164-175 order), or NULL to query the length only. */
int rr_batch_sequence(rr_batch* batch, int32_t i, uint32_t* seq, int64_t seq_stride, int64_t* len);
/* Generators and ranks of all matrices (runs rr_batch_krylov first when it
 * has not run), `workers` generators in flight on streams of their own.
 * ranks[nmat] in the caller's order; RR_ESTATE as rr_rank_from_basis. */
int rr_batch_ranks(rr_batch* batch, int32_t workers, int64_t* ranks);
/* Launch shapes the batch's autotuner picked: the Krylov loop has one phase
 * per distinct set of running matrices (phase k covers applications
 * apps_from[k] .. apps_from[k+1]-1); ctas[k] is the grid of its persistent
 * launch, chosen at create time together with the block shape
 * (rr_batch_tuning_shape) by timing every shape with 1..(co-resident maximum)
 * CTAs per SM.  Call with NULL arrays to get the phase count; *nphases gives
 * the room of the arrays. */
int rr_batch_tuning(const rr_batch* batch, int32_t* nphases, int32_t* ctas, int64_t* apps_from);
/* The block shape the autotuner picked per phase (beside its grid, see
 * rr_batch_tuning): lanes of the block each thread owns (4 or 8) and, from
 * it, the rows a warp walks together (32 * lanes / padded width).  Call with
 * NULL arrays to get the phase count. */
int rr_batch_tuning_shape(const rr_batch* batch, int32_t* nphases, int32_t* lanes_per_thread, int32_t* rows_per_warp);
/* Stacked sizes: rows and columns with padding, nonzeros, applications of
 * B of the longest sequence. */
int rr_batch_info(const rr_batch* batch, int64_t* total_rows, int64_t* total_cols, int64_t* total_nnz,
                  int64_t* max_apps);
/* Check of the device-side grid barrier the batch's persistent Krylov launch
 * uses (no counterpart in the reference): a cooperative launch of `ctas` CTAs
 * passes `rounds` barriers that each wait for `expected` arrivals, giving up
 * after limit_s seconds (0 < limit_s <= 10).  *timed_out = 1 when a wait gave
 * up (expected > ctas makes every wait run out), 0 otherwise; the context
 * stays usable either way.  ctas must fit on the device at once. */
int rr_device_barrier_check(rr_ctx* ctx, int32_t ctas, int32_t expected, int32_t rounds, double limit_s,
                            int32_t* timed_out);

/* ---------------------------------------------------------------- serving */
/* A rank service: requests (one matrix each, with its preconditioners and V)
 * are submitted as they arrive and run concurrently.  A request is admitted
 * when its device footprint fits hbm_budget and fewer than max_active
 * requests are resident; its matrix and Krylov state stay on the device while
 * the scheduler interleaves chunks of chunk_apps applications of B of all
 * running requests over `lanes` streams; when its sequence is complete a
 * worker thread solves the generator and reads off the rank, and its memory
 * admits the next requests.  Each request gets exactly the rank rr_rank
 * gives on the same inputs.  The reference has no service: it ranks one
 * matrix per run of src/main.rs:254-639 (commands.txt). */
typedef struct rr_server_s rr_server;
typedef struct rr_server_config {
  int32_t b;           /* block width of every request */
  uint32_t p;          /* prime */
  int32_t lanes;       /* Krylov streams (0: 4) */
  int32_t workers;     /* loader / generator threads (0: 4) */
  int32_t max_active;  /* requests resident at once (0: 64) */
  int64_t chunk_apps;  /* applications of B per scheduling quantum (0: 64) */
  uint64_t hbm_budget; /* device bytes the resident requests may hold (0: 80% of free memory) */
} rr_server_config;
int rr_server_create(int device, const rr_server_config* cfg, rr_server** out);
/* Copies the request; *id identifies it.  RR_ENOMEM when it alone exceeds the budget. */
int rr_server_submit(rr_server* server, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                     const uint32_t* val, const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* V,
                     uint64_t* id);
/* Waits for request id (timeout_s < 0: no limit; RR_ETIMEOUT when it runs out);
 * *rank as rr_rank, *latency_ms = submit to completion (may be NULL). */
int rr_server_wait(rr_server* server, uint64_t id, double timeout_s, int64_t* rank, double* latency_ms);
/* Requests submitted and completed, latency percentiles of the completed
 * ones and completions per second between the first submit and the last completion. */
int rr_server_stats(rr_server* server, int64_t* submitted, int64_t* completed, double* p50_ms, double* p99_ms,
                    double* ranks_per_s);
int rr_server_destroy(rr_server* server);

/* ---------------------------------------------------------------- several GPUs */
/* No counterpart in the reference (it ranks one matrix per run,
 * src/main.rs:254-639).  Matrices are independent, so the batched and served
 * modes shard by matrix: each matrix is placed whole on one GPU by its device
 * footprint and only its rank comes back; no collective, no peer memory. */

/* Device bytes a matrix of this shape and its Krylov state hold while
 * resident (both CSR copies, blocks, preconditioner forms, sequence of the
 * length rule of src/main.rs:497-504), the figure admission and placement use. */
int rr_footprint(int64_t m, int64_t n, int64_t nnz, int32_t b, uint64_t* bytes);
/* The placement rule (host only): items in decreasing footprint order, each
 * on the device with the most room left (dev_free[d] minus what it already
 * got; ties: lowest index).  device_of[nitems] receives device indices into
 * dev_free; dev_load[ndev] (may be NULL) the bytes placed per device.
 * RR_ENOMEM when an item fits on no device. */
int rr_place_by_footprint(int32_t nitems, const uint64_t* footprint, int32_t ndev, const uint64_t* dev_free,
                          int32_t* device_of, uint64_t* dev_load);

/* One rank service (rr_server_*) per listed device (a device may be listed
 * more than once: several services share it).  A submitted request goes to
 * the service with the most budget left after the requests it holds and
 * follows rr_server's path there, so its rank equals rr_rank's. */
typedef struct rr_fleet_s rr_fleet;
int rr_fleet_create(const int32_t* devices, int32_t ndev, const rr_server_config* cfg, rr_fleet** out);
int rr_fleet_submit(rr_fleet* fleet, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                    const uint32_t* val, const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* V,
                    uint64_t* id);
int rr_fleet_wait(rr_fleet* fleet, uint64_t id, double timeout_s, int64_t* rank, double* latency_ms);
/* The device request id was placed on. */
int rr_fleet_device_of(rr_fleet* fleet, uint64_t id, int32_t* device);
/* rr_server_stats over all services: latency percentiles of all completed
 * requests, completions per second from the first submit to the last completion. */
int rr_fleet_stats(rr_fleet* fleet, int64_t* submitted, int64_t* completed, double* p50_ms, double* p99_ms,
                   double* ranks_per_s);
int rr_fleet_destroy(rr_fleet* fleet);

/* rr_batch_ranks over several devices: the matrices (arguments as for
 * rr_batch_create) are placed by rr_place_by_footprint on 80% of each
 * device's free memory (shared evenly by repeated entries), each device runs
 * one batch of its matrices on a host thread of its own, and ranks[nmat]
 * come back in the caller's order; device_of[nmat] (may be NULL) receives
 * the device of each matrix.  Each rank equals rr_rank's on that matrix. */
int rr_batch_ranks_multi(const int32_t* devices, int32_t ndev, int32_t nmat, const int64_t* m, const int64_t* n,
                         const int64_t* const* rowptr, const int32_t* const* col, const uint32_t* const* val,
                         uint32_t p, int32_t b, const uint32_t* const* row_precond, const uint32_t* const* col_precond,
                         const uint32_t* const* V, int32_t workers, int64_t* ranks, int32_t* device_of);

/* ---------------------------------------------------------------- files */
/* .wdm checkpoint (src/wdm_files.rs:10-19): header "m n p Nlen num_v", then
 * row_precond, col_precond, num_v lines of v, num_v lines of curv and
 * num_v(num_v+1)/2 lines of sequence terms. */
int rr_wdm_save(const char* path, int64_t m, int64_t n, uint32_t p, int32_t b, const uint32_t* row_precond,
                const uint32_t* col_precond, const uint32_t* v, const uint32_t* curv, const uint32_t* seq,
                int64_t seq_stride, int64_t nlen);
/* Two-phase load: call with NULL arrays to read the header into m, n, p, b,
 * nlen; then again with arrays sized row_precond[m], col_precond[n],
 * v[b][n], curv[b][n], seq[b(b+1)/2][seq_stride >= nlen]. */
int rr_wdm_load(const char* path, int64_t* m, int64_t* n, uint32_t* p, int32_t* b, int64_t* nlen,
                uint32_t* row_precond, uint32_t* col_precond, uint32_t* v, uint32_t* curv, uint32_t* seq,
                int64_t seq_stride);
/* SMS text matrix (src/matrices.rs:662-732): "m n M" header then 1-based
 * "i j v" triplets, values reduced mod p.  Two-phase like rr_wdm_load:
 * rowptr[m+1], col[nnz], val[nnz]. */
int rr_sms_load(const char* path, uint32_t p, int64_t* m, int64_t* n, int64_t* nnz, int64_t* rowptr,
                int32_t* col, uint32_t* val);

#ifdef __cplusplus
}
#endif
#endif /* RR_RANK_H */
