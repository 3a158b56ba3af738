// batch.cu -- many matrices in one Krylov launch, then concurrent generators.
//
// The matrices of a batch (graph complexes give one per degree) are stacked
// block-diagonally: every matrix keeps its own degree order, its row block of
// A (and of A^T) is padded to a multiple of 32 rows so that no warp batch and
// no 32-row tensor-core tile straddles two matrices, and the per-matrix Gram
// terms are accumulated in segments (krylov.cu, batched mode).  Matrices are
// stacked by increasing sequence length, so the matrices still running at
// application t form a suffix of the stack and the passes start at that
// suffix.  A phase (the applications between two sequence ends, over one set
// of running matrices) is ONE persistent cooperative launch: the CTAs walk
// the stacked rows of A, meet at a grid-wide barrier, walk the rows of A^T,
// meet again, for every application of the phase.  The whole Krylov loop
// (the initial pass, one launch per phase and the term finalisations) is
// captured once into a CUDA graph and launched as one graph.
//
// The generators: matrices with equal sequence length finish their Krylov
// loops together and are solved in lockstep by one batched PM-basis (one
// leaf-kernel CTA per matrix, one launch per product step for all of them);
// rr_batch_ranks runs these jobs on a few streams at once (one host thread
// and one context per stream), as soon as their sequences are complete.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <string>
#include <mutex>
#include <cstring>
#include <memory>
#include <numeric>
#include <thread>

#include "krylov_params.h"

struct rr_batch_s {
  rr_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;  // Krylov stream, highest priority
  int nmat = 0, b = 0, B = 0, np = 0;
  uint32_t p = 0;
  rr::ModP M{};
  int fold4 = 0;
  int grid = 0;
  std::vector<int> order;        // stack position -> caller's index
  std::vector<int> pos_of;       // caller's index -> stack position
  std::vector<int64_t> m, n;     // per stack position
  std::vector<int64_t> apps;     // applications of B per stack position
  std::vector<int64_t> row_off, col_off;  // padded offsets per stack position (+1 entries)
  std::vector<int64_t> s_off;    // sequence offset (words) per stack position
  rr::DevCsr A, At;
  // lanes-per-thread variants of the persistent kernel (rows per warp batch
  // differ): per variant, the matrix of each row batch of A / A^T and the
  // work prefix over row batches; variant kDefaultVariant is also the shape
  // of the initial pass
  int nvar = 1;
  int lpt[2] = {4, 4};
  rr::DevBuf<int32_t> seg_rows[2], seg_cols[2];
  std::vector<int64_t> work_rows[2], work_cols[2];
  int def_var = 0;
  std::vector<int> phase_var;    // phase -> lanes-per-thread variant (autotuned)
  // equal-work warp runs per phase (a phase = a set of running matrices):
  // runs_*[phase][warp], kPassWarps * grid + 1 entries each
  rr::DevBuf<int32_t> runs_rows, runs_cols;
  std::vector<int> phase_of;     // first running stack position -> phase
  std::vector<int> phase_first;  // phase -> first running stack position
  std::vector<int> phase_grid;   // phase -> CTAs of its pass launches (autotuned)
  std::vector<int64_t> run_off;  // phase -> offset of its warp-run tables (phase_grid * kPassWarps + 1 entries)
  rr::DevBuf<uint32_t> X[2], U, dr_m, dc_m, dc_r, W0;
  rr::DevBuf<unsigned long long> gram_acc;
  rr::DevBuf<unsigned long long> gram_all;  // one Gram slot per (matrix, term): [seg_G_off[s] + t * NP]
  rr::DevBuf<int64_t> d_seg_G_off, d_seg_terms;
  rr::DevBuf<unsigned int> counter;
  rr::DevBuf<uint32_t> S;
  rr::DevBuf<int64_t> d_s_off;
  rr::DevBuf<unsigned int> bar;  // grid barrier of the persistent launches: arrivals, generation
  rr::DevBuf<int> error;         // set when a barrier wait gives up
  int64_t nnz = 0;
  int cur = 0;
  bool done = false;
  ~rr_batch_s() {
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace rr {
namespace {

int64_t default_len(int64_t m, int64_t n, int b) {  // src/main.rs:497-504
  int64_t L = (int64_t)std::floor(2.0f * (float)std::min(m, n) / (float)b + 4.0f);
  if (b > 1) {
    int64_t q = 1;
    while (q < L) q *= 2;
    L = q;
  }
  return L;
}

int64_t pad32(int64_t x) { return (x + 31) / 32 * 32; }

// fn(i) for i < count on the host's cores (each index touches its own data).
template <class F>
void parallel_for(int count, F fn) {
  const int nt = std::max(1, std::min<int>(count, (int)std::thread::hardware_concurrency()));
  if (nt == 1) {
    for (int i = 0; i < count; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1)) fn(i);
    });
  for (auto& th : pool) th.join();
}

PassParams batch_params(rr_batch* bt) {
  PassParams P;
  std::memset(&P, 0, sizeof(P));
  P.gram_acc = bt->gram_acc.ptr;
  P.gram_stride = (int64_t)bt->nmat * (bt->B * (bt->B + 1) / 2);
  P.replicas = 1;
  P.counter = bt->counter.ptr;
  P.gram_mul = 1;
  P.w4 = bt->M.c32;
  P.w5 = (uint32_t)((uint64_t)bt->M.c32 * 256 % bt->p);
  P.w6 = (uint32_t)((uint64_t)P.w5 * 256 % bt->p);
  P.b_real = bt->b;
  P.M = bt->M;
  P.S_all = bt->S.ptr;
  P.S_out = bt->S.ptr;  // non-null: emit terms
  P.seg_S_off = bt->d_s_off.ptr;
  P.gram_all = bt->gram_all.ptr;  // slot per term, finished per group by batch_finalize_kernel
  P.seg_G_off = bt->d_seg_G_off.ptr;
  return P;
}


// Work of a row: its nonzeros plus a fixed cost for the row's epilogue and
// Gram contribution, in units of one gathered nonzero.
constexpr int64_t kRowCost = 3;

// Boundaries that split batches [qb, nb) into `nw` contiguous runs of about
// equal work (prefix = work prefix over batches).
void equal_runs(const std::vector<int64_t>& prefix, int64_t qb, int64_t nb, int nw, int32_t* out) {
  const int64_t base = prefix[qb], total = prefix[nb] - base;
  int64_t q = qb;
  for (int w = 0; w <= nw; ++w) {
    const int64_t target = base + (int64_t)((unsigned __int128)total * (uint64_t)w / (uint64_t)nw);
    while (q < nb && prefix[q] < target) ++q;
    out[w] = (int32_t)q;
  }
  out[nw] = (int32_t)nb;
}

std::vector<int64_t> batch_work(const std::vector<uint32_t>& ptr, int rpb) {
  const int64_t rows = (int64_t)ptr.size() - 1, nb = rows / rpb;
  std::vector<int64_t> pre(nb + 1, 0);
  for (int64_t q = 0; q < nb; ++q)
    pre[q + 1] = pre[q] + (int64_t)(ptr[(q + 1) * rpb] - ptr[q * rpb]) + kRowCost * rpb;
  return pre;
}

// Warp-run tables (both passes) of phase ph for a grid of `grid` CTAs.
void phase_runs(const rr_batch* bt, int ph, int grid, int var, int32_t* ra, int32_t* rt) {
  const int rpb = rows_per_batch(bt->B, bt->lpt[var]), f = bt->phase_first[ph], nw = grid * kPassWarps;
  equal_runs(bt->work_rows[var], bt->row_off[f] / rpb, bt->row_off[bt->nmat] / rpb, nw, ra);
  equal_runs(bt->work_cols[var], bt->col_off[f] / rpb, bt->col_off[bt->nmat] / rpb, nw, rt);
}

// A grid-wide barrier wait gives up after this long (the whole phase then
// stops and rr_batch_krylov / rr_batch_ranks return RR_ETIMEOUT).
constexpr uint64_t kBarrierLimitNs = 2000000000ull;

// Parameters of the persistent launch of phase ph for applications
// [t_begin, t_end) with the given grid and warp-run tables.
PersistParams phase_params(rr_batch* bt, int ph, int var, const int32_t* d_ra, const int32_t* d_rt, int64_t t_begin,
                           int64_t t_end, int cur0) {
  const int rpb = rows_per_batch(bt->B, bt->lpt[var]), nmat = bt->nmat, first = bt->phase_first[ph];
  PersistParams Q;
  std::memset(&Q, 0, sizeof(Q));
  PassParams P = batch_params(bt);
  P.seg_begin = first;
  P.seg_end = nmat;
  P.replicas = std::max(1, std::min(kGramReplicas, 64 / (nmat - first)));
  // rows of A: z = A x, U = D_r z, odd term
  P.rowptr = bt->A.rowptr.ptr;
  P.cv = bt->A.cv.ptr;
  P.rows = bt->row_off[nmat];
  P.scale = bt->dr_m.ptr;
  P.gram_mul = bt->M.r1;
  P.batch_seg = bt->seg_rows[var].ptr;
  P.runs = d_ra;
  P.batch_begin = bt->row_off[first] / rpb;
  Q.odd = P;
  // rows of A^T: w' = D_c A^T U, x' = D_c w', even term
  P.rowptr = bt->At.rowptr.ptr;
  P.cv = bt->At.cv.ptr;
  P.rows = bt->col_off[nmat];
  P.scale = bt->dc_m.ptr;
  P.scale2 = bt->dc_r.ptr;
  P.gram_mul = 1;
  P.batch_seg = bt->seg_cols[var].ptr;
  P.runs = d_rt;
  P.batch_begin = bt->col_off[first] / rpb;
  Q.even = P;
  Q.X[0] = reinterpret_cast<uint4*>(bt->X[0].ptr);
  Q.X[1] = reinterpret_cast<uint4*>(bt->X[1].ptr);
  Q.U = reinterpret_cast<uint4*>(bt->U.ptr);
  Q.cur0 = cur0;
  Q.t_begin = t_begin;
  Q.t_end = t_end;
  Q.bar = bt->bar.ptr;
  Q.error = bt->error.ptr;
  Q.limit_ns = kBarrierLimitNs;
  return Q;
}

int launch_phase(rr_batch* bt, int ph, int var, int grid, const int32_t* d_ra, const int32_t* d_rt, int64_t t_begin,
                 int64_t t_end, int cur0) {
  PersistParams Q = phase_params(bt, ph, var, d_ra, d_rt, t_begin, t_end, cur0);
  RR_CUDA(cudaMemsetAsync(bt->bar.ptr, 0, 2 * sizeof(unsigned int), bt->stream));
  return launch_persistent_raw(bt->stream, bt->B, bt->fold4, grid, bt->lpt[var], Q);
}

// Autotuner: for every phase, time a persistent launch of three
// applications of B with 1..`max_cps` co-resident CTAs per SM and keep the
// fastest.  Few or small running matrices leave each warp only a few row
// batches on the full grid, and the per-warp fixed costs (Gram set-up, flush,
// atomics) and the barriers then dominate; a smaller grid amortises them.
// The timed applications write terms 1..6 of the running matrices and
// scratch blocks only; the slots are cleared and the Krylov loop recomputes
// all of them.
int tune_phases(rr_batch* bt, const int* max_cps) {
  const int nph = (int)bt->phase_first.size(), sms = bt->ctx->num_sms;
  int cps_top = 1;
  for (int v = 0; v < bt->nvar; ++v) cps_top = std::max(cps_top, max_cps[v]);
  const int max_grid = cps_top * sms;
  RR_CUDA(cudaMemsetAsync(bt->X[0].ptr, 0, bt->X[0].bytes(), bt->stream));
  RR_CUDA(cudaMemsetAsync(bt->X[1].ptr, 0, bt->X[1].bytes(), bt->stream));
  RR_CUDA(cudaMemsetAsync(bt->U.ptr, 0, bt->U.bytes(), bt->stream));
  DevBuf<int32_t> dra, drt;
  RR_TRY(dra.alloc((size_t)max_grid * kPassWarps + 1));
  RR_TRY(drt.alloc((size_t)max_grid * kPassWarps + 1));
  std::vector<int32_t> ra((size_t)max_grid * kPassWarps + 1), rt(ra.size());
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  RR_CUDA(cudaEventCreate(&e0));
  RR_CUDA(cudaEventCreate(&e1));
  int status = RR_OK;
  bt->phase_grid.assign(nph, sms);
  bt->phase_var.assign(nph, bt->def_var);
  for (int ph = 0; ph < nph && status == RR_OK; ++ph) {
    float best = -1.f;
    for (int var = 0; var < bt->nvar && status == RR_OK; ++var)
      for (int cps = 1; cps <= std::max(1, max_cps[var]) && status == RR_OK; ++cps) {
        const int grid = cps * sms;
        phase_runs(bt, ph, grid, var, ra.data(), rt.data());
        const size_t words = (size_t)grid * kPassWarps + 1;
        if (cudaMemcpyAsync(dra.ptr, ra.data(), words * 4, cudaMemcpyHostToDevice, bt->stream) != cudaSuccess ||
            cudaMemcpyAsync(drt.ptr, rt.data(), words * 4, cudaMemcpyHostToDevice, bt->stream) != cudaSuccess) {
          status = fail(RR_ECUDA, "tuning upload failed");
          break;
        }
        status = launch_phase(bt, ph, var, grid, dra.ptr, drt.ptr, 0, 1, 0);  // warm-up
        if (status == RR_OK) cudaEventRecord(e0, bt->stream);
        if (status == RR_OK) status = launch_phase(bt, ph, var, grid, dra.ptr, drt.ptr, 0, 3, 0);
        if (status != RR_OK) break;
        cudaEventRecord(e1, bt->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          status = fail(RR_ECUDA, "tuning: %s", cudaGetErrorString(cudaGetLastError()));
          break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best < 0.f || ms < best) {
          best = ms;
          bt->phase_grid[ph] = grid;
          bt->phase_var[ph] = var;
        }
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != RR_OK) return status;
  // final tables with the chosen shapes
  bt->run_off.assign(nph + 1, 0);
  for (int ph = 0; ph < nph; ++ph) bt->run_off[ph + 1] = bt->run_off[ph] + (int64_t)bt->phase_grid[ph] * kPassWarps + 1;
  std::vector<int32_t> fa(bt->run_off[nph]), ft(bt->run_off[nph]);
  for (int ph = 0; ph < nph; ++ph)
    phase_runs(bt, ph, bt->phase_grid[ph], bt->phase_var[ph], fa.data() + bt->run_off[ph], ft.data() + bt->run_off[ph]);
  RR_TRY(bt->runs_rows.alloc(fa.size()));
  RR_TRY(bt->runs_cols.alloc(ft.size()));
  RR_CUDA(cudaMemcpyAsync(bt->runs_rows.ptr, fa.data(), fa.size() * 4, cudaMemcpyHostToDevice, bt->stream));
  RR_CUDA(cudaMemcpyAsync(bt->runs_cols.ptr, ft.data(), ft.size() * 4, cudaMemcpyHostToDevice, bt->stream));
  RR_CUDA(cudaStreamSynchronize(bt->stream));
  return RR_OK;
}

// Completion of the sequences as the Krylov loop publishes them.
struct Progress {
  std::mutex mu;
  std::condition_variable cv;
  int published = 0;  // stack positions [0, published) have complete sequences
  bool failed = false;
};

// The whole Krylov loop on the batch's stream: S_0 and x = D_c V for every
// matrix, then one persistent launch per phase, each followed by the
// finalisation of the terms of the matrices whose sequences end there (and,
// with ev, the record of their events; stack position s is then published).
// The launches are captured into one CUDA graph and launched once.
int krylov_queue(rr_batch* bt, cudaEvent_t* ev) {
  cudaStream_t st = bt->stream;
  const int nmat = bt->nmat;
  {  // x = D_c V and S_0 for every matrix
    PassParams P = batch_params(bt);
    P.rows = bt->col_off[nmat];
    P.X = reinterpret_cast<const uint4*>(bt->W0.ptr);
    P.Y = reinterpret_cast<uint4*>(bt->X[0].ptr);
    P.scale = bt->dc_r.ptr;
    P.batch_seg = bt->seg_cols[bt->def_var].ptr;
    P.batch_begin = 0;
    P.seg_begin = 0;
    P.seg_end = nmat;
    P.term = 0;
    RR_TRY(launch_pass_raw(st, bt->B, bt->fold4, bt->grid, P, kModeInit));
  }
  RR_CUDA(cudaMemsetAsync(bt->error.ptr, 0, sizeof(int), st));
  const int64_t max_apps = bt->apps[nmat - 1];
  int first = 0, cur = 0;
  int64_t t = 0;
  while (t < max_apps) {
    while (first < nmat && bt->apps[first] <= t) ++first;
    const int ph = bt->phase_of[first];
    const int64_t t_end = bt->apps[first];  // the next sequence end
    const size_t run_off = (size_t)bt->run_off[ph];
    RR_TRY(launch_phase(bt, ph, bt->phase_var[ph], bt->phase_grid[ph], bt->runs_rows.ptr + run_off,
                        bt->runs_cols.ptr + run_off, t, t_end, cur));
    cur ^= (int)((t_end - t) & 1);
    t = t_end;
    // matrices whose sequences end here: finish their terms
    int done_to = first;
    while (done_to < nmat && bt->apps[done_to] == t) ++done_to;
    RR_TRY(launch_batch_finalize(st, bt->gram_all.ptr, bt->d_seg_G_off.ptr, bt->S.ptr, bt->d_s_off.ptr,
                                 bt->d_seg_terms.ptr, first, done_to, 2 * t + 1, bt->b, bt->B, bt->M));
    if (ev)
      for (int s = first; s < done_to; ++s) RR_CUDA(cudaEventRecordWithFlags(ev[s], st, cudaEventRecordExternal));
  }
  bt->cur = cur;
  return RR_OK;
}

int krylov_run(rr_batch* bt, cudaEvent_t* ev, Progress* prog) {
  cudaStream_t st = bt->stream;
  cudaGraph_t g = nullptr;
  RR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  const int rc = krylov_queue(bt, ev);
  const cudaError_t ec = cudaStreamEndCapture(st, &g);
  if (rc != RR_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  RR_CUDA(ec);
  cudaGraphExec_t ge = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  RR_CUDA(ei);
  const cudaError_t el = cudaGraphLaunch(ge, st);
  cudaGraphExecDestroy(ge);  // released once the launch completes
  RR_CUDA(el);
  if (ev) {  // everything is queued: the events mark each sequence's completion
    {
      std::lock_guard<std::mutex> lk(prog->mu);
      prog->published = bt->nmat;
    }
    prog->cv.notify_all();
  }
  return RR_OK;
}

// RR_ETIMEOUT when a grid barrier of the persistent launches gave up
// (synchronises the batch's stream).
int krylov_status(rr_batch* bt) {
  int err = 0;
  RR_CUDA(cudaMemcpyAsync(&err, bt->error.ptr, sizeof(int), cudaMemcpyDeviceToHost, bt->stream));
  RR_CUDA(cudaStreamSynchronize(bt->stream));
  if (err) return fail(RR_ETIMEOUT, "a grid barrier of the persistent Krylov launch gave up after %.1f s",
                       (double)kBarrierLimitNs * 1e-9);
  return RR_OK;
}

}  // namespace
}  // namespace rr

using namespace rr;

extern "C" {

int rr_batch_create(rr_ctx* ctx, int32_t nmat, const int64_t* m, const int64_t* n, const int64_t* const* rowptr,
                    const int32_t* const* col, const uint32_t* const* val, uint32_t p, int32_t b,
                    const uint32_t* const* row_precond, const uint32_t* const* col_precond,
                    const uint32_t* const* V, rr_batch** out) {
  if (!ctx || !out || !m || !n || !rowptr || !col || !val || !row_precond || !col_precond || !V)
    return fail(RR_EINVAL, "NULL argument");
  *out = nullptr;
  if (nmat < 1) return fail(RR_EINVAL, "nmat = %d", nmat);
  if (b < 1 || b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", b);
  RR_TRY(rr_prime_check(p));
  RR_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<rr_batch> bt(new rr_batch);
  bt->ctx = ctx;
  bt->nmat = nmat;
  bt->b = b;
  bt->B = b <= 4 ? 4 : b <= 8 ? 8 : b <= 16 ? 16 : 32;
  bt->np = b * (b + 1) / 2;
  bt->p = p;
  bt->M = make_modp(p);
  {
    const unsigned __int128 F = (unsigned __int128)0xffffffffull * bt->M.c32 + 0xffffffffull;
    const unsigned __int128 q = (unsigned __int128)(p - 1) * (p - 1);
    bt->fold4 = (F + 4 * q) < ((unsigned __int128)1 << 64);
  }
  // validate (in parallel over matrices) and order by sequence length
  std::vector<int64_t> len(nmat);
  std::vector<std::string> bad(nmat);
  parallel_for(nmat, [&](int i) {
    char msg[160] = "";
    if (m[i] < 1 || n[i] < 1 || !rowptr[i] || rowptr[i][0] != 0) {
      snprintf(msg, sizeof msg, "matrix %d: bad shape/rowptr", i);
    } else {
      for (int64_t r = 0; r < m[i] && !msg[0]; ++r)
        if (rowptr[i][r + 1] < rowptr[i][r]) snprintf(msg, sizeof msg, "matrix %d: rowptr decreases", i);
      for (int64_t k = 0; !msg[0] && k < rowptr[i][m[i]]; ++k)
        if (col[i][k] < 0 || col[i][k] >= n[i] || val[i][k] >= p)
          snprintf(msg, sizeof msg, "matrix %d: entry %lld invalid", i, (long long)k);
      for (int64_t r = 0; !msg[0] && r < m[i]; ++r)
        if (!row_precond[i][r] || row_precond[i][r] >= p) snprintf(msg, sizeof msg, "matrix %d: row_precond not in [1,p)", i);
      for (int64_t c = 0; !msg[0] && c < n[i]; ++c)
        if (!col_precond[i][c] || col_precond[i][c] >= p) snprintf(msg, sizeof msg, "matrix %d: col_precond not in [1,p)", i);
      for (int64_t e = 0; !msg[0] && e < (int64_t)b * n[i]; ++e)
        if (V[i][e] >= p) snprintf(msg, sizeof msg, "matrix %d: V not reduced", i);
    }
    bad[i] = msg;
    len[i] = msg[0] ? 0 : default_len(m[i], n[i], b);
  });
  for (int i = 0; i < nmat; ++i)
    if (!bad[i].empty()) return fail(RR_EINVAL, "%s", bad[i].c_str());
  bt->order.resize(nmat);
  std::iota(bt->order.begin(), bt->order.end(), 0);
  std::stable_sort(bt->order.begin(), bt->order.end(), [&](int a, int c) { return len[a] < len[c]; });
  bt->pos_of.resize(nmat);
  for (int s = 0; s < nmat; ++s) bt->pos_of[bt->order[s]] = s;
  bt->m.resize(nmat);
  bt->n.resize(nmat);
  bt->apps.resize(nmat);
  bt->row_off.assign(nmat + 1, 0);
  bt->col_off.assign(nmat + 1, 0);
  bt->s_off.assign(nmat + 1, 0);
  int64_t nnz = 0;
  std::vector<int64_t> nnz_off(nmat + 1, 0);
  for (int s = 0; s < nmat; ++s) {
    const int i = bt->order[s];
    bt->m[s] = m[i];
    bt->n[s] = n[i];
    bt->apps[s] = len[i] / 2;  // a fresh start ends at len + 1 terms (src/main.rs:109-156)
    bt->row_off[s + 1] = bt->row_off[s] + pad32(m[i]);
    bt->col_off[s + 1] = bt->col_off[s] + pad32(n[i]);
    bt->s_off[s + 1] = bt->s_off[s] + (int64_t)bt->np * (2 * bt->apps[s] + 1);
    nnz += rowptr[i][m[i]];
    nnz_off[s + 1] = nnz;
  }
  if (nnz >= (1ll << 32) - 1) return fail(RR_EUNSUPPORTED, "batch nnz %lld exceeds 2^32 - 2", (long long)nnz);
  bt->nnz = nnz;
  const int64_t Mtot = bt->row_off[nmat], Ntot = bt->col_off[nmat];
  if (Mtot >= (1ll << 31) || Ntot >= (1ll << 31)) return fail(RR_EUNSUPPORTED, "batch too large");
  // stacked CSR of A (per-matrix degree order) and its transpose
  std::vector<uint32_t> aptr(Mtot + 1, 0), tptr(Ntot + 1, 0);
  std::vector<uint2> acv(std::max<int64_t>(nnz, 1)), tcv(std::max<int64_t>(nnz, 1));
  std::vector<uint32_t> drm(Mtot, 1), dcm(Ntot, 1), dcr(Ntot, 1), w0(Ntot * bt->B, 0);
  const uint64_t R1 = bt->M.r1, R2 = R1 * R1 % p;
  // every matrix fills its own ranges of the stacked arrays: in parallel
  parallel_for(nmat, [&](int s) {
    const int i = bt->order[s];
    const int64_t mi = m[i], ni = n[i];
    std::vector<int64_t> rdeg(mi), cdeg(ni, 0);
    for (int64_t r = 0; r < mi; ++r) rdeg[r] = rowptr[i][r + 1] - rowptr[i][r];
    for (int64_t k = 0; k < rowptr[i][mi]; ++k) cdeg[col[i][k]]++;
    std::vector<int32_t> rperm(mi), cperm(ni), cinv(ni);
    std::iota(rperm.begin(), rperm.end(), 0);
    std::iota(cperm.begin(), cperm.end(), 0);
    std::stable_sort(rperm.begin(), rperm.end(), [&](int32_t a, int32_t c) { return rdeg[a] > rdeg[c]; });
    std::stable_sort(cperm.begin(), cperm.end(), [&](int32_t a, int32_t c) { return cdeg[a] > cdeg[c]; });
    for (int64_t c = 0; c < ni; ++c) cinv[cperm[c]] = (int32_t)c;
    const int64_t r0 = bt->row_off[s], c0 = bt->col_off[s];
    uint32_t o = (uint32_t)nnz_off[s];
    for (int64_t rp = 0; rp < pad32(mi); ++rp) {
      aptr[r0 + rp] = o;
      if (rp < mi) {
        const int64_t r = rperm[rp];
        const uint32_t st = o;
        for (int64_t k = rowptr[i][r]; k < rowptr[i][r + 1]; ++k)
          acv[o++] = make_uint2((uint32_t)(c0 + cinv[col[i][k]]), val[i][k]);
        std::sort(acv.begin() + st, acv.begin() + o, [](const uint2& a, const uint2& c) { return a.x < c.x; });
        drm[r0 + rp] = (uint32_t)(row_precond[i][r] * R2 % p);
      }
    }
    for (int64_t cp = 0; cp < ni; ++cp) {
      const int64_t c = cperm[cp];
      dcm[c0 + cp] = (uint32_t)(col_precond[i][c] * R2 % p);
      dcr[c0 + cp] = (uint32_t)(col_precond[i][c] * R1 % p);
      for (int l = 0; l < b; ++l) w0[(c0 + cp) * bt->B + l] = V[i][(size_t)l * ni + c];
    }
    // this matrix's block of the transpose: its columns are [c0, c1), its
    // entries [nnz_off[s], nnz_off[s + 1]); counting sort, stable by row, into
    // its own range of tptr / tcv only
    const int64_t c1 = bt->col_off[s + 1], r1 = bt->row_off[s + 1], nc = c1 - c0;
    std::vector<uint32_t> start(nc + 1, 0);
    for (int64_t k = nnz_off[s]; k < nnz_off[s + 1]; ++k) start[acv[k].x - c0 + 1]++;
    for (int64_t c = 0; c < nc; ++c) start[c + 1] += start[c];
    std::vector<uint32_t> next(nc);
    for (int64_t c = 0; c < nc; ++c) next[c] = tptr[c0 + c] = (uint32_t)nnz_off[s] + start[c];
    for (int64_t r = r0; r < r1; ++r) {
      const uint32_t kb = aptr[r], ke = r + 1 < r1 ? aptr[r + 1] : (uint32_t)nnz_off[s + 1];
      for (uint32_t k = kb; k < ke; ++k) tcv[next[acv[k].x - c0]++] = make_uint2((uint32_t)r, acv[k].y);
    }
  });
  aptr[Mtot] = (uint32_t)nnz;
  tptr[Ntot] = (uint32_t)nnz;
  // lanes-per-thread variants; the segment of every row batch and the work
  // prefix over row batches for each
  bt->nvar = persistent_lane_options(bt->B, bt->lpt);
  bt->def_var = 0;
  for (int v = 0; v < bt->nvar; ++v)
    if (rows_per_batch(bt->B, bt->lpt[v]) == rows_per_batch(bt->B)) bt->def_var = v;
  std::vector<int32_t> srow[2], scol[2];
  for (int v = 0; v < bt->nvar; ++v) {
    const int rpb = rows_per_batch(bt->B, bt->lpt[v]);
    srow[v].resize(Mtot / rpb);
    scol[v].resize(Ntot / rpb);
    for (int s = 0; s < nmat; ++s) {
      for (int64_t q = bt->row_off[s] / rpb; q < bt->row_off[s + 1] / rpb; ++q) srow[v][q] = s;
      for (int64_t q = bt->col_off[s] / rpb; q < bt->col_off[s + 1] / rpb; ++q) scol[v][q] = s;
    }
    bt->work_rows[v] = batch_work(aptr, rpb);
    bt->work_cols[v] = batch_work(tptr, rpb);
  }
  cudaStream_t st = ctx->stream;
  auto up = [&](auto& buf, const auto& vec) -> int {
    RR_TRY(buf.alloc(std::max<size_t>(vec.size(), 1)));
    if (!vec.empty()) RR_TRY(upload_host(ctx, {{buf.ptr, vec.data(), vec.size() * sizeof(vec[0])}}, st));
    return RR_OK;
  };
  bt->A.rows = Mtot;
  bt->At.rows = Ntot;
  RR_TRY(up(bt->A.rowptr, aptr));
  RR_TRY(up(bt->A.cv, acv));
  RR_TRY(up(bt->At.rowptr, tptr));
  RR_TRY(up(bt->At.cv, tcv));
  for (int v = 0; v < bt->nvar; ++v) {
    RR_TRY(up(bt->seg_rows[v], srow[v]));
    RR_TRY(up(bt->seg_cols[v], scol[v]));
  }
  RR_TRY(up(bt->dr_m, drm));
  RR_TRY(up(bt->dc_m, dcm));
  RR_TRY(up(bt->dc_r, dcr));
  RR_TRY(up(bt->W0, w0));
  RR_TRY(up(bt->d_s_off, bt->s_off));
  RR_TRY(bt->X[0].alloc((size_t)Ntot * bt->B));
  RR_TRY(bt->X[1].alloc((size_t)Ntot * bt->B));
  RR_TRY(bt->U.alloc((size_t)Mtot * bt->B));
  const int NP = bt->B * (bt->B + 1) / 2;
  RR_TRY(bt->gram_acc.alloc((size_t)kGramReplicas * nmat * NP));
  RR_CUDA(cudaMemsetAsync(bt->gram_acc.ptr, 0, bt->gram_acc.bytes(), st));
  RR_TRY(bt->counter.alloc(4));
  RR_CUDA(cudaMemsetAsync(bt->counter.ptr, 0, bt->counter.bytes(), st));
  RR_TRY(bt->S.alloc(std::max<int64_t>(bt->s_off[nmat], 1)));
  {
    std::vector<int64_t> goff(nmat + 1, 0), terms(nmat);
    for (int s = 0; s < nmat; ++s) {
      terms[s] = 2 * bt->apps[s] + 1;
      goff[s + 1] = goff[s] + terms[s] * NP;
    }
    RR_TRY(up(bt->d_seg_G_off, goff));
    RR_TRY(up(bt->d_seg_terms, terms));
    RR_TRY(bt->gram_all.alloc((size_t)std::max<int64_t>(goff[nmat], 1)));
  }
  RR_TRY(bt->bar.alloc(2));
  RR_TRY(bt->error.alloc(1));
  RR_CUDA(cudaMemsetAsync(bt->bar.ptr, 0, bt->bar.bytes(), st));
  RR_CUDA(cudaMemsetAsync(bt->error.ptr, 0, bt->error.bytes(), st));
  int blocks = 1, pblocks[2] = {1, 1};
  RR_TRY(pass_blocks_per_sm(bt->B, bt->fold4, &blocks));
  for (int v = 0; v < bt->nvar; ++v) RR_TRY(persistent_blocks_per_sm(bt->B, bt->fold4, bt->lpt[v], &pblocks[v]));
  bt->grid = std::max(1, blocks) * ctx->num_sms;
  // phases: one per distinct set of running matrices
  bt->phase_of.assign(nmat, -1);
  for (int s = 0; s < nmat; ++s)
    if (s == 0 || bt->apps[s] != bt->apps[s - 1]) {
      bt->phase_of[s] = (int)bt->phase_first.size();
      bt->phase_first.push_back(s);
    }
  int prio_lo = 0, prio_hi = 0;
  RR_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  RR_CUDA(cudaStreamCreateWithPriority(&bt->stream, cudaStreamNonBlocking, prio_hi));
  RR_CUDA(cudaStreamSynchronize(st));
  RR_TRY(tune_phases(bt.get(), pblocks));
  RR_TRY(krylov_status(bt.get()));
  RR_CUDA(cudaMemsetAsync(bt->gram_all.ptr, 0, bt->gram_all.bytes(), bt->stream));
  RR_CUDA(cudaStreamSynchronize(bt->stream));
  RR_CUDA(cudaStreamSynchronize(st));
  *out = bt.release();
  return RR_OK;
}

int rr_batch_tuning(const rr_batch* bt, int32_t* nphases, int32_t* ctas, int64_t* apps_from) {
  if (!bt || !nphases) return fail(RR_EINVAL, "NULL argument");
  const int nph = (int)bt->phase_first.size();
  if (ctas || apps_from) {
    if (*nphases < nph) return fail(RR_EINVAL, "room for %d phases, %d needed", *nphases, nph);
    for (int ph = 0; ph < nph; ++ph) {
      if (ctas) ctas[ph] = bt->phase_grid[ph];
      if (apps_from) apps_from[ph] = bt->phase_first[ph] == 0 ? 0 : bt->apps[bt->phase_first[ph] - 1];
    }
  }
  *nphases = nph;
  return RR_OK;
}

int rr_batch_destroy(rr_batch* bt) {
  if (!bt) return RR_OK;
  cudaSetDevice(bt->ctx->device);
  cudaStreamSynchronize(bt->stream);
  delete bt;
  return RR_OK;
}

// All Krylov sequences of the batch (src/main.rs:88-216 for every matrix):
// S_0 for all, then application t over the matrices with more than t
// applications left.
int rr_batch_krylov(rr_batch* bt) {
  if (!bt) return fail(RR_EINVAL, "NULL handle");
  if (bt->done) return fail(RR_ESTATE, "the batch's sequences were already computed");
  RR_CUDA(cudaSetDevice(bt->ctx->device));
  RR_TRY(krylov_run(bt, nullptr, nullptr));
  RR_TRY(krylov_status(bt));
  bt->done = true;
  return RR_OK;
}

int rr_batch_sequence(rr_batch* bt, int32_t i, uint32_t* seq, int64_t seq_stride, int64_t* len) {
  if (!bt || !len) return fail(RR_EINVAL, "NULL argument");
  if (i < 0 || i >= bt->nmat) return fail(RR_EINVAL, "matrix index %d out of range", i);
  const int s = bt->pos_of[i];
  const int64_t L = 2 * bt->apps[s] + 1;
  *len = L;
  if (!seq) return RR_OK;
  if (!bt->done) return fail(RR_ESTATE, "rr_batch_krylov has not run");
  if (seq_stride < L) return fail(RR_EINVAL, "seq_stride %lld < %lld", (long long)seq_stride, (long long)L);
  RR_CUDA(cudaSetDevice(bt->ctx->device));
  std::vector<uint32_t> tmp((size_t)L * bt->np);
  RR_CUDA(cudaMemcpy(tmp.data(), bt->S.ptr + bt->s_off[s], tmp.size() * 4, cudaMemcpyDeviceToHost));
  for (int64_t t = 0; t < L; ++t)
    for (int q = 0; q < bt->np; ++q) seq[(size_t)q * seq_stride + t] = tmp[(size_t)t * bt->np + q];
  return RR_OK;
}

// Generators and ranks of all matrices (src/main.rs:598-606 per matrix).
// When the sequences are not computed yet, the Krylov loop runs on the
// batch's high-priority stream while `workers` host threads, each with a
// stream of its own, take the matrices in the order their sequences finish
// (shortest first) and solve their generators as soon as they are complete,
// so generator work overlaps the remaining Krylov passes.
int rr_batch_ranks(rr_batch* bt, int32_t workers, int64_t* ranks) {
  if (!bt || !ranks) return fail(RR_EINVAL, "NULL argument");
  RR_CUDA(cudaSetDevice(bt->ctx->device));
  const int nmat = bt->nmat, np = bt->np, b = bt->b;
  std::vector<cudaEvent_t> ev(nmat, nullptr);
  Progress prog;
  const bool overlap = !bt->done;
  if (overlap) {
    for (int s = 0; s < nmat; ++s) {
      cudaError_t e = cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming);
      if (e != cudaSuccess) {
        for (int u = 0; u < s; ++u) cudaEventDestroy(ev[u]);
        return fail(RR_ECUDA, "cudaEventCreate: %s", cudaGetErrorString(e));
      }
    }
  } else {
    prog.published = nmat;
  }
  // generator jobs: runs of stack positions whose generators have the same
  // order d (stack positions are sorted by sequence length, so a run is
  // contiguous and its last position finishes its Krylov loop last), solved
  // in lockstep by one batched PM-basis each; a job holds at most kJobMax
  // generators and stays within a workspace budget, so that the first ones
  // of a long run need not wait for the whole run
  struct Job { int first, count; };
  std::vector<Job> jobs;
  auto order_of = [&](int s) { return generator_order(2 * bt->apps[s] + 1); };
  {
    constexpr size_t kJobBudget = (size_t)8 << 30;
    constexpr int kJobMax = 16;
    for (int s0 = 0; s0 < nmat;) {
      int s1 = s0;
      const int64_t d = order_of(s0);
      while (s1 < nmat && order_of(s1) == d) ++s1;
      const int per = (int)std::min<size_t>(kJobMax, std::max<size_t>(1, kJobBudget / pm_workspace_bytes(b, d)));
      for (int q = s0; q < s1; q += per) jobs.push_back({q, std::min(per, s1 - q)});
      s0 = s1;
    }
  }
  workers = std::max(1, std::min(workers, (int)jobs.size()));
  std::atomic<int> next{0};
  std::vector<int> status(workers, RR_OK);
  std::vector<std::string> errors(workers);
  auto work = [&](int w) {
    cudaSetDevice(bt->ctx->device);
    rr_ctx* c = nullptr;
    int rc = rr_ctx_create(bt->ctx->device, &c);
    if (rc != RR_OK) { status[w] = rc; errors[w] = rr_last_error(); return; }
    std::vector<uint32_t> raw;
    for (;;) {
      const int j = next.fetch_add(1);
      if (j >= (int)jobs.size()) break;
      const int first = jobs[j].first, cnt = jobs[j].count, last = first + cnt - 1;
      {
        std::unique_lock<std::mutex> lk(prog.mu);
        prog.cv.wait(lk, [&] { return prog.published > last || prog.failed; });
        if (prog.published <= last) break;  // the Krylov loop failed
      }
      // equal order d for the whole job; only the first d + 1 terms are read
      const int64_t d = order_of(first), glen = d + 1;
      std::vector<std::vector<uint32_t>> seq(cnt), Mv(cnt);
      std::vector<std::vector<int64_t>> delta(cnt);
      std::vector<const uint32_t*> sp(cnt);
      std::vector<uint32_t*> mp(cnt);
      std::vector<int64_t*> dp(cnt);
      std::vector<int64_t> strides(cnt, glen);
      cudaError_t e = cudaSuccess;
      if (overlap) e = cudaStreamWaitEvent(c->stream, ev[last], 0);
      raw.resize((size_t)np * glen);
      for (int z = 0; z < cnt && e == cudaSuccess; ++z) {
        const int s = first + z;
        e = cudaMemcpyAsync(raw.data(), bt->S.ptr + bt->s_off[s], raw.size() * 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) break;
        seq[z].resize(raw.size());
        for (int64_t t = 0; t < glen; ++t)
          for (int q = 0; q < np; ++q) seq[z][(size_t)q * glen + t] = raw[(size_t)t * np + q];
        Mv[z].resize((size_t)(2 * b) * (2 * b) * (d + 1));
        delta[z].resize(2 * b);
        sp[z] = seq[z].data();
        mp[z] = Mv[z].data();
        dp[z] = delta[z].data();
      }
      if (e != cudaSuccess) {
        status[w] = RR_ECUDA;
        errors[w] = cudaGetErrorString(e);
        break;
      }
      rc = pm_basis_batch_device(c, cnt, sp.data(), strides.data(), b, d, bt->p, mp.data(), dp.data());
      for (int z = 0; z < cnt && rc == RR_OK; ++z)
        rc = rr_rank_from_basis(Mv[z].data(), delta[z].data(), b, d + 1, bt->p, &ranks[bt->order[first + z]]);
      if (rc != RR_OK) { status[w] = rc; errors[w] = rr_last_error(); break; }
    }
    rr_ctx_destroy(c);
  };
  std::vector<std::thread> pool;
  for (int w = 0; w < workers; ++w) pool.emplace_back(work, w);
  int krc = RR_OK;
  std::string kerr;
  if (overlap) {
    krc = krylov_run(bt, ev.data(), &prog);
    if (krc != RR_OK) kerr = rr_last_error();
    {
      std::lock_guard<std::mutex> lk(prog.mu);
      if (krc != RR_OK) prog.failed = true;
    }
    prog.cv.notify_all();
  }
  for (auto& th : pool) th.join();
  if (overlap) {
    if (krc == RR_OK) {
      krc = krylov_status(bt);
      if (krc != RR_OK) kerr = rr_last_error();
    }
    cudaStreamSynchronize(bt->stream);
    for (int s = 0; s < nmat; ++s) cudaEventDestroy(ev[s]);
    if (krc == RR_OK) bt->done = true;
  }
  if (krc != RR_OK) return fail(krc, "%s", kerr.c_str());
  for (int w = 0; w < workers; ++w)
    if (status[w] != RR_OK) return fail(status[w], "generator worker %d: %s", w, errors[w].c_str());
  return RR_OK;
}

int rr_batch_tuning_shape(const rr_batch* bt, int32_t* nphases, int32_t* lanes_per_thread, int32_t* rows_per_warp) {
  if (!bt || !nphases) return fail(RR_EINVAL, "NULL argument");
  const int nph = (int)bt->phase_first.size();
  if (lanes_per_thread || rows_per_warp) {
    if (*nphases < nph) return fail(RR_EINVAL, "room for %d phases, %d needed", *nphases, nph);
    for (int ph = 0; ph < nph; ++ph) {
      const int l = bt->lpt[bt->phase_var[ph]];
      if (lanes_per_thread) lanes_per_thread[ph] = l;
      if (rows_per_warp) rows_per_warp[ph] = rows_per_batch(bt->B, l);
    }
  }
  *nphases = nph;
  return RR_OK;
}

int rr_batch_info(const rr_batch* bt, int64_t* total_rows, int64_t* total_cols, int64_t* total_nnz,
                  int64_t* max_apps) {
  if (!bt || !total_rows || !total_cols || !total_nnz || !max_apps) return fail(RR_EINVAL, "NULL argument");
  *total_rows = bt->row_off[bt->nmat];
  *total_cols = bt->col_off[bt->nmat];
  *total_nnz = bt->nnz;
  *max_apps = bt->apps[bt->nmat - 1];
  return RR_OK;
}

}  // extern "C"
