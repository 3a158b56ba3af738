// batch.cu -- many matrices in one Krylov launch, then concurrent generators.
//
// The matrices of a batch (graph complexes give one per degree) are stacked
// block-diagonally: every matrix keeps its own degree order, its row block of
// A (and of A^T) is padded to a multiple of 32 rows so that no warp batch and
// no 32-row tensor-core tile straddles two matrices, and the per-matrix Gram
// terms are accumulated in segments (krylov.cu, batched mode).  Matrices are
// stacked by increasing sequence length, so the matrices still running at
// application t form a suffix of the stack and the passes start at that
// suffix.  Each application of B is then two launches for the whole batch.
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
  rr::DevBuf<int32_t> seg_rows, seg_cols;  // matrix of each row batch of A / A^T
  // equal-work warp runs per phase (a phase = a set of running matrices):
  // runs_*[phase][warp], kPassWarps * grid + 1 entries each
  rr::DevBuf<int32_t> runs_rows, runs_cols;
  std::vector<int> phase_of;  // first running stack position -> phase
  rr::DevBuf<uint32_t> X[2], U, dr_m, dc_m, dc_r, W0;
  rr::DevBuf<unsigned long long> gram_acc;
  rr::DevBuf<unsigned int> counter;
  rr::DevBuf<uint32_t> S;
  rr::DevBuf<int64_t> d_s_off;
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

// Completion of the sequences as the Krylov loop publishes them.
struct Progress {
  std::mutex mu;
  std::condition_variable cv;
  int published = 0;  // stack positions [0, published) have complete sequences
  bool failed = false;
};

// The whole Krylov loop on the batch's stream.  With ev, the event of stack
// position s is recorded after its last application and s is published.
int krylov_run(rr_batch* bt, cudaEvent_t* ev, Progress* prog) {
  cudaStream_t st = bt->stream;
  const int rpb = rows_per_batch(bt->B);
  const int nmat = bt->nmat;
  {  // x = D_c V and S_0 for every matrix
    PassParams P = batch_params(bt);
    P.rows = bt->col_off[nmat];
    P.X = reinterpret_cast<const uint4*>(bt->W0.ptr);
    P.Y = reinterpret_cast<uint4*>(bt->X[0].ptr);
    P.scale = bt->dc_r.ptr;
    P.batch_seg = bt->seg_cols.ptr;
    P.batch_begin = 0;
    P.seg_begin = 0;
    P.seg_end = nmat;
    P.term = 0;
    RR_TRY(launch_pass_raw(st, bt->B, bt->fold4, bt->grid, P, kModeInit));
  }
  bt->cur = 0;
  const int64_t max_apps = bt->apps[nmat - 1];
  int first = 0;
  for (int64_t t = 0; t < max_apps; ++t) {
    while (first < nmat && bt->apps[first] <= t) ++first;
    const size_t run_off = (size_t)bt->phase_of[first] * (bt->grid * kPassWarps + 1);
    uint32_t* x = bt->X[bt->cur].ptr;
    uint32_t* xn = bt->X[bt->cur ^ 1].ptr;
    PassParams P = batch_params(bt);
    P.seg_begin = first;
    P.seg_end = nmat;
    // few running matrices: spread their accumulators over replicas
    P.replicas = std::max(1, std::min(kGramReplicas, 64 / (nmat - first)));
    // rows of A: z = A x, U = D_r z, odd term
    P.rowptr = bt->A.rowptr.ptr;
    P.cv = bt->A.cv.ptr;
    P.rows = bt->row_off[nmat];
    P.X = reinterpret_cast<const uint4*>(x);
    P.Y = reinterpret_cast<uint4*>(bt->U.ptr);
    P.scale = bt->dr_m.ptr;
    P.gram_mul = bt->M.r1;
    P.batch_seg = bt->seg_rows.ptr;
    P.runs = bt->runs_rows.ptr + run_off;
    P.batch_begin = bt->row_off[first] / rpb;
    P.term = 2 * t + 1;
    RR_TRY(launch_pass_raw(st, bt->B, bt->fold4, bt->grid, P, kModeOdd));
    // rows of A^T: w' = D_c A^T U, x' = D_c w', even term
    P.rowptr = bt->At.rowptr.ptr;
    P.cv = bt->At.cv.ptr;
    P.rows = bt->col_off[nmat];
    P.X = reinterpret_cast<const uint4*>(bt->U.ptr);
    P.Y = reinterpret_cast<uint4*>(xn);
    P.scale = bt->dc_m.ptr;
    P.scale2 = bt->dc_r.ptr;
    P.gram_mul = 1;
    P.batch_seg = bt->seg_cols.ptr;
    P.runs = bt->runs_cols.ptr + run_off;
    P.batch_begin = bt->col_off[first] / rpb;
    P.term = 2 * t + 2;
    RR_TRY(launch_pass_raw(st, bt->B, bt->fold4, bt->grid, P, kModeEven));
    bt->cur ^= 1;
    if (ev) {
      int done_to = first;
      while (done_to < nmat && bt->apps[done_to] == t + 1) {
        RR_CUDA(cudaEventRecord(ev[done_to], st));
        ++done_to;
      }
      if (done_to > first) {
        {
          std::lock_guard<std::mutex> lk(prog->mu);
          prog->published = done_to;
        }
        prog->cv.notify_all();
      }
    }
  }
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
  // validate and order by sequence length
  std::vector<int64_t> len(nmat);
  for (int i = 0; i < nmat; ++i) {
    if (m[i] < 1 || n[i] < 1 || !rowptr[i] || rowptr[i][0] != 0) return fail(RR_EINVAL, "matrix %d: bad shape/rowptr", i);
    for (int64_t r = 0; r < m[i]; ++r)
      if (rowptr[i][r + 1] < rowptr[i][r]) return fail(RR_EINVAL, "matrix %d: rowptr decreases", i);
    for (int64_t k = 0; k < rowptr[i][m[i]]; ++k)
      if (col[i][k] < 0 || col[i][k] >= n[i] || val[i][k] >= p) return fail(RR_EINVAL, "matrix %d: entry %lld invalid", i, (long long)k);
    for (int64_t r = 0; r < m[i]; ++r)
      if (!row_precond[i][r] || row_precond[i][r] >= p) return fail(RR_EINVAL, "matrix %d: row_precond not in [1,p)", i);
    for (int64_t c = 0; c < n[i]; ++c)
      if (!col_precond[i][c] || col_precond[i][c] >= p) return fail(RR_EINVAL, "matrix %d: col_precond not in [1,p)", i);
    for (int64_t e = 0; e < (int64_t)b * n[i]; ++e)
      if (V[i][e] >= p) return fail(RR_EINVAL, "matrix %d: V not reduced", i);
    len[i] = default_len(m[i], n[i], b);
  }
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
  for (int s = 0; s < nmat; ++s) {
    const int i = bt->order[s];
    bt->m[s] = m[i];
    bt->n[s] = n[i];
    bt->apps[s] = len[i] / 2;  // a fresh start ends at len + 1 terms (src/main.rs:109-156)
    bt->row_off[s + 1] = bt->row_off[s] + pad32(m[i]);
    bt->col_off[s + 1] = bt->col_off[s] + pad32(n[i]);
    bt->s_off[s + 1] = bt->s_off[s] + (int64_t)bt->np * (2 * bt->apps[s] + 1);
    nnz += rowptr[i][m[i]];
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
  uint32_t o = 0;
  for (int s = 0; s < nmat; ++s) {
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
  }
  aptr[Mtot] = o;
  for (int64_t k = 0; k < nnz; ++k) tptr[acv[k].x + 1]++;
  for (int64_t c = 0; c < Ntot; ++c) tptr[c + 1] += tptr[c];
  {
    std::vector<uint32_t> next(tptr.begin(), tptr.end() - 1);
    for (int64_t r = 0; r < Mtot; ++r)
      for (uint32_t k = aptr[r]; k < aptr[r + 1]; ++k) tcv[next[acv[k].x]++] = make_uint2((uint32_t)r, acv[k].y);
  }
  // segment of every row batch
  const int rpb = rows_per_batch(bt->B);
  std::vector<int32_t> srow(Mtot / rpb), scol(Ntot / rpb);
  for (int s = 0; s < nmat; ++s) {
    for (int64_t q = bt->row_off[s] / rpb; q < bt->row_off[s + 1] / rpb; ++q) srow[q] = s;
    for (int64_t q = bt->col_off[s] / rpb; q < bt->col_off[s + 1] / rpb; ++q) scol[q] = s;
  }
  cudaStream_t st = ctx->stream;
  auto up = [&](auto& buf, const auto& vec) -> int {
    RR_TRY(buf.alloc(std::max<size_t>(vec.size(), 1)));
    if (!vec.empty())
      RR_CUDA(cudaMemcpyAsync(buf.ptr, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, st));
    return RR_OK;
  };
  bt->A.rows = Mtot;
  bt->At.rows = Ntot;
  RR_TRY(up(bt->A.rowptr, aptr));
  RR_TRY(up(bt->A.cv, acv));
  RR_TRY(up(bt->At.rowptr, tptr));
  RR_TRY(up(bt->At.cv, tcv));
  RR_TRY(up(bt->seg_rows, srow));
  RR_TRY(up(bt->seg_cols, scol));
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
  int blocks = 1;
  RR_TRY(pass_blocks_per_sm(bt->B, bt->fold4, &blocks));
  bt->grid = std::max(1, blocks) * ctx->num_sms;
  {  // phases: one per distinct set of running matrices
    const int nw = bt->grid * kPassWarps;
    std::vector<int> firsts;
    bt->phase_of.assign(nmat, -1);
    for (int s = 0; s < nmat; ++s)
      if (s == 0 || bt->apps[s] != bt->apps[s - 1]) {
        bt->phase_of[s] = (int)firsts.size();
        firsts.push_back(s);
      }
    const std::vector<int64_t> wa = batch_work(aptr, rpb), wt = batch_work(tptr, rpb);
    std::vector<int32_t> ra(firsts.size() * (nw + 1)), rt(firsts.size() * (nw + 1));
    for (size_t ph = 0; ph < firsts.size(); ++ph) {
      const int f = firsts[ph];
      equal_runs(wa, bt->row_off[f] / rpb, Mtot / rpb, nw, ra.data() + ph * (nw + 1));
      equal_runs(wt, bt->col_off[f] / rpb, Ntot / rpb, nw, rt.data() + ph * (nw + 1));
    }
    RR_TRY(up(bt->runs_rows, ra));
    RR_TRY(up(bt->runs_cols, rt));
  }
  int prio_lo = 0, prio_hi = 0;
  RR_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  RR_CUDA(cudaStreamCreateWithPriority(&bt->stream, cudaStreamNonBlocking, prio_hi));
  RR_CUDA(cudaStreamSynchronize(st));
  *out = bt.release();
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
  RR_CUDA(cudaStreamSynchronize(bt->stream));
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
  // generator jobs: runs of stack positions with equal sequence length (they
  // finish their Krylov loops together), solved in lockstep by one batched
  // PM-basis each, split so that a job's workspace stays within a budget
  struct Job { int first, count; };
  std::vector<Job> jobs;
  {
    constexpr size_t kJobBudget = (size_t)8 << 30;
    for (int s0 = 0; s0 < nmat;) {
      int s1 = s0;
      while (s1 < nmat && bt->apps[s1] == bt->apps[s0]) ++s1;
      const int64_t L = 2 * bt->apps[s0] + 1;
      int64_t d = 1;
      while (d <= L) d *= 2;
      d /= 2;
      const int per = (int)std::max<size_t>(1, kJobBudget / pm_workspace_bytes(b, d));
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
      const int64_t L = 2 * bt->apps[first] + 1;
      int64_t d = 1;  // src/main.rs:599-603
      while (d <= L) d *= 2;
      d /= 2;
      std::vector<std::vector<uint32_t>> seq(cnt), Mv(cnt);
      std::vector<std::vector<int64_t>> delta(cnt);
      std::vector<const uint32_t*> sp(cnt);
      std::vector<uint32_t*> mp(cnt);
      std::vector<int64_t*> dp(cnt);
      std::vector<int64_t> strides(cnt, L);
      cudaError_t e = cudaSuccess;
      if (overlap) e = cudaStreamWaitEvent(c->stream, ev[last], 0);
      raw.resize((size_t)np * L);
      for (int z = 0; z < cnt && e == cudaSuccess; ++z) {
        const int s = first + z;
        e = cudaMemcpyAsync(raw.data(), bt->S.ptr + bt->s_off[s], raw.size() * 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) break;
        seq[z].resize(raw.size());
        for (int64_t t = 0; t < L; ++t)
          for (int q = 0; q < np; ++q) seq[z][(size_t)q * L + t] = raw[(size_t)t * np + q];
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
    cudaStreamSynchronize(bt->stream);
    for (int s = 0; s < nmat; ++s) cudaEventDestroy(ev[s]);
    if (krc == RR_OK) bt->done = true;
  }
  if (krc != RR_OK) return fail(krc, "%s", kerr.c_str());
  for (int w = 0; w < workers; ++w)
    if (status[w] != RR_OK) return fail(status[w], "generator worker %d: %s", w, errors[w].c_str());
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
