// server.cpp -- continuous-batching rank service (rr_server_*).
//
// The reference ranks one matrix per process run (src/main.rs:254-639,
// commands.txt); this service takes rank requests as they arrive and keeps
// several in flight on one GPU:
//
//   queued  -> admitted when its device footprint fits the HBM budget and an
//              active slot is free (first come, first served)
//   loading -> a worker thread uploads the matrix (rr_matrix_create) and
//              creates its Krylov state (rr_krylov_create) on one of the
//              service's stream lanes
//   running -> the scheduler thread queues chunks of applications of B for
//              every running request, two chunks in flight per request, so
//              the Krylov steps of different requests interleave on the
//              lanes and overlap on the device
//   solving -> once its sequence is complete a worker thread copies it out
//              and solves the generator on a stream of its own, together
//              with the other complete requests whose generators have the
//              same order d (one batched PM-basis, generators in lockstep),
//              reads off the
//              rank (rr_rank_from_basis) and frees the request's device
//              memory, which admits the next requests
//   done
//
// Every request follows exactly the path of rr_rank on the same inputs
// (sequence length rule of src/main.rs:497-504, PM-basis with d = largest
// power of two <= length), so its rank does not depend on what else runs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "rr_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { kQueued, kLoading, kRunning, kSolving, kDone, kFailed };

constexpr int kMaxSolveBatch = 32;  // generators solved together by one worker
// A complete request waits up to this long for running requests whose
// generators have the same order d and whose last chunks are queued, so that
// the generators are solved in one batch (PM_Basis of order d reads only the
// first d terms, so requests of different sequence lengths but equal d batch).
constexpr auto kSolveWindow = std::chrono::milliseconds(100);

struct Request {
  uint64_t id = 0;
  ReqState state = kQueued;
  int64_t m = 0, n = 0;
  std::vector<int64_t> rowptr;
  std::vector<int32_t> col;
  std::vector<uint32_t> val, rp, cp, V;
  size_t footprint = 0;
  int lane = 0;
  rr_matrix* mat = nullptr;
  rr_krylov* kr = nullptr;
  int64_t apps_total = 0;
  // advanced by the scheduler without the service lock, read by workers
  // under it (the solve-batching window looks at running requests)
  std::atomic<int64_t> apps_queued{0};
  int64_t order = 0;  // generator order d of the complete sequence
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int inflight = 0, ev_head = 0;  // chunks queued and not yet seen complete; oldest event
  int64_t rank = -1;
  int status = RR_OK;
  std::string error;
  Clock::time_point t_submit, t_ready, t_done;
};

}  // namespace

namespace rr {

// Sequence length rule of src/main.rs:497-504.
int64_t max_nlen_for(int64_t m, int64_t n, int b) {
  int64_t L = (int64_t)std::floor(2.0f * (float)std::min(m, n) / (float)b + 4.0f);
  if (b > 1) {
    int64_t q = 1;
    while (q < L) q *= 2;
    L = q;
  }
  return L;
}

int padded(int b) { return b <= 4 ? 4 : b <= 8 ? 8 : b <= 16 ? 16 : 32; }

// Device bytes a request holds while resident: both CSR copies, the Krylov
// blocks and preconditioner forms, and its device sequence.
size_t footprint_of(int64_t m, int64_t n, int64_t nnz, int b, int64_t max_nlen) {
  const int B = padded(b);
  const size_t np = (size_t)b * (b + 1) / 2;
  const size_t csr = 2 * 8 * (size_t)nnz + 8 * (size_t)(m + n + 2) + 4 * (size_t)n;
  const size_t blocks = 4 * (size_t)B * (2 * (size_t)n + (size_t)m) + 4 * (size_t)(m + 3 * n);
  const size_t heavy = 8 * (size_t)B * (size_t)std::max(m, n) / 16;  // generous bound on split rows
  const size_t seq = 4 * np * (size_t)(max_nlen + 2);
  return (size_t)((double)(csr + blocks + heavy + seq) * 1.1) + (1u << 20);
}

}  // namespace rr

namespace {
using rr::footprint_of;
using rr::max_nlen_for;
using rr::padded;
}  // namespace

struct rr_server_s {
  int device = 0;
  rr_server_config cfg{};
  std::vector<rr_ctx*> lanes;
  std::vector<int> lane_load;
  std::mutex mu;
  std::condition_variable cv_sched, cv_work, cv_done;
  std::map<uint64_t, std::unique_ptr<Request>> reqs;
  std::deque<uint64_t> queue;      // submitted, not yet admitted
  std::deque<uint64_t> tasks;      // for the workers: requests to load
  std::deque<uint64_t> solve_q;    // for the workers: requests whose sequences are complete
  std::vector<uint64_t> running;   // for the scheduler
  size_t used = 0;
  int active = 0;
  uint64_t next_id = 1;
  bool stop = false;
  int64_t submitted = 0, completed = 0;
  Clock::time_point t_first, t_last;
  std::vector<double> latencies_ms;
  std::thread sched;
  std::vector<std::thread> workers;

  void admit_locked() {
    while (!queue.empty() && active < cfg.max_active) {
      Request& r = *reqs[queue.front()];
      if (used + r.footprint > cfg.hbm_budget && active > 0) break;  // wait for memory (FIFO)
      queue.pop_front();
      used += r.footprint;
      ++active;
      int best = 0;
      for (int l = 1; l < (int)lanes.size(); ++l)
        if (lane_load[l] < lane_load[best]) best = l;
      r.lane = best;
      ++lane_load[best];
      r.state = kLoading;
      tasks.push_back(r.id);
      cv_work.notify_one();
    }
  }

  void finish_locked(Request& r, int status) {
    r.status = status;
    r.state = status == RR_OK ? kDone : kFailed;
    r.t_done = Clock::now();
    used -= r.footprint;
    --active;
    --lane_load[r.lane];
    ++completed;
    t_last = r.t_done;
    latencies_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
    r.rowptr = {};
    r.col = {};
    r.val = {};
    r.rp = {};
    r.cp = {};
    r.V = {};
    admit_locked();
    cv_done.notify_all();
    cv_sched.notify_one();
  }

  // Worker: upload and create the Krylov state.
  int load(Request& r) {
    rr_ctx* ctx = lanes[r.lane];
    const int b = cfg.b;
    RR_TRY(rr_matrix_create(ctx, r.m, r.n, r.rowptr.data(), r.col.data(), r.val.data(), cfg.p, &r.mat));
    RR_TRY(rr_krylov_create(r.mat, b, r.rp.data(), r.cp.data(), r.V.data(), 0, &r.kr));
    const int64_t L = max_nlen_for(r.m, r.n, b);
    r.apps_total = L / 2;  // src/main.rs:109,131: (max_nlen - 0) / 2 applications, 2 terms each
    r.order = rr::generator_order(1 + 2 * r.apps_total);
    RR_TRY(rr::krylov_reserve(r.kr, 2 * r.apps_total + 2));
    for (auto& e : r.ev) RR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return RR_OK;
  }

  // Worker: sequences -> generators (in lockstep) -> ranks, on the worker's
  // own context, for requests of equal sequence length.
  int solve(std::vector<Request*>& rs, rr_ctx* wctx) {
    const int b = cfg.b, np = b * (b + 1) / 2, cnt = (int)rs.size();
    // one order d for the batch; the generator reads the first d + 1 terms
    const int64_t d = rs[0]->order, L = d + 1;
    RR_CUDA(cudaSetDevice(device));
    // every chunk's event has completed (the scheduler saw them), so the
    // sequences are final in device memory
    std::vector<uint32_t> raw((size_t)L * np);
    std::vector<std::vector<uint32_t>> seq(cnt);
    for (int z = 0; z < cnt; ++z) {
      RR_CUDA(cudaMemcpyAsync(raw.data(), rs[z]->kr->S.ptr, raw.size() * 4, cudaMemcpyDeviceToHost,
                              (cudaStream_t)rr_ctx_stream(wctx)));
      RR_CUDA(cudaStreamSynchronize((cudaStream_t)rr_ctx_stream(wctx)));
      seq[z].resize((size_t)np * L);
      for (int64_t t = 0; t < L; ++t)
        for (int q = 0; q < np; ++q) seq[z][(size_t)q * L + t] = raw[(size_t)t * np + q];
      rr_krylov_destroy(rs[z]->kr);
      rs[z]->kr = nullptr;
      rr_matrix_destroy(rs[z]->mat);
      rs[z]->mat = nullptr;
    }
    std::vector<std::vector<uint32_t>> M(cnt);
    std::vector<std::vector<int64_t>> delta(cnt);
    std::vector<const uint32_t*> sp(cnt);
    std::vector<uint32_t*> mp(cnt);
    std::vector<int64_t*> dp(cnt);
    std::vector<int64_t> strides(cnt, L);
    for (int z = 0; z < cnt; ++z) {
      M[z].resize((size_t)(2 * b) * (2 * b) * (d + 1));
      delta[z].resize(2 * b);
      sp[z] = seq[z].data();
      mp[z] = M[z].data();
      dp[z] = delta[z].data();
    }
    RR_TRY(rr::pm_basis_batch_device(wctx, cnt, sp.data(), strides.data(), b, d, cfg.p, mp.data(), dp.data()));
    for (int z = 0; z < cnt; ++z) RR_TRY(rr_rank_from_basis(M[z].data(), delta[z].data(), b, d + 1, cfg.p, &rs[z]->rank));
    return RR_OK;
  }

  void release(Request& r) {
    for (auto& e : r.ev)
      if (e) {
        cudaEventDestroy(e);
        e = nullptr;
      }
    if (r.kr) rr_krylov_destroy(r.kr);
    if (r.mat) rr_matrix_destroy(r.mat);
    r.kr = nullptr;
    r.mat = nullptr;
  }

  void worker_main() {
    cudaSetDevice(device);
    rr_ctx* wctx = nullptr;
    const int wrc = rr_ctx_create(device, &wctx);
    const std::string werr = wrc == RR_OK ? std::string() : std::string(rr_last_error());
    for (;;) {
      std::vector<Request*> batch;
      bool loading = false;
      {
        std::unique_lock<std::mutex> lk(mu);
        // a complete request may be solved now unless a running request of
        // the same order is about to complete and its window has not run out
        auto solvable = [&](Clock::time_point now) -> int {
          for (size_t q = 0; q < solve_q.size(); ++q) {
            const Request* r = reqs[solve_q[q]].get();
            bool twin_running = false;
            for (uint64_t id : running) {
              const Request* o = reqs[id].get();
              if (o->order == r->order && o->apps_total - o->apps_queued <= 2 * cfg.chunk_apps) {
                twin_running = true;
                break;
              }
            }
            if (!twin_running || now - r->t_ready >= kSolveWindow) return (int)q;
          }
          return -1;
        };
        int pick = -1;
        for (;;) {
          if (stop || !tasks.empty()) break;
          pick = solvable(Clock::now());
          if (pick >= 0) break;
          if (solve_q.empty()) cv_work.wait(lk);
          else cv_work.wait_for(lk, std::chrono::milliseconds(5));
        }
        if (stop) break;
        if (!tasks.empty()) {  // loads first: they keep the Krylov lanes busy
          batch.push_back(reqs[tasks.front()].get());
          tasks.pop_front();
          loading = true;
        } else {
          // this request and every other complete one of the same order
          Request* r0 = reqs[solve_q[pick]].get();
          solve_q.erase(solve_q.begin() + pick);
          batch.push_back(r0);
          for (auto it = solve_q.begin(); it != solve_q.end() && (int)batch.size() < kMaxSolveBatch;) {
            Request* r = reqs[*it].get();
            if (r->order == r0->order) {
              batch.push_back(r);
              it = solve_q.erase(it);
            } else {
              ++it;
            }
          }
        }
      }
      int rc = wrc;
      std::string err = werr;
      if (rc == RR_OK) {
        rc = loading ? load(*batch[0]) : solve(batch, wctx);
        if (rc != RR_OK) err = rr_last_error();
      }
      std::lock_guard<std::mutex> lk(mu);
      for (Request* r : batch) {
        if (rc != RR_OK) {
          r->error = err;
          release(*r);
          finish_locked(*r, rc);
        } else if (loading) {
          r->state = kRunning;
          running.push_back(r->id);
          cv_sched.notify_one();
        } else {
          release(*r);
          finish_locked(*r, RR_OK);
        }
      }
    }
    if (wctx) rr_ctx_destroy(wctx);
  }

  // Scheduler: two chunks of applications in flight per running request;
  // a request whose last chunk completed goes to the workers.
  void sched_main() {
    cudaSetDevice(device);
    std::vector<uint64_t> mine;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (stop) break;
        if (running.empty()) cv_sched.wait_for(lk, std::chrono::milliseconds(2));
        if (stop) break;
        mine = running;
      }
      bool progressed = false;
      std::vector<uint64_t> finished, failed;
      std::vector<std::string> errs;
      for (uint64_t id : mine) {
        Request* r;
        {
          std::lock_guard<std::mutex> lk(mu);
          r = reqs[id].get();
        }
        // retire completed chunks
        while (r->inflight > 0 && cudaEventQuery(r->ev[r->ev_head]) == cudaSuccess) {
          r->ev_head ^= 1;
          --r->inflight;
          progressed = true;
        }
        if (r->apps_queued == r->apps_total && r->inflight == 0) {
          finished.push_back(id);
          continue;
        }
        while (r->inflight < 2 && r->apps_queued < r->apps_total) {
          const int64_t k = std::min<int64_t>(cfg.chunk_apps, r->apps_total - r->apps_queued);
          int rc = rr_krylov_step_device(r->kr, k);
          const int slot = (r->ev_head + r->inflight) % 2;
          if (rc == RR_OK && cudaEventRecord(r->ev[slot], (cudaStream_t)rr_ctx_stream(lanes[r->lane])) != cudaSuccess)
            rc = rr::fail(RR_ECUDA, "cudaEventRecord failed");
          if (rc != RR_OK) {
            failed.push_back(id);
            errs.push_back(rr_last_error());
            break;
          }
          r->apps_queued += k;
          ++r->inflight;
          progressed = true;
        }
      }
      if (!finished.empty() || !failed.empty()) {
        std::lock_guard<std::mutex> lk(mu);
        for (uint64_t id : finished) {
          running.erase(std::find(running.begin(), running.end(), id));
          reqs[id]->state = kSolving;
          reqs[id]->t_ready = Clock::now();
          solve_q.push_back(id);
          cv_work.notify_one();
        }
        for (size_t q = 0; q < failed.size(); ++q) {
          running.erase(std::find(running.begin(), running.end(), failed[q]));
          Request& r = *reqs[failed[q]];
          r.error = errs[q];
          release(r);
          finish_locked(r, RR_ECUDA);
        }
      }
      if (!progressed && finished.empty()) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
};

using namespace rr;

void rr::server_snapshot(rr_server* s, ServerSnapshot* out) {
  std::lock_guard<std::mutex> lk(s->mu);
  out->latencies_ms = s->latencies_ms;
  out->submitted = s->submitted;
  out->completed = s->completed;
  out->t_first = std::chrono::duration<double>(s->t_first.time_since_epoch()).count();
  out->t_last = std::chrono::duration<double>(s->t_last.time_since_epoch()).count();
  out->hbm_budget = s->cfg.hbm_budget;
}

extern "C" {

int rr_server_create(int device, const rr_server_config* cfg, rr_server** out) {
  if (!cfg || !out) return fail(RR_EINVAL, "NULL argument");
  *out = nullptr;
  RR_TRY(rr_prime_check(cfg->p));
  if (cfg->b < 1 || cfg->b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", cfg->b);
  std::unique_ptr<rr_server> s(new rr_server);
  s->device = device;
  s->cfg = *cfg;
  if (s->cfg.lanes <= 0) s->cfg.lanes = 4;
  if (s->cfg.workers <= 0) s->cfg.workers = 4;
  if (s->cfg.max_active <= 0) s->cfg.max_active = 64;
  if (s->cfg.chunk_apps <= 0) s->cfg.chunk_apps = 64;
  RR_CUDA(cudaSetDevice(device));
  if (s->cfg.hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    RR_CUDA(cudaMemGetInfo(&fr, &tot));
    s->cfg.hbm_budget = (uint64_t)(0.8 * (double)fr);
  }
  for (int l = 0; l < s->cfg.lanes; ++l) {
    rr_ctx* c = nullptr;
    const int rc = rr_ctx_create(device, &c);
    if (rc != RR_OK) {
      for (rr_ctx* x : s->lanes) rr_ctx_destroy(x);
      return rc;
    }
    s->lanes.push_back(c);
    s->lane_load.push_back(0);
  }
  rr_server* sp = s.get();
  sp->sched = std::thread([sp] { sp->sched_main(); });
  for (int w = 0; w < s->cfg.workers; ++w) sp->workers.emplace_back([sp] { sp->worker_main(); });
  *out = s.release();
  return RR_OK;
}

int rr_server_submit(rr_server* s, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                     const uint32_t* val, const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* V,
                     uint64_t* id) {
  if (!s || !rowptr || !row_precond || !col_precond || !V || !id) return fail(RR_EINVAL, "NULL argument");
  if (m < 1 || n < 1) return fail(RR_EINVAL, "bad shape %lld x %lld", (long long)m, (long long)n);
  const int64_t nnz = rowptr[m];
  if (nnz < 0 || (nnz > 0 && (!col || !val))) return fail(RR_EINVAL, "bad CSR arrays");
  std::unique_ptr<Request> r(new Request);
  r->m = m;
  r->n = n;
  r->rowptr.assign(rowptr, rowptr + m + 1);
  r->col.assign(col, col + nnz);
  r->val.assign(val, val + nnz);
  r->rp.assign(row_precond, row_precond + m);
  r->cp.assign(col_precond, col_precond + n);
  r->V.assign(V, V + (size_t)s->cfg.b * n);
  r->footprint = footprint_of(m, n, nnz, s->cfg.b, max_nlen_for(m, n, s->cfg.b));
  if (r->footprint > s->cfg.hbm_budget)
    return fail(RR_ENOMEM, "request needs about %zu bytes of device memory, over the budget of %llu", r->footprint,
                (unsigned long long)s->cfg.hbm_budget);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  *id = r->id;
  if (s->submitted == 0) s->t_first = r->t_submit;
  ++s->submitted;
  s->queue.push_back(r->id);
  s->reqs[r->id] = std::move(r);
  s->admit_locked();
  return RR_OK;
}

int rr_server_wait(rr_server* s, uint64_t id, double timeout_s, int64_t* rank, double* latency_ms) {
  if (!s || !rank) return fail(RR_EINVAL, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return fail(RR_EINVAL, "unknown request %llu", (unsigned long long)id);
  Request& r = *it->second;
  auto done = [&] { return r.state == kDone || r.state == kFailed; };
  if (timeout_s < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
    return fail(RR_ETIMEOUT, "request %llu not finished within %.3f s", (unsigned long long)id, timeout_s);
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count();
  if (r.state == kFailed) return fail(r.status, "request %llu failed: %s", (unsigned long long)id, r.error.c_str());
  *rank = r.rank;
  return RR_OK;
}

int rr_server_stats(rr_server* s, int64_t* submitted, int64_t* completed, double* p50_ms, double* p99_ms,
                    double* ranks_per_s) {
  if (!s) return fail(RR_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> lat = s->latencies_ms;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double q) {
    if (lat.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>((double)lat.size() - 1, std::ceil(q * (double)lat.size()) - 1);
    return lat[k];
  };
  if (submitted) *submitted = s->submitted;
  if (completed) *completed = s->completed;
  if (p50_ms) *p50_ms = pct(0.50);
  if (p99_ms) *p99_ms = pct(0.99);
  if (ranks_per_s) {
    const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
    *ranks_per_s = (s->completed > 0 && span > 0) ? (double)s->completed / span : 0.0;
  }
  return RR_OK;
}

int rr_server_destroy(rr_server* s) {
  if (!s) return RR_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_sched.notify_all();
  s->cv_work.notify_all();
  if (s->sched.joinable()) s->sched.join();
  for (auto& t : s->workers)
    if (t.joinable()) t.join();
  for (auto& kv : s->reqs) s->release(*kv.second);
  for (rr_ctx* c : s->lanes) rr_ctx_destroy(c);
  delete s;
  return RR_OK;
}

}  // extern "C"
