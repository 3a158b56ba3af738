// fleet.cpp -- the batched and served modes across several GPUs.
//
// Matrices are independent, so they shard by matrix: each one is placed on
// one GPU by its device footprint (its CSR copies, Krylov state and
// sequence), runs there exactly as it would alone, and only its rank comes
// back to the host.  No collective and no peer memory is involved.
//
//   rr_place_by_footprint   the placement rule (host only; greedy, largest
//                           first, onto the device with the most room left)
//   rr_fleet_*              one rank service (rr_server_*) per device; each
//                           request goes to the device whose service has the
//                           most budget left after the requests it holds
//   rr_batch_ranks_multi    one batch (rr_batch_*) per device over the
//                           matrices placed there, run by one host thread
//                           per device
// The reference ranks one matrix per run (src/main.rs:254-639, commands.txt).
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "rr_internal.h"

namespace rr {

int place_by_footprint(int nitems, const uint64_t* footprint, int ndev, const uint64_t* dev_free, bool allow_over,
                       int32_t* device_of, uint64_t* dev_load) {
  if (nitems < 0 || ndev < 1) return fail(RR_EINVAL, "nitems = %d, ndev = %d", nitems, ndev);
  std::vector<uint64_t> load(ndev, 0);
  std::vector<int> order(nitems);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return footprint[a] > footprint[b]; });
  auto room = [&](int d) { return dev_free[d] > load[d] ? dev_free[d] - load[d] : 0; };
  for (int i : order) {
    int best = 0;
    for (int d = 1; d < ndev; ++d)
      if (room(d) > room(best)) best = d;
    if (footprint[i] > room(best) && !allow_over)
      return fail(RR_ENOMEM, "item %d needs %llu bytes; the most room left on any device is %llu", i,
                  (unsigned long long)footprint[i], (unsigned long long)room(best));
    device_of[i] = best;
    load[best] += footprint[i];
  }
  if (dev_load)
    for (int d = 0; d < ndev; ++d) dev_load[d] = load[d];
  return RR_OK;
}

}  // namespace rr

using namespace rr;

struct rr_fleet_s {
  std::vector<int32_t> devices;
  std::vector<rr_server*> shards;
  std::mutex mu;
  struct Placed {
    int shard;
    uint64_t local_id;
    uint64_t footprint;
    bool finished;
  };
  std::map<uint64_t, Placed> placed;
  std::vector<uint64_t> outstanding;  // bytes of submitted, not yet waited-for requests per shard
  uint64_t next_id = 1;
  int b = 0;
};

extern "C" {

int rr_place_by_footprint(int32_t nitems, const uint64_t* footprint, int32_t ndev, const uint64_t* dev_free,
                          int32_t* device_of, uint64_t* dev_load) {
  if ((nitems > 0 && (!footprint || !device_of)) || !dev_free) return fail(RR_EINVAL, "NULL argument");
  return place_by_footprint(nitems, footprint, ndev, dev_free, false, device_of, dev_load);
}

int rr_footprint(int64_t m, int64_t n, int64_t nnz, int32_t b, uint64_t* bytes) {
  if (!bytes || m < 1 || n < 1 || nnz < 0 || b < 1 || b > 32) return fail(RR_EINVAL, "bad argument");
  *bytes = footprint_of(m, n, nnz, b, max_nlen_for(m, n, b));
  return RR_OK;
}

int rr_fleet_create(const int32_t* devices, int32_t ndev, const rr_server_config* cfg, rr_fleet** out) {
  if (!devices || ndev < 1 || !cfg || !out) return fail(RR_EINVAL, "bad argument");
  *out = nullptr;
  std::unique_ptr<rr_fleet> f(new rr_fleet);
  f->b = cfg->b;
  for (int i = 0; i < ndev; ++i) {
    rr_server* s = nullptr;
    const int rc = rr_server_create(devices[i], cfg, &s);
    if (rc != RR_OK) {
      for (rr_server* x : f->shards) rr_server_destroy(x);
      return rc;
    }
    f->devices.push_back(devices[i]);
    f->shards.push_back(s);
    f->outstanding.push_back(0);
  }
  *out = f.release();
  return RR_OK;
}

int rr_fleet_submit(rr_fleet* f, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col, const uint32_t* val,
                    const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* V, uint64_t* id) {
  if (!f || !rowptr || !id) return fail(RR_EINVAL, "NULL argument");
  if (m < 1 || n < 1) return fail(RR_EINVAL, "bad shape %lld x %lld", (long long)m, (long long)n);
  const uint64_t fp = footprint_of(m, n, rowptr[m], f->b, max_nlen_for(m, n, f->b));
  int shard = 0;
  {
    std::lock_guard<std::mutex> lk(f->mu);
    const int nd = (int)f->shards.size();
    std::vector<uint64_t> room(nd);
    for (int d = 0; d < nd; ++d) {
      ServerSnapshot snap;
      server_snapshot(f->shards[d], &snap);
      room[d] = snap.hbm_budget > f->outstanding[d] ? snap.hbm_budget - f->outstanding[d] : 0;
    }
    int32_t dev = 0;
    RR_TRY(place_by_footprint(1, &fp, nd, room.data(), true, &dev, nullptr));
    shard = dev;
    f->outstanding[shard] += fp;
  }
  uint64_t local = 0;
  const int rc = rr_server_submit(f->shards[shard], m, n, rowptr, col, val, row_precond, col_precond, V, &local);
  std::lock_guard<std::mutex> lk(f->mu);
  if (rc != RR_OK) {
    f->outstanding[shard] -= fp;
    return rc;
  }
  *id = f->next_id++;
  f->placed[*id] = rr_fleet_s::Placed{shard, local, fp, false};
  return RR_OK;
}

int rr_fleet_wait(rr_fleet* f, uint64_t id, double timeout_s, int64_t* rank, double* latency_ms) {
  if (!f || !rank) return fail(RR_EINVAL, "NULL argument");
  rr_fleet_s::Placed pl;
  {
    std::lock_guard<std::mutex> lk(f->mu);
    auto it = f->placed.find(id);
    if (it == f->placed.end()) return fail(RR_EINVAL, "unknown request %llu", (unsigned long long)id);
    pl = it->second;
  }
  const int rc = rr_server_wait(f->shards[pl.shard], pl.local_id, timeout_s, rank, latency_ms);
  if (rc == RR_ETIMEOUT) return rc;
  std::lock_guard<std::mutex> lk(f->mu);
  auto& p = f->placed[id];
  if (!p.finished) {
    p.finished = true;
    f->outstanding[p.shard] -= p.footprint;
  }
  return rc;
}

int rr_fleet_device_of(rr_fleet* f, uint64_t id, int32_t* device) {
  if (!f || !device) return fail(RR_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(f->mu);
  auto it = f->placed.find(id);
  if (it == f->placed.end()) return fail(RR_EINVAL, "unknown request %llu", (unsigned long long)id);
  *device = f->devices[it->second.shard];
  return RR_OK;
}

int rr_fleet_stats(rr_fleet* f, int64_t* submitted, int64_t* completed, double* p50_ms, double* p99_ms,
                   double* ranks_per_s) {
  if (!f) return fail(RR_EINVAL, "NULL argument");
  std::vector<double> lat;
  int64_t sub = 0, done = 0;
  double t0 = 0, t1 = 0;
  bool any = false;
  for (rr_server* s : f->shards) {
    ServerSnapshot snap;
    server_snapshot(s, &snap);
    lat.insert(lat.end(), snap.latencies_ms.begin(), snap.latencies_ms.end());
    sub += snap.submitted;
    done += snap.completed;
    if (snap.submitted > 0) {
      t0 = any ? std::min(t0, snap.t_first) : snap.t_first;
      any = true;
    }
    if (snap.completed > 0) t1 = std::max(t1, snap.t_last);
  }
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double q) {
    if (lat.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>((double)lat.size() - 1, std::ceil(q * (double)lat.size()) - 1);
    return lat[k];
  };
  if (submitted) *submitted = sub;
  if (completed) *completed = done;
  if (p50_ms) *p50_ms = pct(0.50);
  if (p99_ms) *p99_ms = pct(0.99);
  if (ranks_per_s) *ranks_per_s = (done > 0 && t1 > t0) ? (double)done / (t1 - t0) : 0.0;
  return RR_OK;
}

int rr_fleet_destroy(rr_fleet* f) {
  if (!f) return RR_OK;
  for (rr_server* s : f->shards) rr_server_destroy(s);
  delete f;
  return RR_OK;
}

int rr_batch_ranks_multi(const int32_t* devices, int32_t ndev, int32_t nmat, const int64_t* m, const int64_t* n,
                         const int64_t* const* rowptr, const int32_t* const* col, const uint32_t* const* val,
                         uint32_t p, int32_t b, const uint32_t* const* row_precond, const uint32_t* const* col_precond,
                         const uint32_t* const* V, int32_t workers, int64_t* ranks, int32_t* device_of) {
  if (!devices || ndev < 1 || nmat < 1 || !m || !n || !rowptr || !col || !val || !row_precond || !col_precond || !V ||
      !ranks)
    return fail(RR_EINVAL, "bad argument");
  if (b < 1 || b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", b);
  std::vector<uint64_t> fp(nmat), room(ndev);
  for (int i = 0; i < nmat; ++i) {
    if (m[i] < 1 || n[i] < 1 || !rowptr[i]) return fail(RR_EINVAL, "matrix %d: bad shape or NULL rowptr", i);
    fp[i] = footprint_of(m[i], n[i], rowptr[i][m[i]], b, max_nlen_for(m[i], n[i], b));
  }
  int dev0 = 0;
  RR_CUDA(cudaGetDevice(&dev0));
  for (int d = 0; d < ndev; ++d) {
    RR_CUDA(cudaSetDevice(devices[d]));
    size_t fr = 0, tot = 0;
    RR_CUDA(cudaMemGetInfo(&fr, &tot));
    // a device listed k times shares its memory k ways
    const int k = (int)std::count(devices, devices + ndev, devices[d]);
    room[d] = (uint64_t)(0.8 * (double)fr / k);
  }
  RR_CUDA(cudaSetDevice(dev0));
  std::vector<int32_t> where(nmat);
  RR_TRY(place_by_footprint(nmat, fp.data(), ndev, room.data(), false, where.data(), nullptr));
  std::vector<int> status(ndev, RR_OK);
  std::vector<std::string> errors(ndev);
  std::vector<std::thread> pool;
  for (int d = 0; d < ndev; ++d) {
    pool.emplace_back([&, d] {
      std::vector<int> idx;
      for (int i = 0; i < nmat; ++i)
        if (where[i] == d) idx.push_back(i);
      if (idx.empty()) return;
      std::vector<int64_t> mm, nn;
      std::vector<const int64_t*> rp;
      std::vector<const int32_t*> cc;
      std::vector<const uint32_t*> vv, dr, dc, vs;
      for (int i : idx) {
        mm.push_back(m[i]);
        nn.push_back(n[i]);
        rp.push_back(rowptr[i]);
        cc.push_back(col[i]);
        vv.push_back(val[i]);
        dr.push_back(row_precond[i]);
        dc.push_back(col_precond[i]);
        vs.push_back(V[i]);
      }
      rr_ctx* ctx = nullptr;
      rr_batch* bt = nullptr;
      std::vector<int64_t> rk(idx.size());
      int rc = rr_ctx_create(devices[d], &ctx);
      if (rc == RR_OK)
        rc = rr_batch_create(ctx, (int32_t)idx.size(), mm.data(), nn.data(), rp.data(), cc.data(), vv.data(), p, b,
                             dr.data(), dc.data(), vs.data(), &bt);
      if (rc == RR_OK) rc = rr_batch_ranks(bt, workers, rk.data());
      if (rc != RR_OK) errors[d] = rr_last_error();
      if (bt) rr_batch_destroy(bt);
      if (ctx) rr_ctx_destroy(ctx);
      status[d] = rc;
      if (rc == RR_OK)
        for (size_t j = 0; j < idx.size(); ++j) ranks[idx[j]] = rk[j];
    });
  }
  for (auto& t : pool) t.join();
  for (int d = 0; d < ndev; ++d)
    if (status[d] != RR_OK) return fail(status[d], "device %d: %s", devices[d], errors[d].c_str());
  if (device_of)
    for (int i = 0; i < nmat; ++i) device_of[i] = devices[where[i]];
  return RR_OK;
}

}  // extern "C"
