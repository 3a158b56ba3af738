// api.cu -- the C ABI (include/rr_rank.h): contexts, matrices, Krylov handles,
// generator and rank entry points.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>

#include "krylov_params.h"

namespace rr {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}

int fail(int status, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return status;
}

uint32_t host_powmod(uint32_t a, uint64_t e, uint32_t p) {
  uint64_t r = 1 % p, b = a % p;
  while (e) {
    if (e & 1) r = r * b % p;
    b = b * b % p;
    e >>= 1;
  }
  return (uint32_t)r;
}

uint32_t host_invmod(uint32_t a, uint32_t p) { return host_powmod(a, p - 2, p); }

bool is_prime_u32(uint32_t p) {
  if (p < 2) return false;
  if (p % 2 == 0) return p == 2;
  for (uint64_t d = 3; d * d <= p; d += 2)
    if (p % d == 0) return false;
  return true;
}

ModP make_modp(uint32_t p) {
  ModP M;
  M.p = p;
  M.c32 = (uint32_t)((((uint64_t)1) << 32) % p);
  M.mu = (uint64_t)(~0ull) / p;  // floor((2^64 - 1) / p) == floor(2^64 / p) for odd p
  uint32_t inv = p;              // Newton iteration for p^{-1} mod 2^32 (p odd)
  for (int i = 0; i < 5; ++i) inv *= 2u - p * inv;
  M.pinv = (uint32_t)(0u - inv);
  M.r1 = M.c32;
  return M;
}

int launch_scatter_block(rr_krylov* kr, const uint32_t* d_V, uint32_t* d_out);
int launch_precond(rr_krylov* kr, const uint32_t* d_rp, const uint32_t* d_cp, const int32_t* d_rowperm);

}  // namespace rr

using namespace rr;

// ---------------------------------------------------------------- Krylov
static int padded_width(int b) { return b <= 4 ? 4 : b <= 8 ? 8 : b <= 16 ? 16 : 32; }

static int ensure_capacity(rr_krylov* kr, int64_t terms) {
  const int np = kr->b * (kr->b + 1) / 2;
  if (terms <= kr->cap) return RR_OK;
  int64_t ncap = std::max<int64_t>(terms, 2 * kr->cap);
  cudaStream_t s = kr->mat->ctx->stream;
  DevBuf<uint32_t> nb;
  RR_TRY(nb.alloc_async((size_t)ncap * np, s));
  if (kr->cap > 0) RR_CUDA(cudaMemcpyAsync(nb.ptr, kr->S.ptr, (size_t)kr->cap * np * 4, cudaMemcpyDeviceToDevice, s));
  // stream-ordered: the old buffer is freed after the copy and every queued step
  std::swap(kr->S.ptr, nb.ptr);
  std::swap(kr->S.n, nb.n);
  std::swap(kr->S.stream, nb.stream);
  std::swap(kr->S.ordered, nb.ordered);
  // the kernels find S through device memory (captured launches stay valid)
  RR_CUDA(cudaMemcpyAsync(kr->d_sptr.ptr, &kr->S.ptr, sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
  RR_CUDA(cudaStreamSynchronize(s));  // the source is a host field that may change again
  kr->cap = ncap;
  return RR_OK;
}

namespace rr {
// Device sequence buffer sized for `terms` terms up front (no regrowth, and
// so no stream synchronisation, while the handle is stepped).
int krylov_reserve(rr_krylov* kr, int64_t terms) {
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  return ensure_capacity(kr, terms);
}
}  // namespace rr

extern "C" {

const char* rr_status_string(int s) {
  switch (s) {
    case RR_OK: return "ok";
    case RR_EINVAL: return "invalid argument";
    case RR_EPRIME: return "unsupported modulus";
    case RR_ENOMEM: return "out of memory";
    case RR_ECUDA: return "CUDA error";
    case RR_ETIMEOUT: return "device wait timed out";
    case RR_EIO: return "I/O error";
    case RR_ESTATE: return "invalid state";
    case RR_EUNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

const char* rr_last_error(void) { return g_err.c_str(); }

const char* rr_version(void) { return "rr_b200 0.1 (sm_100a)"; }

int rr_prime_check(uint32_t p) {
  if (p <= 2 || p >= (1u << 31) || !is_prime_u32(p)) return fail(RR_EPRIME, "p = %u must be a prime in (2, 2^31)", p);
  return RR_OK;
}

int rr_ctx_create(int device, rr_ctx** out) {
  if (!out) return fail(RR_EINVAL, "out is NULL");
  *out = nullptr;
  int count = 0;
  RR_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return fail(RR_EINVAL, "device %d not present (%d devices)", device, count);
  RR_CUDA(cudaSetDevice(device));
  // two attributes, not cudaGetDeviceProperties: contexts are created per
  // worker thread inside timed work, and the full property query is slow
  int major = 0, minor = 0, sms = 0;
  RR_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  RR_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  RR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  if (major < 10)
    return fail(RR_EUNSUPPORTED, "device %d is sm_%d%d; this build targets sm_100a", device, major, minor);
  {
    // keep freed stream-ordered memory in this process's pool instead of
    // returning it to the driver at every synchronisation (the generator
    // allocates its NTT workspace per call)
    cudaMemPool_t pool;
    RR_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = ~0ull;
    RR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  std::unique_ptr<rr_ctx> c(new rr_ctx);
  c->device = device;
  c->num_sms = sms;
  RR_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = c.release();
  return RR_OK;
}

int rr_ctx_destroy(rr_ctx* ctx) {
  if (!ctx) return RR_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  rr::staging_destroy(ctx->staging);
  delete ctx;
  return RR_OK;
}

void* rr_ctx_stream(rr_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int rr_ctx_set_pm_tensor_cores(rr_ctx* ctx, int32_t enable) {
  if (!ctx) return fail(RR_EINVAL, "NULL context");
  ctx->pm_tensor_cores = enable ? 1 : 0;
  return RR_OK;
}

int rr_ctx_synchronize(rr_ctx* ctx) {
  if (!ctx) return fail(RR_EINVAL, "ctx is NULL");
  RR_CUDA(cudaSetDevice(ctx->device));
  RR_CUDA(cudaStreamSynchronize(ctx->stream));
  return RR_OK;
}

int rr_matrix_create(rr_ctx* ctx, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                     const uint32_t* val, uint32_t p, rr_matrix** out) {
  if (!ctx || !out || !rowptr) return fail(RR_EINVAL, "NULL argument");
  *out = nullptr;
  RR_TRY(rr_prime_check(p));
  if (m < 1 || n < 1 || m >= (1ll << 31) || n >= (1ll << 31)) return fail(RR_EINVAL, "bad shape %lld x %lld", (long long)m, (long long)n);
  if (rowptr[0] != 0) return fail(RR_EINVAL, "rowptr[0] must be 0");
  const int64_t nnz = rowptr[m];
  if (nnz < 0) return fail(RR_EINVAL, "rowptr[m] = %lld < 0", (long long)nnz);
  if (nnz >= (1ll << 32) - 1) return fail(RR_EUNSUPPORTED, "nnz = %lld exceeds 2^32 - 2", (long long)nnz);
  if (nnz > 0 && (!col || !val)) return fail(RR_EINVAL, "NULL col/val");
  RR_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<rr_matrix> mat(new rr_matrix);
  mat->ctx = ctx;
  mat->m = m;
  mat->n = n;
  mat->nnz = nnz;
  mat->p = p;
  // offsets, columns and values are checked on the device during the build
  RR_TRY(matrix_build_device(ctx, m, n, rowptr, col, val, p, mat.get()));
  *out = mat.release();
  return RR_OK;
}

int rr_matrix_destroy(rr_matrix* mat) {
  if (!mat) return RR_OK;
  cudaSetDevice(mat->ctx->device);
  delete mat;  // stream-ordered frees: after the work queued on the context's stream
  return RR_OK;
}

int rr_matrix_max_nnzs(const rr_matrix* mat, int64_t* max_row, int64_t* max_col) {
  if (!mat || !max_row || !max_col) return fail(RR_EINVAL, "NULL argument");
  *max_row = mat->max_row_nnz;
  *max_col = mat->max_col_nnz;
  return RR_OK;
}

int rr_matrix_shape(const rr_matrix* mat, int64_t* m, int64_t* n, int64_t* nnz) {
  if (!mat || !m || !n || !nnz) return fail(RR_EINVAL, "NULL argument");
  *m = mat->m;
  *n = mat->n;
  *nnz = mat->nnz;
  return RR_OK;
}

int rr_krylov_create(rr_matrix* mat, int32_t b, const uint32_t* row_precond, const uint32_t* col_precond,
                     const uint32_t* curv, int64_t seq_len, rr_krylov** out) {
  if (!mat || !out || !row_precond || !col_precond || !curv) return fail(RR_EINVAL, "NULL argument");
  *out = nullptr;
  if (b < 1 || b > 32) return fail(RR_EINVAL, "block width b = %d must be in [1, 32]", b);
  if (seq_len < 0) return fail(RR_EINVAL, "seq_len < 0");
  const uint32_t p = mat->p;
  const int64_t m = mat->m, n = mat->n;
  // input checks on the host's cores (the first offending index is reported)
  {
    int64_t i = host_first_index(m, [&](int64_t k) { return row_precond[k] == 0 || row_precond[k] >= p; });
    if (i < m) return fail(RR_EINVAL, "row_precond[%lld] not in [1, p)", (long long)i);
    i = host_first_index(n, [&](int64_t k) { return col_precond[k] == 0 || col_precond[k] >= p; });
    if (i < n) return fail(RR_EINVAL, "col_precond[%lld] not in [1, p)", (long long)i);
    i = host_first_index((int64_t)b * n, [&](int64_t k) { return curv[k] >= p; });
    if (i < (int64_t)b * n) return fail(RR_EINVAL, "curv entry %lld not reduced mod p", (long long)i);
  }
  rr_ctx* ctx = mat->ctx;
  RR_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  std::unique_ptr<rr_krylov> kr(new rr_krylov);
  kr->mat = mat;
  kr->b = b;
  kr->B = padded_width(b);
  kr->M = make_modp(p);
  {
    // four products fit between folds iff (2^32-1)*c32 + 2^32 - 1 + 4 (p-1)^2 < 2^64
    const unsigned __int128 F = (unsigned __int128)0xffffffffull * kr->M.c32 + 0xffffffffull;
    const unsigned __int128 q = (unsigned __int128)(p - 1) * (p - 1);
    kr->fold4 = (F + 4 * q) < ((unsigned __int128)1 << 64);
  }
  // preconditioners in device order, in the forms the epilogues use:
  // d_r R^2, d_c R^2, d_c R and d_c^{-1} (all mod p), computed on the device
  // from the caller's arrays and the row renumbering
  {
    DevBuf<uint32_t> rp, cp;
    RR_TRY(rp.alloc_async(std::max<int64_t>(m, 1), s));
    RR_TRY(cp.alloc_async(std::max<int64_t>(n, 1), s));
    RR_TRY(kr->dr_m.alloc_async(m, s));
    RR_TRY(kr->dc_m.alloc_async(n, s));
    RR_TRY(kr->dc_r.alloc_async(n, s));
    RR_TRY(kr->dcinv.alloc_async(n, s));
    // + 4: the Gram pass copies row scales in 16-byte pieces
    RR_TRY(kr->drinv_r.alloc_async(m + 4, s));
    RR_TRY(kr->dcinv_r.alloc_async(n + 4, s));
    RR_TRY(rr::upload_host(mat->ctx, {{rp.ptr, row_precond, (size_t)m * 4}, {cp.ptr, col_precond, (size_t)n * 4}}, s));
    RR_TRY(launch_precond(kr.get(), rp.ptr, cp.ptr, mat->d_rowperm.ptr));
  }  // the staging buffers are freed in stream order, after the kernel
  const int B = kr->B;
  RR_TRY(kr->X[0].alloc_async((size_t)n * B, s));
  RR_TRY(kr->X[1].alloc_async((size_t)n * B, s));
  RR_TRY(kr->U.alloc_async((size_t)m * B, s));
  const int64_t heavy = std::max<int64_t>(std::max(mat->A.heavy_rows, mat->At.heavy_rows), 1);
  RR_TRY(kr->heavy_acc.alloc_async((size_t)heavy * B, s));
  RR_CUDA(cudaMemsetAsync(kr->heavy_acc.ptr, 0, kr->heavy_acc.bytes(), s));
  RR_TRY(kr->gram_acc.alloc_async((size_t)kGramReplicas * (B * (B + 1) / 2), s));
  RR_CUDA(cudaMemsetAsync(kr->gram_acc.ptr, 0, kr->gram_acc.bytes(), s));
  RR_TRY(kr->d_status.alloc_async(1, s));
  RR_CUDA(cudaMemsetAsync(kr->d_status.ptr, 0, sizeof(int), s));
  RR_TRY(kr->counter.alloc_async(4, s));
  RR_CUDA(cudaMemsetAsync(kr->counter.ptr, 0, kr->counter.bytes(), s));
  RR_TRY(kr->d_term.alloc_async(1, s));
  RR_TRY(kr->chunk_next.alloc_async(2, s));
  RR_CUDA(cudaMemsetAsync(kr->chunk_next.ptr, 0, 2 * sizeof(unsigned int), s));
  RR_TRY(kr->d_sptr.alloc_async(1, s));
  {
    // first application's odd term: slot 1 after S_0 of a fresh start, slot 0 on resume
    const unsigned int slot0 = seq_len == 0 ? 1u : 0u;
    RR_CUDA(cudaMemcpyAsync(kr->d_term.ptr, &slot0, sizeof(slot0), cudaMemcpyHostToDevice, s));
    RR_CUDA(cudaStreamSynchronize(s));
  }
  RR_TRY(krylov_occupancy(kr.get()));
  kr->base = seq_len;
  kr->len = seq_len;
  RR_TRY(ensure_capacity(kr.get(), 64));
  // upload curv (vector-major), scatter into device order, x = D_c w
  {
    DevBuf<uint32_t> v;
    RR_TRY(v.alloc_async((size_t)b * n, s));
    RR_TRY(rr::upload_host(mat->ctx, {{v.ptr, curv, (size_t)b * n * 4}}, s));
    RR_TRY(launch_scatter_block(kr.get(), v.ptr, kr->X[1].ptr));
    kr->cur = 0;
    // S_0 is computed now into slot 0 and published by the first advance
    RR_TRY(krylov_launch_init(kr.get(), kr->X[1].ptr, seq_len == 0));
    RR_CUDA(cudaStreamSynchronize(s));
  }
  *out = kr.release();
  return RR_OK;
}

int rr_krylov_destroy(rr_krylov* kr) {
  if (!kr) return RR_OK;
  cudaSetDevice(kr->mat->ctx->device);
  delete kr;  // stream-ordered frees: after the work queued on the context's stream
  return RR_OK;
}

// Applications per captured graph (even, so the block buffers end where they
// started and the graph can be replayed), and the run length that uses it.
constexpr int64_t kGraphApps = 16;
constexpr int64_t kGraphMinRun = 2 * kGraphApps;

// Captures kGraphApps applications (they are recorded, not run: the host
// state the launches advance is restored afterwards).  The capture runs on a
// private stream, so other threads may keep queuing work on the context's
// stream meanwhile; the graph is launched on the context's stream.
static int capture_graph(rr_krylov* kr) {
  cudaStream_t s = nullptr;
  RR_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int64_t len0 = kr->len, launches0 = kr->launches;
  const int cur0 = kr->cur;
  const cudaError_t eb = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (eb != cudaSuccess) {
    cudaStreamDestroy(s);
    RR_CUDA(eb);
  }
  kr->launch_stream = s;
  int st = RR_OK;
  for (int64_t i = 0; i < kGraphApps && st == RR_OK; ++i) st = krylov_launch_application(kr, nullptr);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  kr->launch_stream = nullptr;
  cudaStreamDestroy(s);
  kr->graph_launches = kr->launches - launches0;
  kr->len = len0;
  kr->cur = cur0;
  kr->launches = launches0;
  if (st != RR_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  RR_CUDA(e);
  const cudaError_t ei = cudaGraphInstantiate(&kr->graph, g, 0);
  cudaGraphDestroy(g);
  RR_CUDA(ei);
  kr->graph_cur = cur0;
  return RR_OK;
}

static int queue_apps(rr_krylov* kr, int64_t n_apps) {
  if (kr->len == 0) kr->len = 1;  // publish S_0
  RR_TRY(ensure_capacity(kr, kr->len - kr->base + 2 * n_apps + 1));
  int64_t i = 0;
  if (n_apps >= kGraphMinRun) {
    if (!kr->graph) RR_TRY(capture_graph(kr));
    if (kr->cur != kr->graph_cur) {
      RR_TRY(krylov_launch_application(kr, nullptr));
      ++i;
    }
    for (; n_apps - i >= kGraphApps; i += kGraphApps) {
      RR_CUDA(cudaGraphLaunch(kr->graph, kr->mat->ctx->stream));
      kr->len += 2 * kGraphApps;
      kr->launches += kr->graph_launches;
    }
  }
  for (; i < n_apps; ++i) RR_TRY(krylov_launch_application(kr, nullptr));
  return RR_OK;
}

int rr_krylov_step_device(rr_krylov* kr, int64_t n_apps) {
  if (!kr) return fail(RR_EINVAL, "NULL handle");
  if (n_apps < 0) return fail(RR_EINVAL, "n_apps < 0");
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  return queue_apps(kr, n_apps);
}

int rr_krylov_fetch(rr_krylov* kr, int64_t from, int64_t to, uint32_t* seq, int64_t seq_stride) {
  if (!kr || (!seq && to > from)) return fail(RR_EINVAL, "NULL argument");
  if (from < kr->base || to > kr->len || from > to)
    return fail(RR_EINVAL, "terms [%lld, %lld) not held (held: [%lld, %lld))", (long long)from, (long long)to,
                (long long)kr->base, (long long)kr->len);
  if (seq_stride < to) return fail(RR_EINVAL, "seq_stride %lld < %lld", (long long)seq_stride, (long long)to);
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  const int np = kr->b * (kr->b + 1) / 2;
  const int64_t cnt = to - from;
  if (cnt == 0) return RR_OK;
  std::vector<uint32_t> tmp((size_t)cnt * np);
  int dstat = 0;
  RR_CUDA(cudaMemcpyAsync(tmp.data(), kr->S.ptr + (size_t)(from - kr->base) * np, tmp.size() * 4,
                          cudaMemcpyDeviceToHost, kr->mat->ctx->stream));
  RR_CUDA(cudaMemcpyAsync(&dstat, kr->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, kr->mat->ctx->stream));
  RR_CUDA(cudaStreamSynchronize(kr->mat->ctx->stream));
  if (dstat) return fail(RR_ETIMEOUT, "a device-side wait of the Gram pass gave up; the terms are not valid");
  for (int64_t t = 0; t < cnt; ++t)
    for (int q = 0; q < np; ++q) seq[(size_t)q * seq_stride + from + t] = tmp[(size_t)t * np + q];
  return RR_OK;
}

int rr_krylov_advance_report(rr_krylov* kr, int64_t max_nlen, uint32_t* seq, int64_t seq_stride,
                             int64_t chunk_terms, rr_progress_fn fn, void* user, int64_t* new_len) {
  if (!kr || !seq || !new_len) return fail(RR_EINVAL, "NULL argument");
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  const int64_t L0 = kr->len;
  const int64_t to_be_produced = max_nlen - L0;  // src/main.rs:109
  if (to_be_produced < 0) {
    *new_len = L0;
    return RR_OK;
  }
  const int64_t final_len = (L0 == 0 ? 1 : L0) + 2 * (to_be_produced / 2);
  if (seq_stride < final_len) return fail(RR_EINVAL, "seq_stride %lld < %lld terms", (long long)seq_stride, (long long)final_len);
  const int64_t apps = to_be_produced / 2;
  const int64_t chunk = chunk_terms > 1 ? chunk_terms / 2 : std::max<int64_t>(apps, 1);
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  auto t_last = t0;
  int64_t fetched = L0, done = 0, len_last = L0;
  do {
    const int64_t k = std::min(chunk, apps - done);
    RR_TRY(queue_apps(kr, k));
    RR_TRY(rr_krylov_fetch(kr, fetched, kr->len, seq, seq_stride));  // waits for the chunk
    fetched = kr->len;
    done += k;
    if (fn) {  // report_progress (src/main.rs:57-85)
      const auto now = clk::now();
      const double dt = std::chrono::duration<double>(now - t_last).count();
      const double rate = dt > 0 ? (double)(kr->len - len_last) / dt : 0.0;
      t_last = now;
      len_last = kr->len;
      if (fn(user, kr->len, final_len, std::chrono::duration<double>(now - t0).count(), rate) != 0) break;
    }
  } while (done < apps);
  *new_len = kr->len;
  return RR_OK;
}

int rr_krylov_advance(rr_krylov* kr, int64_t max_nlen, uint32_t* seq, int64_t seq_stride, int64_t* new_len) {
  return rr_krylov_advance_report(kr, max_nlen, seq, seq_stride, 0, nullptr, nullptr, new_len);
}

int rr_krylov_fill_status(rr_krylov* kr, char* buf, int64_t cap) {
  if (!kr || !buf || cap < 1) return fail(RR_EINVAL, "bad argument");
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  // terms queued on the context's stream and how many of them have finished
  int64_t finished = kr->len;
  const cudaError_t q = cudaStreamQuery(kr->mat->ctx->stream);
  if (q == cudaErrorNotReady) finished = -1;
  else if (q != cudaSuccess) RR_CUDA(q);
  if (finished < 0)
    snprintf(buf, (size_t)cap, "%lld terms queued on the device, work in flight", (long long)kr->len);
  else
    snprintf(buf, (size_t)cap, "%lld terms computed, device idle", (long long)kr->len);
  return RR_OK;
}

int rr_device_barrier_check(rr_ctx* ctx, int32_t ctas, int32_t expected, int32_t rounds, double limit_s,
                            int32_t* timed_out) {
  if (!ctx || !timed_out || ctas < 1 || expected < 1 || rounds < 1 || !(limit_s > 0) || limit_s > 10)
    return fail(RR_EINVAL, "bad argument");
  RR_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  DevBuf<unsigned int> bar;
  DevBuf<int> err;
  RR_TRY(bar.alloc_async(2, s));
  RR_TRY(err.alloc_async(1, s));
  RR_CUDA(cudaMemsetAsync(bar.ptr, 0, 2 * sizeof(unsigned int), s));
  RR_CUDA(cudaMemsetAsync(err.ptr, 0, sizeof(int), s));
  RR_TRY(launch_barrier_check(s, ctas, bar.ptr, err.ptr, (uint64_t)(limit_s * 1e9), (unsigned)expected, rounds));
  int e = 0;
  RR_CUDA(cudaMemcpyAsync(&e, err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  *timed_out = e;
  return RR_OK;
}

int rr_krylov_length(const rr_krylov* kr, int64_t* len) {
  if (!kr || !len) return fail(RR_EINVAL, "NULL argument");
  *len = kr->len;
  return RR_OK;
}

int rr_krylov_get_curv(rr_krylov* kr, uint32_t* curv) {
  if (!kr || !curv) return fail(RR_EINVAL, "NULL argument");
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  DevBuf<uint32_t> out;
  RR_TRY(out.alloc_async((size_t)kr->b * kr->mat->n, kr->mat->ctx->stream));
  RR_TRY(krylov_launch_get_curv(kr, out.ptr));
  RR_CUDA(cudaMemcpyAsync(curv, out.ptr, out.bytes(), cudaMemcpyDeviceToHost, kr->mat->ctx->stream));
  RR_CUDA(cudaStreamSynchronize(kr->mat->ctx->stream));
  return RR_OK;
}

int rr_krylov_bytes_per_application(const rr_krylov* kr, double* bytes) {
  if (!kr || !bytes) return fail(RR_EINVAL, "NULL argument");
  const rr_matrix* m = kr->mat;
  const double csr = 2.0 * (8.0 * (double)m->nnz) + 4.0 * ((double)m->m + 1) + 4.0 * ((double)m->n + 1);
  *bytes = csr + 4.0 * kr->b * 2.0 * ((double)m->m + (double)m->n);
  return RR_OK;
}

int rr_krylov_phase_bytes(const rr_krylov* kr, double* bytes2) {
  if (!kr || !bytes2) return fail(RR_EINVAL, "NULL argument");
  const rr_matrix* m = kr->mat;
  const double dense = 4.0 * kr->b * ((double)m->m + (double)m->n);
  bytes2[0] = 8.0 * (double)m->nnz + 4.0 * ((double)m->m + 1) + dense;
  bytes2[1] = 8.0 * (double)m->nnz + 4.0 * ((double)m->n + 1) + dense;
  return RR_OK;
}

int rr_krylov_profile(rr_krylov* kr, int64_t n_apps, double* ms3) {
  if (!kr || !ms3 || n_apps < 1) return fail(RR_EINVAL, "bad argument");
  RR_CUDA(cudaSetDevice(kr->mat->ctx->device));
  if (kr->len == 0) kr->len = 1;
  RR_TRY(ensure_capacity(kr, kr->len - kr->base + 2 * n_apps + 1));
  std::vector<cudaEvent_t> ev((size_t)4 * n_apps, nullptr);
  int status = RR_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) { status = fail(RR_ECUDA, "cudaEventCreate failed"); break; }
  for (int64_t i = 0; i < n_apps && status == RR_OK; ++i) status = krylov_launch_application(kr, &ev[(size_t)4 * i]);
  double acc[3] = {0, 0, 0};
  if (status == RR_OK && cudaStreamSynchronize(kr->mat->ctx->stream) != cudaSuccess)
    status = fail(RR_ECUDA, "stream synchronize failed: %s", cudaGetErrorString(cudaGetLastError()));
  for (int64_t i = 0; i < n_apps && status == RR_OK; ++i)
    for (int k = 0; k < 3; ++k) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[(size_t)4 * i + k], ev[(size_t)4 * i + k + 1]);
      acc[k] += ms;
    }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  if (status != RR_OK) return status;
  for (int k = 0; k < 3; ++k) ms3[k] = acc[k] / (double)n_apps;
  return RR_OK;
}

int rr_krylov_launch_count(const rr_krylov* kr, int64_t* count) {
  if (!kr || !count) return fail(RR_EINVAL, "NULL argument");
  *count = kr->launches;
  return RR_OK;
}

// ---------------------------------------------------------------- generator
int rr_pm_basis(rr_ctx* ctx, const uint32_t* seq, int64_t seq_stride, int32_t b, int64_t nlen, int64_t d, uint32_t p,
                uint32_t* M, int64_t* delta) {
  if (!ctx || !seq || !M || !delta) return fail(RR_EINVAL, "NULL argument");
  RR_TRY(rr_prime_check(p));
  if (b < 1 || b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", b);
  if (seq_stride < nlen) return fail(RR_EINVAL, "seq_stride < nlen");
  int64_t dd = 1;
  while (dd < d) dd *= 2;
  if (dd >= nlen) return fail(RR_EINVAL, "sequence too short: d = %lld, nlen = %lld", (long long)dd, (long long)nlen);
  RR_CUDA(cudaSetDevice(ctx->device));
  return pm_basis_device(ctx, seq, seq_stride, b, nlen, dd, p, M, delta);
}

int rr_pm_basis_batch(rr_ctx* ctx, int32_t count, const uint32_t* const* seqs, const int64_t* seq_strides, int32_t b,
                      int64_t nlen, int64_t d, uint32_t p, uint32_t* const* M, int64_t* const* delta) {
  if (!ctx || count < 0 || (count > 0 && (!seqs || !seq_strides || !M || !delta))) return fail(RR_EINVAL, "NULL argument");
  RR_TRY(rr_prime_check(p));
  if (b < 1 || b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", b);
  int64_t dd = 1;
  while (dd < d) dd *= 2;
  if (dd >= nlen) return fail(RR_EINVAL, "sequence too short: d = %lld, nlen = %lld", (long long)dd, (long long)nlen);
  for (int z = 0; z < count; ++z) {
    if (!seqs[z] || !M[z] || !delta[z]) return fail(RR_EINVAL, "NULL array for generator %d", z);
    if (seq_strides[z] < nlen) return fail(RR_EINVAL, "seq_strides[%d] < nlen", z);
  }
  RR_CUDA(cudaSetDevice(ctx->device));
  return pm_basis_batch_device(ctx, count, seqs, seq_strides, b, dd, p, M, delta);
}

int rr_rank_from_basis(const uint32_t* M, const int64_t* delta, int32_t b, int64_t len, uint32_t p, int64_t* rank) {
  if (!M || !delta || !rank) return fail(RR_EINVAL, "NULL argument");
  if (b < 1 || len < 1) return fail(RR_EINVAL, "bad sizes");
  return rank_from_basis_host(M, delta, b, len, p, rank);
}

int rr_rank(rr_matrix* mat, int32_t b, const uint32_t* row_precond, const uint32_t* col_precond, const uint32_t* V,
            int64_t max_nlen, int64_t* rank) {
  if (!mat || !rank) return fail(RR_EINVAL, "NULL argument");
  if (b < 1 || b > 32) return fail(RR_EINVAL, "b = %d must be in [1, 32]", b);
  if (max_nlen <= 0) {  // src/main.rs:497-504
    const float dmin = (float)std::min(mat->m, mat->n);
    max_nlen = (int64_t)std::floor(2.0f * dmin / (float)b + 4.0f);
  }
  if (b > 1) {
    int64_t q = 1;
    while (q < max_nlen) q *= 2;
    max_nlen = q;
  }
  rr_krylov* kr = nullptr;
  RR_TRY(rr_krylov_create(mat, b, row_precond, col_precond, V, 0, &kr));
  std::unique_ptr<rr_krylov, int (*)(rr_krylov*)> guard(kr, rr_krylov_destroy);
  const int np = b * (b + 1) / 2;
  const int64_t stride = max_nlen + 1;
  std::vector<uint32_t> seq((size_t)np * stride);
  int64_t L = 0;
  RR_TRY(rr_krylov_advance(kr, max_nlen, seq.data(), stride, &L));
  const int64_t d = generator_order(L);
  std::vector<uint32_t> M((size_t)(2 * b) * (2 * b) * (d + 1));
  std::vector<int64_t> delta(2 * b);
  RR_TRY(rr_pm_basis(mat->ctx, seq.data(), stride, b, L, d, mat->p, M.data(), delta.data()));
  return rr_rank_from_basis(M.data(), delta.data(), b, d + 1, mat->p, rank);
}

}  // extern "C"
