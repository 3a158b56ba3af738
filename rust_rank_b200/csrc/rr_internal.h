// rr_internal.h -- host-side internals shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "rr_modp.cuh"
#include "rr_rank.h"

namespace rr {

// Thread-local error message behind rr_last_error().
void set_error(const char* fmt, ...);
int fail(int status, const char* fmt, ...);

#define RR_CUDA(call)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return ::rr::fail(e_ == cudaErrorMemoryAllocation ? RR_ENOMEM : RR_ECUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                      \
  } while (0)

#define RR_TRY(expr)          \
  do {                        \
    int s_ = (expr);          \
    if (s_ != RR_OK) return s_; \
  } while (0)

ModP make_modp(uint32_t p);
bool is_prime_u32(uint32_t p);
uint32_t host_powmod(uint32_t a, uint64_t e, uint32_t p);
uint32_t host_invmod(uint32_t a, uint32_t p);

// fn(lo, hi) over contiguous ranges covering [0, n), run on the host's cores
// (ranges of at least `grain` elements; one range, on the calling thread,
// when n is small).
template <class F>
inline void host_parallel_ranges(int64_t n, int64_t grain, F fn) {
  const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw, n / std::max<int64_t>(grain, 1)));
  if (nt == 1) {
    if (n > 0) fn((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int64_t t = 0; t < nt; ++t) pool.emplace_back([&fn, n, nt, t] { fn(n * t / nt, n * (t + 1) / nt); });
  for (auto& th : pool) th.join();
}

// Smallest i < n with bad(i), or n; scanned on the host's cores.
template <class F>
inline int64_t host_first_index(int64_t n, F bad) {
  std::atomic<int64_t> first{n};
  host_parallel_ranges(n, (int64_t)1 << 16, [&](int64_t lo, int64_t hi) {
    for (int64_t i = lo; i < hi && i < first.load(std::memory_order_relaxed); ++i)
      if (bad(i)) {
        int64_t cur = first.load();
        while (i < cur && !first.compare_exchange_weak(cur, i)) {
        }
        break;
      }
  });
  return first.load();
}

// Owning device buffer.
template <class T>
struct DevBuf {
  T* ptr = nullptr;
  size_t n = 0;
  cudaStream_t stream = nullptr;  // set for stream-ordered buffers
  bool ordered = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) {
      if (ordered) cudaFreeAsync(ptr, stream);
      else cudaFree(ptr);
    }
    ptr = nullptr;
    n = 0;
    ordered = false;
  }
  // Stream-ordered allocation: no device-wide synchronisation on free, so
  // work on other streams keeps running.
  int alloc_async(size_t count, cudaStream_t s) {
    release();
    if (count == 0) return RR_OK;
    cudaError_t e = cudaMallocAsync((void**)&ptr, count * sizeof(T), s);
    if (e != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      return fail(RR_ENOMEM, "cudaMallocAsync of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
    n = count;
    stream = s;
    ordered = true;
    return RR_OK;
  }
  int alloc(size_t count) {
    release();
    if (count == 0) return RR_OK;
    cudaError_t e = cudaMalloc((void**)&ptr, count * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      cudaGetLastError();
      return fail(RR_ENOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
    n = count;
    return RR_OK;
  }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace rr

namespace rr {
struct Staging;  // pinned staging buffers of host-to-device copies (upload.cpp)
}

struct rr_ctx_s {
  rr::Staging* staging = nullptr;  // created at the first staged copy
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int pm_tensor_cores = 1;  // PM-basis contractions on the int8 tensor cores (0: CUDA cores)
};

namespace rr {

// Degree-sorted CSR resident on the device.  Rows [0, heavy_rows) have more
// than kHeavyDegree entries and are processed by the chunk kernel.
struct DevCsr {
  DevBuf<uint32_t> rowptr;  // rows + 1 offsets
  DevBuf<uint2> cv;         // packed (column, value) per entry
  int64_t rows = 0, cols = 0, nnz = 0;
  int64_t heavy_rows = 0;
  int64_t live_rows = 0;    // rows with at least one entry: rows [0, live_rows)
  int64_t nchunks = 0;
  DevBuf<uint32_t> chunk_row, chunk_begin, chunk_end;
};

// Host arrays to copy to the device: pageable arrays of 4 MB and more go
// through the context's pinned staging buffers, several host threads copying
// pieces while earlier pieces are in flight; the rest straight to
// cudaMemcpyAsync.  Returns when the host arrays may be reused.
struct HostSegment {
  void* dst;
  const void* src;
  size_t bytes;
};
int upload_host(rr_ctx* ctx, const std::vector<HostSegment>& segs, cudaStream_t s);
void staging_destroy(Staging* st);

constexpr int64_t kHeavyDegree = 32;   // rows longer than this are split
constexpr int64_t kChunkNnz = 1024;    // nonzeros per chunk of a split row

}  // namespace rr

struct rr_matrix_s {
  rr_ctx* ctx = nullptr;
  int64_t m = 0, n = 0, nnz = 0;
  uint32_t p = 0;
  int64_t max_row_nnz = 0, max_col_nnz = 0;
  rr::DevCsr A;   // rows of A in degree order, columns renumbered in degree order
  rr::DevCsr At;  // its transpose
  rr::DevBuf<int32_t> d_rowperm;  // d_rowperm[r'] = original row
  rr::DevBuf<int32_t> d_colperm;  // d_colperm[c'] = original column
};

struct rr_krylov_s {
  rr_matrix* mat = nullptr;
  int b = 0;   // real block width
  int B = 0;   // padded width (4, 8, 16, 32)
  rr::ModP M{};
  int fold4 = 0;  // 1 when four products fit between folds
  // preconditioners in device order, in the forms the epilogues use:
  // d_r R^2, d_c R^2, d_c R (mod p, R = 2^32), d_c^{-1}, and the Gram passes'
  // d_r^{-1} R and d_c^{-1} R
  rr::DevBuf<uint32_t> dr_m, dc_m, dc_r, dcinv, drinv_r, dcinv_r;
  rr::DevBuf<uint32_t> X[2];           // x_k = D_c w_k, n x B interleaved
  rr::DevBuf<uint32_t> U;              // D_r A x_k, m x B
  rr::DevBuf<unsigned long long> heavy_acc;
  rr::DevBuf<unsigned long long> gram_acc;
  rr::DevBuf<unsigned int> counter;
  rr::DevBuf<uint32_t> S;  // device sequence, [cap][np]
  int64_t cap = 0;
  int64_t base = 0; // first term held in S
  int64_t len = 0;  // terms queued so far
  int cur = 0;      // index of the current X
  int grid_pass = 0, grid_chunk = 0, grid_lean = 0;
  rr::DevBuf<int> d_status;  // set by a device-side wait that gave up (tcgen05 Gram pass)
  int64_t launches = 0;  // kernels launched by this handle
  // device-indexed sequence output: next slot (len - base) and the S pointer
  rr::DevBuf<unsigned int> d_term;
  rr::DevBuf<unsigned int> chunk_next;  // chunk_kernel dispenser
  rr::DevBuf<uint32_t*> d_sptr;
  // a captured run of kGraphApps applications, replayable when cur == graph_cur
  cudaGraphExec_t graph = nullptr;
  cudaStream_t launch_stream = nullptr;  // set while capturing (a private stream), else the context's
  int graph_cur = 0;
  int64_t graph_launches = 0;
  ~rr_krylov_s() {
    if (graph) cudaGraphExecDestroy(graph);
  }
};

namespace rr {
int krylov_launch_init(rr_krylov* kr, const uint32_t* d_w, bool emit_s0);
int krylov_reserve(rr_krylov* kr, int64_t terms);
int krylov_launch_application(rr_krylov* kr, cudaEvent_t* ev);
int krylov_launch_get_curv(rr_krylov* kr, uint32_t* d_out);
int krylov_occupancy(rr_krylov* kr);
// Sequence length rule of src/main.rs:497-504; padded block width; device
// bytes a matrix and its Krylov state hold while resident (server.cpp).
int64_t max_nlen_for(int64_t m, int64_t n, int b);
int padded(int b);
size_t footprint_of(int64_t m, int64_t n, int64_t nnz, int b, int64_t max_nlen);
struct ServerSnapshot {
  std::vector<double> latencies_ms;
  int64_t submitted = 0, completed = 0;
  double t_first = 0, t_last = 0;  // seconds on the steady clock
  uint64_t hbm_budget = 0;
};
void server_snapshot(rr_server* s, ServerSnapshot* out);
// Greedy placement by footprint: items in decreasing size order, each on the
// device with the most room left (ties: lowest index).  With allow_over, an
// item that fits nowhere goes to the device with the most room anyway;
// otherwise that is RR_ENOMEM.  device_of[i] receives item i's device index.
int place_by_footprint(int nitems, const uint64_t* footprint, int ndev, const uint64_t* dev_free, bool allow_over,
                       int32_t* device_of, uint64_t* dev_load);

// The degree-ordered CSR of A and of its transpose, built on the device
// (build.cu); validates the input (RR_EINVAL with the first bad index).
int matrix_build_device(rr_ctx* ctx, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                        const uint32_t* val, uint32_t p, rr_matrix* mat);
// PM-basis on the device; M (host) [2b][2b][d+1], delta (host) [2b].
int pm_basis_device(rr_ctx* ctx, const uint32_t* seq, int64_t seq_stride, int b, int64_t nlen, int64_t d,
                    uint32_t p, uint32_t* M, int64_t* delta);
// The same for nb generators with equal b, d and p in lockstep (one launch per
// step for all); seqs[z] is [b(b+1)/2][seq_strides[z]], Mh[z] and deltah[z] as above.
int pm_basis_batch_device(rr_ctx* ctx, int nb, const uint32_t* const* seqs, const int64_t* seq_strides, int b,
                          int64_t d, uint32_t p, uint32_t* const* Mh, int64_t* const* deltah);
// Device bytes pm_basis_batch_device needs per generator.
size_t pm_workspace_bytes(int b, int64_t d);
// Order d of the generator computed from a sequence of nlen terms: the largest
// power of two <= nlen (src/main.rs:598-603).  PM_Basis of order d reads only
// the first d terms (M_Basis uses coefficient 0, src/sigma_basis.rs:198, and
// every product is truncated to d + 1 coefficients, src/sigma_basis.rs:205, of
// which the deepest leaf sees coefficient d - 1), so sequences of different
// lengths with equal d are solved in one batch.
inline int64_t generator_order(int64_t nlen) {
  int64_t d = 1;
  while (d <= nlen) d *= 2;
  return d / 2;
}
int rank_from_basis_host(const uint32_t* M, const int64_t* delta, int b, int64_t len, uint32_t p, int64_t* rank);
}  // namespace rr
