// upload.cpp -- host-to-device copies of the caller's host arrays.
//
// Matrices and blocks arrive as ordinary (pageable) host memory: numpy arrays,
// Rust Vecs.  A cudaMemcpyAsync from pageable memory is staged by the driver
// through its own pinned buffer on the calling thread alone.  Here several host
// threads copy pieces into pinned staging buffers of the context while the
// pieces copied before them are in flight over the bus: the host copies and
// the transfers overlap, and the host copy itself runs on several cores.
// Arrays already in pinned memory go straight to cudaMemcpyAsync.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "rr_internal.h"

namespace rr {

namespace {
constexpr size_t kPiece = 2u << 20;     // bytes per staged piece
constexpr size_t kStageMin = 4u << 20;  // smaller copies go straight to the driver
constexpr int kMaxStageThreads = 8;
}  // namespace

// Per-context staging: two pinned buffers and two events per copy thread,
// allocated at the first staged copy, freed with the context.
struct Staging {
  std::mutex mu;
  int threads = 0;
  std::vector<void*> buf;
  std::vector<cudaEvent_t> ev;
  ~Staging() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    for (void* b : buf)
      if (b) cudaFreeHost(b);
  }
};

void staging_destroy(Staging* st) { delete st; }

static bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int upload_host(rr_ctx* ctx, const std::vector<HostSegment>& segs, cudaStream_t s) {
  size_t staged = 0;
  for (const HostSegment& g : segs) {
    if (g.bytes == 0) continue;
    if (g.bytes < kStageMin || is_pinned(g.src)) {
      RR_CUDA(cudaMemcpyAsync(g.dst, g.src, g.bytes, cudaMemcpyHostToDevice, s));
    } else {
      staged += g.bytes;
    }
  }
  if (staged == 0) return RR_OK;
  // pieces of the segments that go through the staging buffers
  struct Piece {
    char* dst;
    const char* src;
    size_t bytes;
  };
  std::vector<Piece> pieces;
  for (const HostSegment& g : segs) {
    if (g.bytes < kStageMin || is_pinned(g.src)) continue;
    for (size_t off = 0; off < g.bytes; off += kPiece)
      pieces.push_back({static_cast<char*>(g.dst) + off, static_cast<const char*>(g.src) + off,
                        std::min(kPiece, g.bytes - off)});
  }
  {
    static std::mutex create_mu;
    std::lock_guard<std::mutex> lk(create_mu);
    if (!ctx->staging) ctx->staging = new Staging();
  }
  Staging& st = *ctx->staging;
  std::lock_guard<std::mutex> lk(st.mu);
  if (st.threads == 0) {
    const int nt = std::max(1, std::min<int>(kMaxStageThreads, (int)std::thread::hardware_concurrency()));
    st.buf.assign(2 * nt, nullptr);
    st.ev.assign(2 * nt, nullptr);
    for (int i = 0; i < 2 * nt; ++i) {
      RR_CUDA(cudaHostAlloc(&st.buf[i], kPiece, cudaHostAllocDefault));
      RR_CUDA(cudaEventCreateWithFlags(&st.ev[i], cudaEventDisableTiming));
    }
    st.threads = nt;
  }
  const int nt = std::min<int>(st.threads, (int)pieces.size());
  std::vector<cudaError_t> cerr(nt, cudaSuccess);
  auto work = [&](int w) {
    cudaError_t e = cudaSetDevice(ctx->device);
    int k = 0;
    for (size_t i = (size_t)w; i < pieces.size() && e == cudaSuccess; i += (size_t)nt, ++k) {
      const int b = 2 * w + (k & 1);
      e = cudaEventSynchronize(st.ev[b]);  // the previous transfer from this buffer is done
      if (e != cudaSuccess) break;
      std::memcpy(st.buf[b], pieces[i].src, pieces[i].bytes);
      e = cudaMemcpyAsync(pieces[i].dst, st.buf[b], pieces[i].bytes, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaEventRecord(st.ev[b], s);
    }
    cerr[w] = e;
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < nt; ++w) pool.emplace_back(work, w);
  work(0);
  for (std::thread& t : pool) t.join();
  for (int w = 0; w < nt; ++w)
    if (cerr[w] != cudaSuccess)
      return fail(RR_ECUDA, "staged host-to-device copy failed: %s", cudaGetErrorString(cerr[w]));
  return RR_OK;
}

}  // namespace rr
