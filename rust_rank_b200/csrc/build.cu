// build.cu -- the matrix build on the device.
//
// rr_matrix_create uploads the caller's CSR (int64 row offsets, int32
// columns, uint32 values: the reference's CsrMatrix<u32>, src/matrices.rs:53-64)
// and builds everything the Krylov kernels read, on the device:
//
//   * validation (offsets non-decreasing, columns in range, values < p), the
//     row and column degrees (src/matrices.rs:842-860 max_nnzs);
//   * the degree orders: rows and columns renumbered by decreasing degree,
//     ties by index (a stable sort of the keys maxdeg - deg);
//   * A in the new order with each row's entries sorted by new column, and its
//     transpose with each row's entries sorted by new row index -- the
//     counting-sort transpose of src/matrices.rs:734-778, stable by row.  Both
//     come from one list of entries keyed (row', col') and (col', row') and
//     sorted by radix sort;
//   * the chunk lists of rows longer than kHeavyDegree.
//
// The two key sorts, the degree-order sorts and the offset scans use CUB
// (DeviceRadixSort, DeviceScan) from the CUDA toolkit; everything else is the
// kernels below.  The result is the same CSR the host build produced.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "rr_internal.h"

namespace rr {

namespace {

constexpr int kBuildThreads = 256;

int build_grid(int64_t work) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((work + kBuildThreads - 1) / kBuildThreads, 148 * 16));
}

int bits_for(uint64_t x) {  // bits needed to hold values in [0, x]
  int b = 1;
  while (b < 64 && (x >> b) != 0) ++b;
  return b;
}

// Row degrees and the check of the offsets: bad[0] = first row whose offsets
// decrease or leave [0, nnz]; maxdeg[0] = largest row degree.
__global__ void row_degrees_kernel(const int64_t* __restrict__ rowptr, int64_t m, int64_t nnz,
                                   uint32_t* __restrict__ rdeg, unsigned long long* bad, unsigned int* maxdeg) {
  unsigned int mx = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = rowptr[r], b = rowptr[r + 1];
    uint32_t d = 0;
    if (a < 0 || b < a || b > nnz) atomicMin(&bad[0], (unsigned long long)r);
    else d = (uint32_t)(b - a);
    rdeg[r] = d;
    mx = max(mx, d);
  }
  for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(&maxdeg[0], mx);
}

// Column degrees (warp-aggregated atomics: Zipf-heavy columns are hit by many
// entries at once) and the checks of columns and values: bad[1] = first entry
// with a column outside [0, n), bad[2] = first entry with a value >= p.
__global__ void col_degrees_kernel(const int32_t* __restrict__ col, const uint32_t* __restrict__ val, int64_t nnz,
                                   int64_t n, uint32_t p, uint32_t* __restrict__ cdeg, unsigned long long* bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t rounds = (nnz + stride - 1) / stride;
  for (int64_t it = 0; it < rounds; ++it) {  // every lane runs every round: full-warp collectives
    const int64_t k = first + it * stride;
    int c = -1;
    if (k < nnz) {
      c = col[k];
      if (c < 0 || c >= n) {
        atomicMin(&bad[1], (unsigned long long)k);
        c = -1;
      }
      if (val[k] >= p) atomicMin(&bad[2], (unsigned long long)k);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, c);
    const int leader = __ffs(peers) - 1;
    if (c >= 0 && (threadIdx.x & 31) == leader) atomicAdd(&cdeg[c], (unsigned)__popc(peers));
  }
}

__global__ void max_kernel(const uint32_t* __restrict__ x, int64_t n, unsigned int* out) {
  unsigned int mx = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    mx = max(mx, x[i]);
  for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// keys[i] = maxd - deg[i] (ascending key = decreasing degree), idx[i] = i.
__global__ void order_keys_kernel(const uint32_t* __restrict__ deg, int64_t n, uint32_t maxd, uint32_t* __restrict__ keys,
                                  int32_t* __restrict__ idx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    keys[i] = maxd - deg[i];
    idx[i] = (int32_t)i;
  }
}

// inv[perm[i]] = i; newdeg[i] = deg[perm[i]].
__global__ void invert_kernel(const int32_t* __restrict__ perm, const uint32_t* __restrict__ deg, int64_t n,
                              int32_t* __restrict__ inv, uint32_t* __restrict__ newdeg) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t o = perm[i];
    inv[o] = (int32_t)i;
    newdeg[i] = deg[o];
  }
}

// One warp per original row: entry k of row r gets the keys
// (row' << bits_n | col') for A and (col' << bits_m | row') for A^T.
__global__ void entry_keys_kernel(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col, int64_t m,
                                  const int32_t* __restrict__ inv_row, const int32_t* __restrict__ inv_col, int bits_n,
                                  int bits_m, uint64_t* __restrict__ keyA, uint64_t* __restrict__ keyT) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = w0; r < m; r += nw) {
    const uint64_t rn = (uint64_t)inv_row[r];
    const int64_t b = rowptr[r + 1];
    for (int64_t k = rowptr[r] + lane; k < b; k += 32) {
      const uint64_t cn = (uint64_t)inv_col[col[k]];
      keyA[k] = (rn << bits_n) | cn;
      keyT[k] = (cn << bits_m) | rn;
    }
  }
}

// cv[i] = (key & mask, value): the packed entries of a sorted key list.
__global__ void pack_kernel(const uint64_t* __restrict__ key, const uint32_t* __restrict__ v, int64_t nnz,
                            uint64_t mask, uint2* __restrict__ cv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x)
    cv[i] = make_uint2((uint32_t)(key[i] & mask), v[i]);
}

// count[0] += rows of degree > kHeavyDegree.
__global__ void count_above_kernel(const uint32_t* __restrict__ deg, int64_t n, uint32_t above, unsigned int* count) {
  unsigned int c = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    c += deg[i] > above;
  for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// pos[r * (P + 1) + j] = first entry of heavy row r whose column is >= j *
// panel (j = 0..P; entries of a row are sorted by column).
__global__ void panel_bounds_kernel(const uint2* __restrict__ cv, const uint32_t* __restrict__ ptr, int64_t heavy,
                                    int P, uint32_t panel, uint32_t* __restrict__ pos) {
  const int64_t total = heavy * (P + 1);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / (P + 1);
    const int j = (int)(e - r * (P + 1));
    uint32_t lo = ptr[r], hi = ptr[r + 1];
    const uint64_t key = (uint64_t)j * panel;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if ((uint64_t)cv[mid].x < key) lo = mid + 1;
      else hi = mid;
    }
    pos[e] = lo;
  }
}

__global__ void chunk_keys_kernel(const uint2* __restrict__ cv, const uint32_t* __restrict__ begin, int64_t nchunks,
                                  uint32_t* __restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nchunks; i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = cv[begin[i]].x;
}

// Stable sort of (key, value) pairs on the first `bits` key bits.
template <class K, class V>
int radix_sort_pairs(const K* kin, K* kout, const V* vin, V* vout, int64_t n, int bits, cudaStream_t s) {
  size_t tmp = 0;
  RR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, (int64_t)n, 0, bits, s));
  DevBuf<unsigned char> t;
  RR_TRY(t.alloc_async(std::max<size_t>(tmp, 1), s));
  RR_CUDA(cub::DeviceRadixSort::SortPairs(t.ptr, tmp, kin, kout, vin, vout, (int64_t)n, 0, bits, s));
  return RR_OK;
}

// out[0] = 0, out[i + 1] = sum of in[0..i].
int offsets_from_degrees(const uint32_t* in, uint32_t* out, int64_t n, cudaStream_t s) {
  RR_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), s));
  if (n == 0) return RR_OK;
  size_t tmp = 0;
  RR_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, in, out + 1, (int64_t)n, s));
  DevBuf<unsigned char> t;
  RR_TRY(t.alloc_async(std::max<size_t>(tmp, 1), s));
  RR_CUDA(cub::DeviceScan::InclusiveSum(t.ptr, tmp, in, out + 1, (int64_t)n, s));
  return RR_OK;
}

// The degree order of n indices by decreasing deg (ties in index order):
// perm[i'] = original index, inv[original] = i', newdeg[i'] = its degree.
int degree_order_device(const uint32_t* deg, int64_t n, uint32_t maxd, DevBuf<int32_t>& perm, DevBuf<int32_t>& inv,
                        DevBuf<uint32_t>& newdeg, cudaStream_t s) {
  DevBuf<uint32_t> kin, kout;
  DevBuf<int32_t> idx;
  RR_TRY(kin.alloc_async(n, s));
  RR_TRY(kout.alloc_async(n, s));
  RR_TRY(idx.alloc_async(n, s));
  RR_TRY(perm.alloc_async(n, s));
  RR_TRY(inv.alloc_async(n, s));
  RR_TRY(newdeg.alloc_async(n, s));
  order_keys_kernel<<<build_grid(n), kBuildThreads, 0, s>>>(deg, n, maxd, kin.ptr, idx.ptr);
  RR_CUDA(cudaGetLastError());
  RR_TRY(radix_sort_pairs(kin.ptr, kout.ptr, idx.ptr, perm.ptr, n, bits_for(maxd), s));
  invert_kernel<<<build_grid(n), kBuildThreads, 0, s>>>(perm.ptr, deg, n, inv.ptr, newdeg.ptr);
  RR_CUDA(cudaGetLastError());
  return RR_OK;
}

// Rows [0, heavy) of d are longer than kHeavyDegree: cut them into chunks of
// at most kChunkNnz entries, ordered (stably) by their first column, so that
// chunks gathering the same region of the input block run together.  A row
// whose chunks would each span more than one panel of kPanelCols columns of
// the input block (rows of at least kPanelDense entries per panel are dense
// enough not to) is first cut at the panel boundaries, as long as its pieces
// keep kMinPiece entries on average: the pieces of different rows that fall in
// one panel then run together and gather from one L2-sized slice of the block.
constexpr uint32_t kPanelCols = 1u << 18;
constexpr int64_t kMinPiece = 64;
constexpr int64_t kPanelDense = 1024;

int build_chunks(DevCsr& d, int64_t heavy, cudaStream_t s) {
  d.heavy_rows = heavy;
  d.nchunks = 0;
  if (heavy == 0) return RR_OK;
  std::vector<uint32_t> ptr(heavy + 1);
  RR_CUDA(cudaMemcpyAsync(ptr.data(), d.rowptr.ptr, (heavy + 1) * 4, cudaMemcpyDeviceToHost, s));
  const int P = (int)std::max<int64_t>(1, (d.cols + kPanelCols - 1) / kPanelCols);
  std::vector<uint32_t> pos;
  if (P > 1) {
    DevBuf<uint32_t> dpos;
    RR_TRY(dpos.alloc_async((size_t)heavy * (P + 1), s));
    panel_bounds_kernel<<<build_grid(heavy * (P + 1)), kBuildThreads, 0, s>>>(d.cv.ptr, d.rowptr.ptr, heavy, P,
                                                                                 kPanelCols, dpos.ptr);
    RR_CUDA(cudaGetLastError());
    pos.resize((size_t)heavy * (P + 1));
    RR_CUDA(cudaMemcpyAsync(pos.data(), dpos.ptr, pos.size() * 4, cudaMemcpyDeviceToHost, s));
  }
  RR_CUDA(cudaStreamSynchronize(s));
  std::vector<uint32_t> row, beg, end;
  auto cut = [&](int64_t r, uint32_t a, uint32_t b) {
    for (uint32_t k = a; k < b; k += (uint32_t)kChunkNnz) {
      row.push_back((uint32_t)r);
      beg.push_back(k);
      end.push_back(std::min<uint32_t>(b, k + (uint32_t)kChunkNnz));
    }
  };
  for (int64_t r = 0; r < heavy; ++r) {
    const int64_t deg = (int64_t)ptr[r + 1] - ptr[r];
    if (P > 1 && deg >= kMinPiece * P && deg < kPanelDense * P) {
      const uint32_t* pr = pos.data() + (size_t)r * (P + 1);
      for (int j = 0; j < P; ++j) cut(r, j == 0 ? ptr[r] : pr[j], j == P - 1 ? ptr[r + 1] : pr[j + 1]);
    } else {
      cut(r, ptr[r], ptr[r + 1]);
    }
  }
  const int64_t nc = (int64_t)row.size();
  DevBuf<uint32_t> dbeg, dkeys;
  RR_TRY(dbeg.alloc_async(nc, s));
  RR_TRY(dkeys.alloc_async(nc, s));
  RR_CUDA(cudaMemcpyAsync(dbeg.ptr, beg.data(), nc * 4, cudaMemcpyHostToDevice, s));
  chunk_keys_kernel<<<build_grid(nc), kBuildThreads, 0, s>>>(d.cv.ptr, dbeg.ptr, nc, dkeys.ptr);
  RR_CUDA(cudaGetLastError());
  std::vector<uint32_t> keys(nc);
  RR_CUDA(cudaMemcpyAsync(keys.data(), dkeys.ptr, nc * 4, cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  std::vector<int64_t> order(nc);
  for (int64_t i = 0; i < nc; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });
  std::vector<uint32_t> cr(nc), cb(nc), ce(nc);
  for (int64_t i = 0; i < nc; ++i) {
    cr[i] = row[order[i]];
    cb[i] = beg[order[i]];
    ce[i] = end[order[i]];
  }
  d.nchunks = nc;
  RR_TRY(d.chunk_row.alloc_async(nc, s));
  RR_TRY(d.chunk_begin.alloc_async(nc, s));
  RR_TRY(d.chunk_end.alloc_async(nc, s));
  RR_CUDA(cudaMemcpyAsync(d.chunk_row.ptr, cr.data(), nc * 4, cudaMemcpyHostToDevice, s));
  RR_CUDA(cudaMemcpyAsync(d.chunk_begin.ptr, cb.data(), nc * 4, cudaMemcpyHostToDevice, s));
  RR_CUDA(cudaMemcpyAsync(d.chunk_end.ptr, ce.data(), nc * 4, cudaMemcpyHostToDevice, s));
  RR_CUDA(cudaStreamSynchronize(s));  // the host vectors die at scope end
  return RR_OK;
}

// Rows of degree above `above` (rows are in decreasing degree order, so these
// are the first ones).
int rows_above(const uint32_t* deg, int64_t n, uint32_t above, cudaStream_t s, int64_t* count) {
  DevBuf<unsigned int> cnt;
  RR_TRY(cnt.alloc_async(1, s));
  RR_CUDA(cudaMemsetAsync(cnt.ptr, 0, 4, s));
  count_above_kernel<<<build_grid(n), kBuildThreads, 0, s>>>(deg, n, above, cnt.ptr);
  RR_CUDA(cudaGetLastError());
  unsigned int h = 0;
  RR_CUDA(cudaMemcpyAsync(&h, cnt.ptr, 4, cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  *count = h;
  return RR_OK;
}

}  // namespace

int matrix_build_device(rr_ctx* ctx, int64_t m, int64_t n, const int64_t* rowptr, const int32_t* col,
                        const uint32_t* val, uint32_t p, rr_matrix* mat) {
  cudaStream_t s = ctx->stream;
  const int64_t nnz = rowptr[m];
  DevBuf<int64_t> d_rowptr;
  DevBuf<int32_t> d_col;
  DevBuf<uint32_t> d_val, rdeg, cdeg;
  DevBuf<unsigned long long> bad;
  DevBuf<unsigned int> maxdeg;
  RR_TRY(d_rowptr.alloc_async(m + 1, s));
  RR_TRY(d_col.alloc_async(std::max<int64_t>(nnz, 1), s));
  RR_TRY(d_val.alloc_async(std::max<int64_t>(nnz, 1), s));
  RR_TRY(rdeg.alloc_async(m, s));
  RR_TRY(cdeg.alloc_async(n, s));
  RR_TRY(bad.alloc_async(3, s));
  RR_TRY(maxdeg.alloc_async(2, s));
  RR_TRY(upload_host(ctx,
                     {{d_rowptr.ptr, rowptr, (size_t)(m + 1) * 8},
                      {d_col.ptr, col, (size_t)nnz * 4},
                      {d_val.ptr, val, (size_t)nnz * 4}},
                     s));
  RR_CUDA(cudaMemsetAsync(bad.ptr, 0xff, 3 * 8, s));
  RR_CUDA(cudaMemsetAsync(maxdeg.ptr, 0, 2 * 4, s));
  RR_CUDA(cudaMemsetAsync(cdeg.ptr, 0, n * 4, s));
  row_degrees_kernel<<<build_grid(m), kBuildThreads, 0, s>>>(d_rowptr.ptr, m, nnz, rdeg.ptr, bad.ptr, maxdeg.ptr);
  RR_CUDA(cudaGetLastError());
  if (nnz) {
    col_degrees_kernel<<<build_grid(nnz), kBuildThreads, 0, s>>>(d_col.ptr, d_val.ptr, nnz, n, p, cdeg.ptr, bad.ptr);
    RR_CUDA(cudaGetLastError());
  }
  max_kernel<<<build_grid(n), kBuildThreads, 0, s>>>(cdeg.ptr, n, maxdeg.ptr + 1);
  RR_CUDA(cudaGetLastError());
  unsigned long long hbad[3];
  unsigned int hmax[2];
  RR_CUDA(cudaMemcpyAsync(hbad, bad.ptr, sizeof(hbad), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaMemcpyAsync(hmax, maxdeg.ptr, sizeof(hmax), cudaMemcpyDeviceToHost, s));
  RR_CUDA(cudaStreamSynchronize(s));
  if (hbad[0] != ~0ull) return fail(RR_EINVAL, "rowptr decreases (or leaves [0, nnz]) at row %llu", hbad[0]);
  if (hbad[1] != ~0ull) return fail(RR_EINVAL, "column index %d out of range at entry %llu", col[hbad[1]], hbad[1]);
  if (hbad[2] != ~0ull)
    return fail(RR_EINVAL, "value %u at entry %llu is not reduced mod p", val[hbad[2]], hbad[2]);
  mat->max_row_nnz = hmax[0];
  mat->max_col_nnz = hmax[1];

  // degree orders
  DevBuf<int32_t> inv_row, inv_col;
  DevBuf<uint32_t> rdeg_new, cdeg_new;
  RR_TRY(degree_order_device(rdeg.ptr, m, hmax[0], mat->d_rowperm, inv_row, rdeg_new, s));
  RR_TRY(degree_order_device(cdeg.ptr, n, hmax[1], mat->d_colperm, inv_col, cdeg_new, s));

  // offsets of A and A^T in the new orders
  DevCsr& A = mat->A;
  DevCsr& At = mat->At;
  A.rows = m, A.cols = n, A.nnz = nnz;
  At.rows = n, At.cols = m, At.nnz = nnz;
  RR_TRY(A.rowptr.alloc_async(m + 1, s));
  RR_TRY(At.rowptr.alloc_async(n + 1, s));
  RR_TRY(offsets_from_degrees(rdeg_new.ptr, A.rowptr.ptr, m, s));
  RR_TRY(offsets_from_degrees(cdeg_new.ptr, At.rowptr.ptr, n, s));
  RR_TRY(A.cv.alloc_async(std::max<int64_t>(nnz, 1), s));
  RR_TRY(At.cv.alloc_async(std::max<int64_t>(nnz, 1), s));
  if (nnz) {
    const int bits_m = bits_for((uint64_t)(m - 1)), bits_n = bits_for((uint64_t)(n - 1));
    DevBuf<uint64_t> keyA, keyT, ksort;
    DevBuf<uint32_t> vsort;
    RR_TRY(keyA.alloc_async(nnz, s));
    RR_TRY(keyT.alloc_async(nnz, s));
    entry_keys_kernel<<<build_grid(m * 32), kBuildThreads, 0, s>>>(d_rowptr.ptr, d_col.ptr, m, inv_row.ptr, inv_col.ptr,
                                                                   bits_n, bits_m, keyA.ptr, keyT.ptr);
    RR_CUDA(cudaGetLastError());
    d_col.release();
    RR_TRY(ksort.alloc_async(nnz, s));
    RR_TRY(vsort.alloc_async(nnz, s));
    // A: rows in the new order, entries of a row by new column
    RR_TRY(radix_sort_pairs(keyA.ptr, ksort.ptr, d_val.ptr, vsort.ptr, nnz, bits_m + bits_n, s));
    pack_kernel<<<build_grid(nnz), kBuildThreads, 0, s>>>(ksort.ptr, vsort.ptr, nnz, (1ull << bits_n) - 1, A.cv.ptr);
    RR_CUDA(cudaGetLastError());
    keyA.release();
    // A^T: columns in the new order, entries by new row (stable by row)
    RR_TRY(radix_sort_pairs(keyT.ptr, ksort.ptr, d_val.ptr, vsort.ptr, nnz, bits_m + bits_n, s));
    pack_kernel<<<build_grid(nnz), kBuildThreads, 0, s>>>(ksort.ptr, vsort.ptr, nnz, (1ull << bits_m) - 1, At.cv.ptr);
    RR_CUDA(cudaGetLastError());
  }
  int64_t heavyA = 0, heavyT = 0;
  RR_TRY(rows_above(rdeg_new.ptr, m, (uint32_t)kHeavyDegree, s, &heavyA));
  RR_TRY(rows_above(cdeg_new.ptr, n, (uint32_t)kHeavyDegree, s, &heavyT));
  RR_TRY(rows_above(rdeg_new.ptr, m, 0u, s, &A.live_rows));
  RR_TRY(rows_above(cdeg_new.ptr, n, 0u, s, &At.live_rows));
  RR_TRY(build_chunks(A, heavyA, s));
  RR_TRY(build_chunks(At, heavyT, s));
  RR_CUDA(cudaStreamSynchronize(s));
  return RR_OK;
}

}  // namespace rr
