// tensor.cu -- block-sparse tensor storage on the device.
//
// Layout (the reference's single-rank layout, src/Tensor/BaseTensor.cpp:117-251): blocks are
// identified by the column-major rolled id over the block grid, stored sorted by id, each
// block dense and column-major, packed back to back in one pool allocation; offsets[] is the
// running element count in id order.  Device side keeps ids (int64), offsets (int64) and the
// per-block extents dims[b*order + d] (int32) that the contraction kernels read.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <cmath>
#include <numeric>

#include "device_common.cuh"

namespace sht {

TensorMeta make_meta(const sht_tensor* t) {
  TensorMeta m{};
  m.order = t->order;
  int pos = 0;
  for (int d = 0; d < t->order; ++d) {
    m.nblk[d] = t->nblk[d];
    m.bstart[d] = pos;
    m.gstride[d] = t->gstride[d];
    pos += t->nblk[d];
  }
  m.bsizes = t->d_bsizes.as<int>();
  return m;
}

int64_t block_size_of(const sht_tensor* t, int64_t id) {
  int64_t s = 1;
  for (int d = 0; d < t->order; ++d) s *= t->bs[d][(id / t->gstride[d]) % t->nblk[d]];
  return s;
}

// per-block extents and element counts from ids
__global__ void k_block_dims(TensorMeta m, const long long* __restrict__ ids, long long n,
                             int* __restrict__ dims, long long* __restrict__ sizes) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n;
       b += (long long)gridDim.x * blockDim.x) {
    int c[kMaxOrder];
    const long long id = ids[b];
    unroll_block(m, id >= 0 ? id : -(id + 1), c);  // filter marks a block as -(id)-1
    long long s = 1;
    for (int d = 0; d < m.order; ++d) {
      const int e = m.bsizes[m.bstart[d] + c[d]];
      dims[b * m.order + d] = e;
      s *= e;
    }
    if (sizes) sizes[b] = s;
  }
}

void block_dims_sizes(const sht_tensor* t, const long long* ids, long long n, int* dims, long long* sizes,
                      cudaStream_t s) {
  if (n <= 0) return;
  k_block_dims<<<grid_for(n, 256), 256, 0, s>>>(make_meta(t), ids, n, dims, sizes);
  SHT_CUDA(cudaGetLastError());
}

// Host-built index (reserve): ids sorted and unique on the host.
void tensor_set_index(sht_tensor* t, std::vector<int64_t>&& ids, cudaStream_t s) {
  DevicePool* pool = t->ctx->pool.get();
  t->ids = std::move(ids);
  t->has_marked = false;
  {
    std::lock_guard<std::mutex> lk(t->hmu);
    t->hdims_valid = false;
  }
  t->nblocks = static_cast<int64_t>(t->ids.size());
  t->offsets.resize(t->ids.size());
  int64_t off = 0;
  for (size_t i = 0; i < t->ids.size(); ++i) { t->offsets[i] = off; off += block_size_of(t, t->ids[i]); }
  t->nnz = off;
  t->rows.assign(t->nblk[0], 0);
  {
    std::vector<int64_t> cnt(t->nblk[0], 0);
    for (int64_t id : t->ids) cnt[id % t->nblk[0]]++;
    int64_t acc = 0;
    for (int r = 0; r < t->nblk[0]; ++r) { t->rows[r] = acc; acc += cnt[r]; }
  }
  t->host_stale = false;
  t->d_ids = PoolBuf(pool, std::max<int64_t>(t->nblocks, 1) * 8, s);
  t->d_offsets = PoolBuf(pool, std::max<int64_t>(t->nblocks, 1) * 8, s);
  t->d_dims = PoolBuf(pool, std::max<int64_t>(t->nblocks, 1) * t->order * 4, s);
  t->d_data = PoolBuf(pool, std::max<int64_t>(t->nnz, 1) * t->esize(), s);
  if (t->nblocks) {
    SHT_CUDA(cudaMemcpyAsync(t->d_ids.ptr, t->ids.data(), t->nblocks * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(t->d_offsets.ptr, t->offsets.data(), t->nblocks * 8, cudaMemcpyHostToDevice, s));
    k_block_dims<<<grid_for(t->nblocks, 256), 256, 0, s>>>(make_meta(t), t->d_ids.as<long long>(),
                                                          t->nblocks, t->d_dims.as<int>(), nullptr);
    SHT_CUDA(cudaGetLastError());
  }
  SHT_CUDA(cudaMemsetAsync(t->d_data.ptr, 0, std::max<int64_t>(t->nnz, 1) * t->esize(), s));
  // the host vectors above are pageable: the copies complete before return
  SHT_CUDA(cudaStreamSynchronize(s));
}

static void host_index_arrays(sht_tensor* t) {
  std::lock_guard<std::mutex> lk(t->hmu);
  if (t->hdims_valid) return;
  const size_t n = std::max<size_t>(t->ids.size() * t->order, 1);
  t->hdims.resize(n);
  t->hcoords.resize(n);
  for (size_t b = 0; b < t->ids.size(); ++b) {
    const int64_t id = t->ids[b] >= 0 ? t->ids[b] : -(t->ids[b] + 1);  // marked ids are -(id)-1
    for (int d = 0; d < t->order; ++d) {
      const int x = (int)((id / t->gstride[d]) % t->nblk[d]);
      t->hcoords[b * t->order + d] = x;
      t->hdims[b * t->order + d] = t->bs[d][x];
    }
  }
  t->hdims_valid = true;
}

const int* tensor_host_dims(sht_tensor* t) {
  host_index_arrays(t);
  return t->hdims.data();
}

const int* tensor_host_coords(sht_tensor* t) {
  host_index_arrays(t);
  return t->hcoords.data();
}

// ---------------------------------------------------------------------------------------
// reserve from index lists already on the device (BaseTensor::reserve, BaseTensor.cpp:117-251,
// with the ids, their sort and the offsets built on the GPU)
// ---------------------------------------------------------------------------------------
// idx is mode-major (idx[d * n + b]) like sht_tensor_reserve's host lists.  Bad entries set bit 0
// of *bad and give id 0 (the build is then abandoned).
__global__ void k_ids_from_lists(TensorMeta m, const int* __restrict__ idx, long long n, long long* __restrict__ ids,
                                 int* __restrict__ bad) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    long long id = 0;
    bool ok = true;
    for (int d = 0; d < m.order; ++d) {
      const int v = idx[(long long)d * n + b];
      if (v < 0 || v >= m.nblk[d]) ok = false;
      else id += (long long)v * m.gstride[d];
    }
    if (!ok) {
      atomicOr(bad, 1);
      id = 0;
    }
    ids[b] = id;
  }
}

// On the sorted ids: bit 1 for a repeated id, bit 2 for a block of 2^31 elements or more; the
// last thread also leaves the element count (offset + size of the last block) in *nnz.
__global__ void k_reserve_checks(const long long* __restrict__ ids, const long long* __restrict__ sizes,
                                 const long long* __restrict__ offs, long long n, int* __restrict__ bad,
                                 long long* __restrict__ nnz) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    if (b > 0 && ids[b] == ids[b - 1]) atomicOr(bad, 2);
    if (sizes[b] >= (1LL << 31)) atomicOr(bad, 4);
    if (b == n - 1) *nnz = offs[b] + sizes[b];
  }
}

void tensor_reserve_device(sht_tensor* t, long long n, const int* d_idx, cudaStream_t s) {
  if (n < 0 || (n > 0 && !d_idx)) fail(SHT_ERR_INVALID, "bad index list");
  if (n > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "reserve: more than 2^31 blocks");
  DevicePool* pool = t->ctx->pool.get();
  tensor_touch(t, s);
  const long long nn = std::max(n, 1LL);
  PoolBuf ids(pool, nn * 8, s), sorted(pool, nn * 8, s), dims(pool, nn * t->order * 4, s), sizes(pool, nn * 8, s),
      offs(pool, nn * 8, s), word(pool, 16, s);
  SHT_CUDA(cudaMemsetAsync(word.ptr, 0, 16, s));
  const TensorMeta m = make_meta(t);
  if (n > 0) {
    k_ids_from_lists<<<grid_for(n, 256), 256, 0, s>>>(m, d_idx, n, ids.as<long long>(), word.as<int>());
    SHT_CUDA(cudaGetLastError());
    long double grid = 1;
    for (int d = 0; d < t->order; ++d) grid *= t->nblk[d];
    int bits = 1;
    while (bits < 63 && (long double)(1ULL << bits) < grid) ++bits;
    size_t tb = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, ids.as<long long>(), sorted.as<long long>(), (int)n, 0, bits, s);
    {
      PoolBuf tmp(pool, tb, s);
      cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, ids.as<long long>(), sorted.as<long long>(), (int)n, 0, bits, s);
    }
    k_block_dims<<<grid_for(n, 256), 256, 0, s>>>(m, sorted.as<long long>(), n, dims.as<int>(), sizes.as<long long>());
    SHT_CUDA(cudaGetLastError());
    cub::DeviceScan::ExclusiveSum(nullptr, tb, sizes.as<long long>(), offs.as<long long>(), (int)n, s);
    {
      PoolBuf tmp(pool, tb, s);
      cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, sizes.as<long long>(), offs.as<long long>(), (int)n, s);
    }
    k_reserve_checks<<<grid_for(n, 256), 256, 0, s>>>(sorted.as<long long>(), sizes.as<long long>(),
                                                      offs.as<long long>(), n, word.as<int>(),
                                                      word.as<long long>() + 1);
    SHT_CUDA(cudaGetLastError());
  }
  long long h[2] = {0, 0};
  SHT_CUDA(cudaMemcpyAsync(h, word.ptr, 16, cudaMemcpyDeviceToHost, s));  // pageable: returns when done
  const int bad = (int)(h[0] & 0xffffffff);
  if (bad & 1) fail(SHT_ERR_INVALID, "reserve: block index out of range");
  if (bad & 2) fail(SHT_ERR_INVALID, "reserve: duplicate block index");
  if (bad & 4) fail(SHT_ERR_UNSUPPORTED, "block above 2^31 elements");
  const long long nnz = h[1];
  t->d_ids = std::move(sorted);
  t->d_offsets = std::move(offs);
  t->d_dims = std::move(dims);
  t->d_data = PoolBuf(pool, std::max(nnz, 1LL) * t->esize(), s);
  SHT_CUDA(cudaMemsetAsync(t->d_data.ptr, 0, std::max(nnz, 1LL) * t->esize(), s));
  // the zero fill is done before the call returns, as for the host reserve: a later upload on
  // another stream cannot be overtaken by it
  SHT_CUDA(cudaStreamSynchronize(s));
  t->nblocks = n;
  t->nnz = nnz;
  t->host_stale = true;  // the host mirror is read back when a host-side step needs it
}

void tensor_touch(sht_tensor* t, cudaStream_t s) {
  for (PoolBuf* b : {&t->d_bsizes, &t->d_bstart, &t->d_ids, &t->d_offsets, &t->d_dims, &t->d_data}) b->use_on(s);
}

// Pull the device index back to the host mirror when a device-side operation rebuilt it.
void tensor_sync_host(sht_tensor* t, cudaStream_t s) {
  if (!t->host_stale) return;
  {
    std::lock_guard<std::mutex> lk(t->hmu);
    t->hdims_valid = false;
  }
  t->ids.resize(t->nblocks);
  t->offsets.resize(t->nblocks);
  if (t->nblocks) {
    SHT_CUDA(cudaMemcpyAsync(t->ids.data(), t->d_ids.ptr, t->nblocks * 8, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaMemcpyAsync(t->offsets.data(), t->d_offsets.ptr, t->nblocks * 8, cudaMemcpyDeviceToHost, s));
  }
  SHT_CUDA(cudaStreamSynchronize(s));
  t->rows.assign(t->nblk[0], 0);
  std::vector<int64_t> cnt(t->nblk[0], 0);
  bool marked = false;
  for (int64_t id : t->ids) {
    marked = marked || id < 0;
    cnt[(id >= 0 ? id : -(id + 1)) % t->nblk[0]]++;  // marked ids are -(id)-1
  }
  t->has_marked = marked;
  int64_t acc = 0;
  for (int r = 0; r < t->nblk[0]; ++r) { t->rows[r] = acc; acc += cnt[r]; }
  t->host_stale = false;
}

// ---------------------------------------------------------------------------------------
// Block norms (BlockSpan::get_norm, src/Basics/BlockSpan.h:140-164).
// FROBENIUS and MAXABS are evaluated in a fixed order that parallelises within a block, so
// that a block of millions of elements is spread over many CTAs while the CPU restatement
// still reproduces the result bit for bit:
//   the block's n elements are cut into chunks of kNormChunk = 4096 consecutive elements;
//   in chunk c, lane j (0..127) folds elements c*4096 + j + 128*i, i = 0, 1, ... ascending
//   (FROBENIUS: p = fma(v, v, p); MAXABS: p = max(p, |v|));
//   the 128 lane values are halved in place, p[j] op= p[j + h] for h = 64, 32, ..., 1;
//   the chunk results are folded in ascending chunk order, starting from chunk 0;
//   FROBENIUS takes a correctly rounded sqrt at the end.
// REFCOMPAT evaluates the reference's int accumulator (acc = int(acc + v*v)) sequentially,
// one thread per block, as the reference does.
// ---------------------------------------------------------------------------------------
constexpr int kNormChunk = 4096;
constexpr int kNormLanes = 128;

__global__ void k_norm_chunk_counts(const int* __restrict__ dims, int order, long long n,
                                    long long* __restrict__ nchunks) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    long long sz = 1;
    for (int d = 0; d < order; ++d) sz *= dims[b * order + d];
    nchunks[b] = (sz + kNormChunk - 1) / kNormChunk;
  }
}

// one 128-thread CTA per chunk (grid-stride); chunk -> block by binary search on the starts
template <typename T>
__global__ void __launch_bounds__(kNormLanes) k_norm_chunks(const T* __restrict__ data,
                                                            const long long* __restrict__ offsets,
                                                            const int* __restrict__ dims, int order, long long n,
                                                            const long long* __restrict__ cstart,
                                                            const long long* __restrict__ nchunks, int maxabs,
                                                            double* __restrict__ partial) {
  __shared__ double red[kNormLanes];
  const int j = threadIdx.x;
  const long long total = cstart[n - 1] + nchunks[n - 1];
  for (long long c = blockIdx.x; c < total; c += gridDim.x) {
    long long lo = 0, hi = n - 1;  // last block whose first chunk <= c
    while (lo < hi) {
      const long long mid = (lo + hi + 1) >> 1;
      if (cstart[mid] <= c) lo = mid; else hi = mid - 1;
    }
    long long sz = 1;
    for (int d = 0; d < order; ++d) sz *= dims[lo * order + d];
    const long long base = (c - cstart[lo]) * kNormChunk;
    const long long end = min(sz, base + kNormChunk);
    const T* p = data + offsets[lo];
    double r = 0.0;
    long long e = base + j;
    // eight loads in flight per thread, folded in the same element order as one at a time
    for (; e + 7 * kNormLanes < end; e += 8 * kNormLanes) {
      T x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) x[u] = p[e + u * kNormLanes];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const double v = (double)x[u];
        r = maxabs ? fmax(r, fabs(v)) : __fma_rn(v, v, r);
      }
    }
    for (; e < end; e += kNormLanes) {
      const double v = (double)p[e];
      r = maxabs ? fmax(r, fabs(v)) : __fma_rn(v, v, r);
    }
    red[j] = r;
    __syncthreads();
    for (int h = kNormLanes / 2; h >= 1; h >>= 1) {
      if (j < h) red[j] = maxabs ? fmax(red[j], red[j + h]) : __dadd_rn(red[j], red[j + h]);
      __syncthreads();
    }
    if (j == 0) partial[c] = red[0];
    __syncthreads();
  }
}

__global__ void k_norm_finish(const long long* __restrict__ cstart, const long long* __restrict__ nchunks, long long n,
                              const double* __restrict__ partial, int maxabs, double* __restrict__ out) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    const long long c0 = cstart[b], nc = nchunks[b];
    double r = 0.0;
    for (long long c = 0; c < nc; ++c) {
      const double v = partial[c0 + c];
      r = c == 0 ? v : (maxabs ? fmax(r, v) : __dadd_rn(r, v));
    }
    out[b] = maxabs ? r : sqrt(r);
  }
}

template <typename T>
__global__ void k_norm_refcompat(const T* __restrict__ data, const long long* __restrict__ offsets,
                                 const int* __restrict__ dims, int order, long long n, double* __restrict__ out) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    long long sz = 1;
    for (int d = 0; d < order; ++d) sz *= dims[b * order + d];
    const T* p = data + offsets[b];
    int acc = 0;
    for (long long e = 0; e < sz; ++e) {
      const double v = (double)p[e];
      acc = (int)__dadd_rn((double)acc, __dmul_rn(v, v));
    }
    out[b] = sqrt((double)acc);
  }
}

template <typename T>
static void norms_typed(sht_tensor* t, sht_norm norm, double* d_out, cudaStream_t s) {
  const T* data = t->d_data.as<T>();
  const long long n = t->nblocks;
  const long long* offs = t->d_offsets.as<long long>();
  const int* dims = t->d_dims.as<int>();
  if (norm == SHT_NORM_FROBENIUS_REFCOMPAT) {
    k_norm_refcompat<T><<<grid_for(n, 128), 128, 0, s>>>(data, offs, dims, t->order, n, d_out);
    SHT_CUDA(cudaGetLastError());
    return;
  }
  DevicePool* pool = t->ctx->pool.get();
  PoolBuf cnt(pool, n * 8, s), start(pool, n * 8, s);
  k_norm_chunk_counts<<<grid_for(n, 256), 256, 0, s>>>(dims, t->order, n, cnt.as<long long>());
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<long long>(), start.as<long long>(), (int)n, s);
  {
    PoolBuf tmp(pool, tb, s);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, cnt.as<long long>(), start.as<long long>(), (int)n, s);
  }
  // every block has at most sz/4096 + 1 chunks: the total is bounded without reading it back
  const long long bound = t->nnz / kNormChunk + n;
  PoolBuf partial(pool, std::max(bound, 1LL) * 8, s);
  const int maxabs = norm == SHT_NORM_MAXABS;
  const int grid = (int)std::min<long long>(bound, (long long)t->ctx->num_sms * 16);
  k_norm_chunks<T><<<grid, kNormLanes, 0, s>>>(data, offs, dims, t->order, n, start.as<long long>(),
                                               cnt.as<long long>(), maxabs, partial.as<double>());
  k_norm_finish<<<grid_for(n, 128), 128, 0, s>>>(start.as<long long>(), cnt.as<long long>(), n,
                                                 partial.as<double>(), maxabs, d_out);
  SHT_CUDA(cudaGetLastError());
}

void tensor_norms_device(sht_tensor* t, sht_norm norm, double* d_out, cudaStream_t s) {
  if (t->nblocks == 0) return;
  tensor_touch(t, s);
  if (t->dtype == SHT_F64)
    norms_typed<double>(t, norm, d_out, s);
  else
    norms_typed<float>(t, norm, d_out, s);
}

// ---------------------------------------------------------------------------------------
// filter / compress (Tensor::filter, src/Tensor/Tensor.h:337-363; BaseTensor::compress,
// src/Tensor/BaseTensor.cpp:253-354).  Marking writes -(id)-1 into the id like the
// reference.  Compaction keeps unmarked blocks in id order and moves each block's real
// extent (the reference multiplies into a block size initialised to 0, :283-288).
// ---------------------------------------------------------------------------------------
__global__ void k_mark(long long* ids, const double* norms, long long n, double eps) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x)
    if (ids[b] >= 0 && norms[b] < eps) ids[b] = -ids[b] - 1;
}

__global__ void k_keep_flags(const long long* ids, const long long* sizes, long long n, int* keep,
                             long long* keep_sizes) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    keep[b] = ids[b] >= 0;
    keep_sizes[b] = ids[b] >= 0 ? sizes[b] : 0;
  }
}

// one CTA per old block: copy kept blocks to their new offsets
template <typename T>
__global__ void k_compact(const T* __restrict__ src, T* __restrict__ dst, const long long* ids,
                          const long long* old_off, const long long* new_off, const long long* sizes,
                          const int* new_pos, long long n, long long* out_ids, long long* out_off) {
  for (long long b = blockIdx.x; b < n; b += gridDim.x) {
    if (ids[b] < 0) continue;
    const long long s = sizes[b];
    const T* p = src + old_off[b];
    T* q = dst + new_off[b];
    for (long long e = threadIdx.x; e < s; e += blockDim.x) q[e] = p[e];
    if (threadIdx.x == 0) {
      out_ids[new_pos[b]] = ids[b];
      out_off[new_pos[b]] = new_off[b];
    }
  }
}

void tensor_compress_device(sht_tensor* t, cudaStream_t s) {
  DevicePool* pool = t->ctx->pool.get();
  tensor_touch(t, s);
  const long long n = t->nblocks;
  if (n == 0) return;
  PoolBuf sizes(pool, n * 8, s), keep(pool, n * 4, s), keep_sizes(pool, n * 8, s), pos(pool, n * 4, s),
      new_off(pool, n * 8, s);
  {
    PoolBuf dims(pool, n * t->order * 4, s);
    k_block_dims<<<grid_for(n, 256), 256, 0, s>>>(make_meta(t), t->d_ids.as<long long>(), n, dims.as<int>(),
                                                  sizes.as<long long>());
  }
  k_keep_flags<<<grid_for(n, 256), 256, 0, s>>>(t->d_ids.as<long long>(), sizes.as<long long>(), n,
                                                 keep.as<int>(), keep_sizes.as<long long>());
  size_t tb1 = 0, tb2 = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb1, keep.as<int>(), pos.as<int>(), (int)n, s);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, keep_sizes.as<long long>(), new_off.as<long long>(), (int)n, s);
  PoolBuf tmp(pool, std::max(tb1, tb2), s);
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb1, keep.as<int>(), pos.as<int>(), (int)n, s);
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb2, keep_sizes.as<long long>(), new_off.as<long long>(), (int)n, s);
  int last_pos = 0, last_keep = 0;
  long long last_off = 0, last_size = 0;
  SHT_CUDA(cudaMemcpyAsync(&last_pos, pos.as<int>() + n - 1, 4, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaMemcpyAsync(&last_keep, keep.as<int>() + n - 1, 4, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaMemcpyAsync(&last_off, new_off.as<long long>() + n - 1, 8, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaMemcpyAsync(&last_size, keep_sizes.as<long long>() + n - 1, 8, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  const long long nkeep = last_pos + last_keep;
  const long long nnz = last_off + last_size;
  PoolBuf nids(pool, std::max(nkeep, 1LL) * 8, s), noffs(pool, std::max(nkeep, 1LL) * 8, s),
      ndata(pool, std::max(nnz, 1LL) * t->esize(), s);
  const int grid = (int)std::min<long long>(n, (long long)t->ctx->num_sms * 8);
  if (t->dtype == SHT_F64)
    k_compact<double><<<grid, 256, 0, s>>>(t->d_data.as<double>(), ndata.as<double>(), t->d_ids.as<long long>(),
                                           t->d_offsets.as<long long>(), new_off.as<long long>(), sizes.as<long long>(),
                                           pos.as<int>(), n, nids.as<long long>(), noffs.as<long long>());
  else
    k_compact<float><<<grid, 256, 0, s>>>(t->d_data.as<float>(), ndata.as<float>(), t->d_ids.as<long long>(),
                                          t->d_offsets.as<long long>(), new_off.as<long long>(), sizes.as<long long>(),
                                          pos.as<int>(), n, nids.as<long long>(), noffs.as<long long>());
  SHT_CUDA(cudaGetLastError());
  PoolBuf ndims(pool, std::max(nkeep, 1LL) * t->order * 4, s);
  if (nkeep)
    k_block_dims<<<grid_for(nkeep, 256), 256, 0, s>>>(make_meta(t), nids.as<long long>(), nkeep, ndims.as<int>(), nullptr);
  t->d_ids = std::move(nids);
  t->d_offsets = std::move(noffs);
  t->d_data = std::move(ndata);
  t->d_dims = std::move(ndims);
  t->nblocks = nkeep;
  t->nnz = nnz;
  t->host_stale = true;
  tensor_sync_host(t, s);
}

void tensor_filter_device(sht_tensor* t, double eps, sht_norm norm, int compress, cudaStream_t s) {
  DevicePool* pool = t->ctx->pool.get();
  const long long n = t->nblocks;
  if (n == 0) return;
  PoolBuf norms(pool, n * 8, s);
  tensor_norms_device(t, norm, norms.as<double>(), s);
  k_mark<<<grid_for(n, 256), 256, 0, s>>>(t->d_ids.as<long long>(), norms.as<double>(), n, eps);
  SHT_CUDA(cudaGetLastError());
  t->host_stale = true;
  if (compress) {
    tensor_compress_device(t, s);
  } else {
    tensor_sync_host(t, s);
  }
}

// ---------------------------------------------------------------------------------------
// Error of X against Ref over the same block pattern: max |x - r|, sum (x-r)^2, sum r^2, and the
// number of elements whose bit patterns differ (signed zeros and NaN payloads count).
// ---------------------------------------------------------------------------------------
__global__ void k_compare(const double* __restrict__ x, const double* __restrict__ r, long long n,
                          unsigned long long* __restrict__ maxbits, double* __restrict__ sums,
                          unsigned long long* __restrict__ ndiff) {
  double mx = 0.0, d2 = 0.0, r2 = 0.0;
  unsigned long long nd = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double xi = x[i], ri = r[i];
    const double d = xi - ri;
    mx = fmax(mx, fabs(d));
    d2 = fma(d, d, d2);
    r2 = fma(ri, ri, r2);
    nd += __double_as_longlong(xi) != __double_as_longlong(ri);
  }
  for (int off = 16; off >= 1; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    d2 += __shfl_down_sync(0xffffffffu, d2, off);
    r2 += __shfl_down_sync(0xffffffffu, r2, off);
    nd += __shfl_down_sync(0xffffffffu, nd, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));  // non-negative: bit order = value order
    atomicAdd(&sums[0], d2);
    atomicAdd(&sums[1], r2);
    atomicAdd(ndiff, nd);
  }
}

void tensor_compare_device(sht_tensor* X, sht_tensor* R, double* max_abs, double* rel_fro, long long* ndiff,
                           cudaStream_t s) {
  tensor_sync_host(X, s);
  tensor_sync_host(R, s);
  if (X->dtype != SHT_F64 || R->dtype != SHT_F64) fail(SHT_ERR_UNSUPPORTED, "compare runs on FP64 tensors");
  if (X->ids != R->ids || X->nnz != R->nnz) fail(SHT_ERR_SIZE, "compare needs the same block pattern");
  PoolBuf acc(X->ctx->pool.get(), 64, s);
  SHT_CUDA(cudaMemsetAsync(acc.ptr, 0, 64, s));
  if (X->nnz)
    k_compare<<<grid_for(X->nnz, 256, X->ctx->num_sms * 8), 256, 0, s>>>(
        X->d_data.as<double>(), R->d_data.as<double>(), X->nnz, acc.as<unsigned long long>(), acc.as<double>() + 1,
        acc.as<unsigned long long>() + 3);
  SHT_CUDA(cudaGetLastError());
  double h[4];
  SHT_CUDA(cudaMemcpyAsync(h, acc.ptr, 32, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  unsigned long long nd;
  std::memcpy(&nd, &h[3], 8);
  if (max_abs) *max_abs = h[0];
  if (rel_fro) *rel_fro = h[2] > 0 ? std::sqrt(h[1] / h[2]) : std::sqrt(h[1]);
  if (ndiff) *ndiff = (long long)nd;
}

}  // namespace sht
