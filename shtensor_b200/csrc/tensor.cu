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

void tensor_touch(sht_tensor* t, cudaStream_t s) {
  for (PoolBuf* b : {&t->d_bsizes, &t->d_bstart, &t->d_ids, &t->d_offsets, &t->d_dims, &t->d_data}) b->use_on(s);
}

// Pull the device index back to the host mirror when a device-side operation rebuilt it.
void tensor_sync_host(sht_tensor* t, cudaStream_t s) {
  if (!t->host_stale) return;
  t->ids.resize(t->nblocks);
  t->offsets.resize(t->nblocks);
  if (t->nblocks) {
    SHT_CUDA(cudaMemcpyAsync(t->ids.data(), t->d_ids.ptr, t->nblocks * 8, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaMemcpyAsync(t->offsets.data(), t->d_offsets.ptr, t->nblocks * 8, cudaMemcpyDeviceToHost, s));
  }
  SHT_CUDA(cudaStreamSynchronize(s));
  t->rows.assign(t->nblk[0], 0);
  std::vector<int64_t> cnt(t->nblk[0], 0);
  for (int64_t id : t->ids) cnt[(id >= 0 ? id : -(id + 1)) % t->nblk[0]]++;  // marked ids are -(id)-1
  int64_t acc = 0;
  for (int r = 0; r < t->nblk[0]; ++r) { t->rows[r] = acc; acc += cnt[r]; }
  t->host_stale = false;
}

// ---------------------------------------------------------------------------------------
// Block norms (BlockSpan::get_norm, src/Basics/BlockSpan.h:140-164).  One warp per block.
// FROBENIUS: lane l accumulates fma(v,v,acc) over elements l, l+32, ... in ascending order,
// then a shuffle-down tree (16, 8, 4, 2, 1) and a correctly rounded sqrt: a fixed order,
// so the CPU restatement reproduces it bit for bit.  MAXABS is order-free.  REFCOMPAT
// evaluates the reference's int accumulator (acc = int(acc + v*v)) sequentially on lane 0.
// ---------------------------------------------------------------------------------------
template <typename T>
__global__ void k_block_norms(const T* __restrict__ data, const long long* __restrict__ offsets,
                              const int* __restrict__ dims, int order, long long n, int norm,
                              double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long b = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); b < n; b += warps) {
    long long sz = 1;
    for (int d = 0; d < order; ++d) sz *= dims[b * order + d];
    const T* p = data + offsets[b];
    double r = 0.0;
    if (norm == SHT_NORM_MAXABS) {
      for (long long e = lane; e < sz; e += 32) r = fmax(r, fabs((double)p[e]));
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, off));
    } else if (norm == SHT_NORM_FROBENIUS) {
      for (long long e = lane; e < sz; e += 32) {
        const double v = (double)p[e];
        r = __fma_rn(v, v, r);
      }
#pragma unroll
      for (int off = 16; off >= 1; off >>= 1) r = __dadd_rn(r, __shfl_down_sync(0xffffffffu, r, off));
      r = sqrt(r);
    } else {
      if (lane == 0) {
        int acc = 0;
        for (long long e = 0; e < sz; ++e) {
          const double v = (double)p[e];
          acc = (int)__dadd_rn((double)acc, __dmul_rn(v, v));
        }
        r = sqrt((double)acc);
      }
    }
    if (lane == 0) out[b] = r;
  }
}

void tensor_norms_device(sht_tensor* t, sht_norm norm, double* d_out, cudaStream_t s) {
  if (t->nblocks == 0) return;
  tensor_touch(t, s);
  const int threads = 256;
  const int grid = grid_for(t->nblocks * 32, threads, t->ctx->num_sms * 16);
  if (t->dtype == SHT_F64)
    k_block_norms<double><<<grid, threads, 0, s>>>(t->d_data.as<double>(), t->d_offsets.as<long long>(),
                                                   t->d_dims.as<int>(), t->order, t->nblocks, (int)norm, d_out);
  else
    k_block_norms<float><<<grid, threads, 0, s>>>(t->d_data.as<float>(), t->d_offsets.as<long long>(),
                                                  t->d_dims.as<int>(), t->order, t->nblocks, (int)norm, d_out);
  SHT_CUDA(cudaGetLastError());
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
// Error of X against Ref over the same block pattern: max |x - r|, sum (x-r)^2, sum r^2.
// ---------------------------------------------------------------------------------------
__global__ void k_compare(const double* __restrict__ x, const double* __restrict__ r, long long n,
                          unsigned long long* __restrict__ maxbits, double* __restrict__ sums) {
  double mx = 0.0, d2 = 0.0, r2 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = x[i] - r[i];
    mx = fmax(mx, fabs(d));
    d2 = fma(d, d, d2);
    r2 = fma(r[i], r[i], r2);
  }
  for (int off = 16; off >= 1; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    d2 += __shfl_down_sync(0xffffffffu, d2, off);
    r2 += __shfl_down_sync(0xffffffffu, r2, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));  // non-negative: bit order = value order
    atomicAdd(&sums[0], d2);
    atomicAdd(&sums[1], r2);
  }
}

void tensor_compare_device(sht_tensor* X, sht_tensor* R, double* max_abs, double* rel_fro, cudaStream_t s) {
  tensor_sync_host(X, s);
  tensor_sync_host(R, s);
  if (X->dtype != SHT_F64 || R->dtype != SHT_F64) fail(SHT_ERR_UNSUPPORTED, "compare runs on FP64 tensors");
  if (X->ids != R->ids || X->nnz != R->nnz) fail(SHT_ERR_SIZE, "compare needs the same block pattern");
  PoolBuf acc(X->ctx->pool.get(), 64, s);
  SHT_CUDA(cudaMemsetAsync(acc.ptr, 0, 64, s));
  if (X->nnz)
    k_compare<<<grid_for(X->nnz, 256, X->ctx->num_sms * 8), 256, 0, s>>>(
        X->d_data.as<double>(), R->d_data.as<double>(), X->nnz, acc.as<unsigned long long>(), acc.as<double>() + 1);
  SHT_CUDA(cudaGetLastError());
  double h[3];
  SHT_CUDA(cudaMemcpyAsync(h, acc.ptr, 24, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  unsigned long long bits;
  std::memcpy(&bits, &h[0], 8);
  if (max_abs) *max_abs = h[0];
  if (rel_fro) *rel_fro = h[2] > 0 ? std::sqrt(h[1] / h[2]) : std::sqrt(h[1]);
}

}  // namespace sht
