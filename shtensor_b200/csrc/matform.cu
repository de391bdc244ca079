// matform.cu -- per-block permute into matrix form (the reference's Utils::reshape step).
//
// The LAPACK path of the reference reshapes every block to (rows || cols) order before its
// GEMM (src/Kernel/KernelImpl.cpp:171-173 with src/Basics/Utils.h:315-359).  Here each stored
// block of an operand is written once per execute into a padded, 16-byte aligned matrix:
//   A block: m_pad x K4, column-major (rows = A's free modes, first listed fastest), the
//            element scaled by alpha (the XMM kernel's a*alpha), K padding = -0.0;
//   B block: n_pad x K4 with columns fastest (columns = B's free modes), K padding = +0.0;
// m_pad/n_pad are the free extents rounded up to even, K4 the contracted extent rounded up to
// 4, so the tile kernel copies 16-byte pairs and multiplies whole m8n8k4 steps.  One CTA per
// block: the free/contracted offsets of the block are tabulated in shared memory, then
// warps walk k and lanes walk rows, so stores are contiguous.
#include <algorithm>

#include "contract.h"
#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

constexpr int kMatTab = 4096;  // table entries per dimension held in shared memory

__global__ void __launch_bounds__(256) k_matform(const double* __restrict__ src, const long long* __restrict__ src_off,
                                                 const int* __restrict__ dims, int order, ModeMap fm, ModeMap km,
                                                 const long long* __restrict__ dst_off, const int* __restrict__ ld,
                                                 double* __restrict__ dst, double scale, int scale_on, double kpad,
                                                 long long nblocks) {
  __shared__ int fo[kMatTab], ko[kMatTab];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (long long b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int* d = dims + b * order;
    int st[kMaxOrder];
    block_strides(d, order, st);
    int m = 1, K = 1;
    for (int t = 0; t < fm.n; ++t) m *= d[fm.x[t]];
    for (int t = 0; t < km.n; ++t) K *= d[km.x[t]];
    const int L = ld[b], K4 = (K + 3) & ~3;
    const bool tab = m <= kMatTab && K <= kMatTab;
    auto offset = [&](const ModeMap& mm, int idx) {
      int off = 0;
      for (int t = 0; t < mm.n; ++t) {
        const int e = d[mm.x[t]];
        off += (idx % e) * st[mm.x[t]];
        idx /= e;
      }
      return off;
    };
    if (tab) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) fo[i] = offset(fm, i);
      for (int i = threadIdx.x; i < K; i += blockDim.x) ko[i] = offset(km, i);
    }
    __syncthreads();
    const double* s = src + src_off[b];
    double* o = dst + dst_off[b];
    for (int k = warp; k < K4; k += nwarps) {
      const int okk = (k < K) ? (tab ? ko[k] : offset(km, k)) : 0;
      for (int r = lane; r < L; r += 32) {
        double v;
        if (k >= K) {
          v = kpad;
        } else if (r < m) {
          v = s[(tab ? fo[r] : offset(fm, r)) + okk];
          if (scale_on) v = mul_rn(scale, v);
        } else {
          v = 0.0;
        }
        o[(long long)k * L + r] = v;
      }
    }
    __syncthreads();
  }
}

// Plan-time layout: per block leading dimension (free extent rounded up to even) and offset.
static void layout(const sht_tensor* T, const std::vector<int>& free_modes, const std::vector<int>& k_modes,
                   std::vector<long long>& off, std::vector<int>& ld, std::vector<int>& k4, long long& total) {
  const long long n = T->nblocks;
  off.resize(n);
  ld.resize(n);
  k4.resize(n);
  total = 0;
  for (long long b = 0; b < n; ++b) {
    const int64_t id = T->ids[b];
    long long m = 1, K = 1;
    for (int ax : free_modes) m *= T->bs[ax][(id / T->gstride[ax]) % T->nblk[ax]];
    for (int ax : k_modes) K *= T->bs[ax][(id / T->gstride[ax]) % T->nblk[ax]];
    const long long L = (m + 1) & ~1LL, K4 = (K + 3) & ~3LL;
    if (L * K4 >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "matrix form of a block above 2^31 elements");
    off[b] = total;
    ld[b] = (int)L;
    k4[b] = (int)K4;
    total += L * K4;
  }
}

void matform_prepare(sht_plan* p, cudaStream_t s) {
  DevicePool* pool = p->ctx->pool.get();
  std::vector<long long> oa, ob;
  std::vector<int> la, lb, ka, kb;
  long long ta = 0, tb = 0;
  layout(p->A, p->maps.rowA, p->maps.colA, oa, la, ka, ta);
  layout(p->B, p->maps.colB, p->maps.rowB, ob, lb, kb, tb);
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  p->mf_a = PoolBuf(pool, std::max(ta, 2LL) * 8, s);
  p->mf_b = PoolBuf(pool, std::max(tb, 2LL) * 8, s);
  p->mf_aoff = PoolBuf(pool, std::max(nA, 1LL) * 8, s);
  p->mf_boff = PoolBuf(pool, std::max(nB, 1LL) * 8, s);
  p->mf_ald = PoolBuf(pool, std::max(nA, 1LL) * 4, s);
  p->mf_bld = PoolBuf(pool, std::max(nB, 1LL) * 4, s);
  p->mf_ak4 = PoolBuf(pool, std::max(nA, 1LL) * 4, s);
  if (nA) {
    SHT_CUDA(cudaMemcpyAsync(p->mf_aoff.ptr, oa.data(), nA * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_ald.ptr, la.data(), nA * 4, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_ak4.ptr, ka.data(), nA * 4, cudaMemcpyHostToDevice, s));
  }
  if (nB) {
    SHT_CUDA(cudaMemcpyAsync(p->mf_boff.ptr, ob.data(), nB * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_bld.ptr, lb.data(), nB * 4, cudaMemcpyHostToDevice, s));
  }
  SHT_CUDA(cudaStreamSynchronize(s));  // host vectors are pageable
  p->mf_elems = ta + tb;
}

static ModeMap modes_of(const std::vector<int>& v) {
  ModeMap m{};
  m.n = (int)v.size();
  for (size_t i = 0; i < v.size(); ++i) m.x[i] = m.y[i] = v[i];
  return m;
}

void matform_execute(sht_plan* p, double alpha, cudaStream_t s) {
  const int grid_cap = p->ctx->num_sms * 8;
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  if (nA)
    k_matform<<<(int)std::min<long long>(nA, grid_cap), 256, 0, s>>>(
        p->A->d_data.as<double>(), p->A->d_offsets.as<long long>(), p->A->d_dims.as<int>(), p->A->order,
        modes_of(p->maps.rowA), modes_of(p->maps.colA), p->mf_aoff.as<long long>(), p->mf_ald.as<int>(),
        p->mf_a.as<double>(), alpha, alpha != 1.0, -0.0, nA);
  if (nB)
    k_matform<<<(int)std::min<long long>(nB, grid_cap), 256, 0, s>>>(
        p->B->d_data.as<double>(), p->B->d_offsets.as<long long>(), p->B->d_dims.as<int>(), p->B->order,
        modes_of(p->maps.colB), modes_of(p->maps.rowB), p->mf_boff.as<long long>(), p->mf_bld.as<int>(),
        p->mf_b.as<double>(), 1.0, 0, 0.0, nB);
  SHT_CUDA(cudaGetLastError());
}

}  // namespace sht
