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
// item (a block, or a slab of a large block's contracted index): the free/contracted offsets
// are tabulated in shared memory, then warps walk k and lanes walk rows, so stores are
// contiguous.
#include <algorithm>

#include "contract.h"
#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

constexpr int kMatTab = 4096;  // table entries per dimension held in shared memory

// One CTA per item: an item is a slab [k0, k1) of one block's contracted index, so a block of
// millions of elements is spread over many CTAs while small blocks take one item each.
__global__ void __launch_bounds__(256) k_matform(const double* __restrict__ src, const long long* __restrict__ src_off,
                                                 const int* __restrict__ dims, int order, ModeMap fm, ModeMap km,
                                                 const long long* __restrict__ dst_off, const int* __restrict__ ld,
                                                 const int4* __restrict__ items, long long nitems,
                                                 double* __restrict__ dst, double scale, int scale_on, double kpad) {
  __shared__ int fo[kMatTab], ko[kMatTab];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (long long it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int4 item = items[it];
    const long long b = item.x;
    const int k0 = item.y, k1 = item.z;
    const int* d = dims + b * order;
    int st[kMaxOrder];
    block_strides(d, order, st);
    int m = 1, K = 1;
    for (int t = 0; t < fm.n; ++t) m *= d[fm.x[t]];
    for (int t = 0; t < km.n; ++t) K *= d[km.x[t]];
    const int L = ld[b];
    const bool tab = m <= kMatTab && k1 - k0 <= kMatTab;
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
      for (int i = threadIdx.x; i < k1 - k0; i += blockDim.x) ko[i] = k0 + i < K ? offset(km, k0 + i) : 0;
    }
    __syncthreads();
    const double* s = src + src_off[b];
    double* o = dst + dst_off[b];
    for (int k = k0 + warp; k < k1; k += nwarps) {
      const int okk = (k < K) ? (tab ? ko[k - k0] : offset(km, k)) : 0;
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
// Items: slabs of about kSlabElems matrix-form elements (whole blocks when smaller).
constexpr long long kSlabElems = 1 << 15;

static void layout(sht_tensor* T, const std::vector<int>& free_modes, const std::vector<int>& k_modes,
                   std::vector<long long>& off, std::vector<int>& ld, std::vector<int>& k4, long long& total,
                   std::vector<int4>& items) {
  const long long n = T->nblocks;
  const int* dims = tensor_host_dims(T);
  off.resize(n);
  ld.resize(n);
  k4.resize(n);
  total = 0;
  for (long long b = 0; b < n; ++b) {
    const int* d = dims + b * T->order;
    long long m = 1, K = 1;
    for (int ax : free_modes) m *= d[ax];
    for (int ax : k_modes) K *= d[ax];
    const long long L = (m + 1) & ~1LL, K4 = (K + 3) & ~3LL;
    if (L * K4 >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "matrix form of a block above 2^31 elements");
    off[b] = total;
    ld[b] = (int)L;
    k4[b] = (int)K4;
    total += L * K4;
    const long long slab = std::min(K4, std::max(4LL, (kSlabElems / L + 3) & ~3LL));
    for (long long k0 = 0; k0 < K4; k0 += slab)
      items.push_back(make_int4((int)b, (int)k0, (int)std::min(K4, k0 + slab), 0));
  }
}

void matform_prepare(sht_plan* p, cudaStream_t s) {
  DevicePool* pool = p->ctx->pool.get();
  std::vector<long long> oa, ob;
  std::vector<int> la, lb, ka, kb;
  std::vector<int4> ia, ib;
  long long ta = 0, tb = 0;
  layout(p->A, p->maps.rowA, p->maps.colA, oa, la, ka, ta, ia);
  layout(p->B, p->maps.colB, p->maps.rowB, ob, lb, kb, tb, ib);
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  p->mf_a = PoolBuf(pool, std::max(ta, 2LL) * 8, s);
  p->mf_b = PoolBuf(pool, std::max(tb, 2LL) * 8, s);
  p->mf_aoff = PoolBuf(pool, std::max(nA, 1LL) * 8, s);
  p->mf_boff = PoolBuf(pool, std::max(nB, 1LL) * 8, s);
  p->mf_ald = PoolBuf(pool, std::max(nA, 1LL) * 4, s);
  p->mf_bld = PoolBuf(pool, std::max(nB, 1LL) * 4, s);
  p->mf_ak4 = PoolBuf(pool, std::max(nA, 1LL) * 4, s);
  p->mf_aitems = PoolBuf(pool, std::max<size_t>(ia.size(), 1) * sizeof(int4), s);
  p->mf_bitems = PoolBuf(pool, std::max<size_t>(ib.size(), 1) * sizeof(int4), s);
  p->mf_naitems = (long long)ia.size();
  p->mf_nbitems = (long long)ib.size();
  if (!ia.empty())
    SHT_CUDA(cudaMemcpyAsync(p->mf_aitems.ptr, ia.data(), ia.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  if (!ib.empty())
    SHT_CUDA(cudaMemcpyAsync(p->mf_bitems.ptr, ib.data(), ib.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
  if (nA) {
    SHT_CUDA(cudaMemcpyAsync(p->mf_aoff.ptr, oa.data(), nA * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_ald.ptr, la.data(), nA * 4, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_ak4.ptr, ka.data(), nA * 4, cudaMemcpyHostToDevice, s));
  }
  if (nB) {
    SHT_CUDA(cudaMemcpyAsync(p->mf_boff.ptr, ob.data(), nB * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->mf_bld.ptr, lb.data(), nB * 4, cudaMemcpyHostToDevice, s));
  }
  // (copies from pageable memory have consumed their source when they return)
  p->mf_elems = ta + tb;
}

static ModeMap modes_of(const std::vector<int>& v) {
  ModeMap m{};
  m.n = (int)v.size();
  for (size_t i = 0; i < v.size(); ++i) m.x[i] = m.y[i] = v[i];
  return m;
}

void matform_execute(sht_plan* p, double alpha, cudaStream_t s) {
  const long long grid_cap = (long long)p->ctx->num_sms * 8;
  if (p->mf_naitems)
    k_matform<<<(int)std::min(p->mf_naitems, grid_cap), 256, 0, s>>>(
        p->A->d_data.as<double>(), p->A->d_offsets.as<long long>(), p->A->d_dims.as<int>(), p->A->order,
        modes_of(p->maps.rowA), modes_of(p->maps.colA), p->mf_aoff.as<long long>(), p->mf_ald.as<int>(),
        p->mf_aitems.as<int4>(), p->mf_naitems, p->mf_a.as<double>(), alpha, alpha != 1.0, -0.0);
  if (p->mf_nbitems)
    k_matform<<<(int)std::min(p->mf_nbitems, grid_cap), 256, 0, s>>>(
        p->B->d_data.as<double>(), p->B->d_offsets.as<long long>(), p->B->d_dims.as<int>(), p->B->order,
        modes_of(p->maps.colB), modes_of(p->maps.rowB), p->mf_boff.as<long long>(), p->mf_bld.as<int>(),
        p->mf_bitems.as<int4>(), p->mf_nbitems, p->mf_b.as<double>(), 1.0, 0, 0.0);
  SHT_CUDA(cudaGetLastError());
}

}  // namespace sht
