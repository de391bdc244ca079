// batched.cu -- the batched FP64 form: one persistent kernel over a size-class work list.
//
// Products run on the FP64 tensor cores (mma.sync m8n8k4, bit-identical to the fma chain).
// Every C block is put in a size class by its matrix extents (m, n); each class has a tile
// shape (picked by the autotuner, or by a padded-area model until tuned).  The plan builds a
// single work list of (C block, tile, shape) items ordered by estimated cost, heaviest first;
// a persistent grid of 128-thread CTAs (SMs x resident CTAs) pulls items from an atomic
// counter and runs the pipelined tile (tile_pipe.cuh) of the item's shape.  Execute is a
// counter reset plus one launch, and is what sht_plan_execute_graph captures.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <numeric>
#include <cstdio>
#include <sstream>

#include <cub/cub.cuh>

#include "contract.h"
#include "device_common.cuh"
#include "tile_pipe.cuh"

namespace sht {

// tile shapes (all 128 threads); few, so the persistent kernel's code stays in cache
using B0 = PipeCfg<64, 64, 2>;   // 2x2 warps of 32x32
using B1 = PipeCfg<128, 32, 4>;  // 4x1 warps of 32x32
using B2 = PipeCfg<32, 128, 1>;  // 1x4 warps of 32x32
using B3 = PipeCfg<128, 16, 4>;  // 4x1 warps of 32x16
constexpr int kNumB = 4;
static const int kBTM[kNumB] = {64, 128, 32, 128};
static const int kBTN[kNumB] = {64, 32, 128, 16};

constexpr size_t smax(size_t a, size_t b) { return a > b ? a : b; }
constexpr size_t kBatchedSmem =
    smax(smax(sizeof(PipeSmem<B0>), sizeof(PipeSmem<B1>)), smax(sizeof(PipeSmem<B2>), sizeof(PipeSmem<B3>)));

struct BatchedArgs {
  TileMaps mp;
  TileScalars<double> sc;
  const double* Am; const long long* aoff; const int* ald; const int* ak4;  // A in matrix form
  const double* Bm; const long long* boff; const int* bld;                  // B in matrix form
  double* C; const long long* offC; const int* dimsC;
  const int* pair_a; const int* pair_b; const int* pstart;
  const int4* work;
  int nwork;
  int* counter;
  // serving launch: the requests' descriptors; request r owns launch items
  // [multi[r].first, multi[r].first + multi[r].nwork)
  const BatchedArgs* multi;
  int nmulti;
  int first;
};

template <class Cfg>
__device__ __forceinline__ void run_item(const BatchedArgs& g, int4 w, unsigned char* smem) {
  PipeSmem<Cfg>& sm = *reinterpret_cast<PipeSmem<Cfg>*>(smem);
  const int c = w.x;
  auto getc = [&](double*& p, const int*& d) {
    p = g.C + g.offC[c];
    d = g.dimsC + (long long)c * g.mp.oC;
  };
  auto getpair = [&](int p, PairView& v) {
    const int ia = g.pair_a[p], ib = g.pair_b[p];
    v.a = g.Am + g.aoff[ia];
    v.lda = g.ald[ia];
    v.K4 = g.ak4[ia];
    v.b = g.Bm + g.boff[ib];
    v.ldb = g.bld[ib];
  };
  tile_run_pipe<Cfg>(g.mp, g.sc, w.y, getc, getpair, g.pstart[c], g.pstart[c + 1], sm);
}

// Persistent kernel: each CTA takes items off the shared counter until the list is drained.
// kMulti: the work of several executes in one launch (serving); a launch item is mapped to
// its request by a binary search over the requests' first items.
template <bool kMulti>
__global__ void __launch_bounds__(128, 4) k_batched(BatchedArgs g) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_item, s_req;
  for (;;) {
    if (threadIdx.x == 0) {
      const int item = atomicAdd(g.counter, 1);
      s_item = item;
      if (kMulti && item < g.nwork) {
        int lo = 0, hi = g.nmulti - 1;  // last request whose first item <= item
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (g.multi[mid].first <= item) lo = mid; else hi = mid - 1;
        }
        s_req = lo;
      }
    }
    __syncthreads();
    const int item = s_item;
    const int req = kMulti ? s_req : 0;
    __syncthreads();
    if (item >= g.nwork) break;
    if constexpr (kMulti) {
      const BatchedArgs& r = g.multi[req];
      const int4 w = r.work[item - r.first];
      switch (w.z) {
        case 0: run_item<B0>(r, w, smem); break;
        case 1: run_item<B1>(r, w, smem); break;
        case 2: run_item<B2>(r, w, smem); break;
        default: run_item<B3>(r, w, smem); break;
      }
    } else {
      const int4 w = g.work[item];
      switch (w.z) {
        case 0: run_item<B0>(g, w, smem); break;
        case 1: run_item<B1>(g, w, smem); break;
        case 2: run_item<B2>(g, w, smem); break;
        default: run_item<B3>(g, w, smem); break;
      }
    }
  }
}

// resident CTAs for the persistent grid (the same for both instantiations: same smem, bounds)
static int batched_grid(sht_ctx* ctx) {
  static std::once_flag once;
  static int per_sm = 1;
  std::call_once(once, [] {
    SHT_CUDA(cudaFuncSetAttribute(k_batched<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchedSmem));
    SHT_CUDA(cudaFuncSetAttribute(k_batched<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBatchedSmem));
    int a = 0, b = 0;
    SHT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_batched<false>, 128, kBatchedSmem));
    SHT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batched<true>, 128, kBatchedSmem));
    per_sm = std::max(1, std::min(a, b));
  });
  return ctx->num_sms * per_sm;
}

// ------------------------------------------------------------------ size classes
static int ilog2ceil(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b;
}

struct ClassKey {
  int lm, ln, lk;
  std::string str() const { return std::to_string(lm) + "," + std::to_string(ln) + "," + std::to_string(lk); }
};

// padded-area cost model: MACs the tile shape runs (padding included) + a per-tile cost
static int model_shape(long long m, long long n) {
  double best = 1e300;
  int bi = 0;
  for (int s = 0; s < kNumB; ++s) {
    const long long tm = kBTM[s], tn = kBTN[s];
    const long long tiles = ((m + tm - 1) / tm) * ((n + tn - 1) / tn);
    const double cost = (double)tiles * (double)(tm * tn) + 3072.0 * (double)tiles;
    if (cost < best) { best = cost; bi = s; }
  }
  return bi;
}

struct HostPlanView {
  std::vector<long long> m, n, ksum;  // per C block
  std::vector<int> pstart;
  std::vector<ClassKey> key;
};

static HostPlanView host_view(sht_plan* p, cudaStream_t s) {
  HostPlanView v;
  sht_tensor *A = p->A, *B = p->B, *C = p->C;
  (void)B;
  tensor_sync_host(C, s);
  const long long nc = p->ncblk;
  v.pstart.resize(nc + 1);
  SHT_CUDA(cudaMemcpyAsync(v.pstart.data(), p->d_pstart.ptr, (nc + 1) * 4, cudaMemcpyDeviceToHost, s));
  std::vector<int> pa(p->npairs);
  if (p->npairs) SHT_CUDA(cudaMemcpyAsync(pa.data(), p->d_pair_a.ptr, p->npairs * 4, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  v.m.resize(nc);
  v.n.resize(nc);
  v.ksum.resize(nc);
  v.key.resize(nc);
  for (long long c = 0; c < nc; ++c) {
    const int64_t id = C->ids[c];
    long long m = 1, n = 1;
    for (int ax : p->maps.rowC) m *= C->bs[ax][(id / C->gstride[ax]) % C->nblk[ax]];
    for (int ax : p->maps.colC) n *= C->bs[ax][(id / C->gstride[ax]) % C->nblk[ax]];
    long long ks = 0;
    for (int q = v.pstart[c]; q < v.pstart[c + 1]; ++q) {
      const int64_t ida = A->ids[pa[q]];
      long long k = 1;
      for (int ax : p->maps.colA) k *= A->bs[ax][(ida / A->gstride[ax]) % A->nblk[ax]];
      ks += k;
    }
    v.m[c] = m;
    v.n[c] = n;
    v.ksum[c] = ks;
    const long long kavg = (v.pstart[c + 1] > v.pstart[c]) ? ks / (v.pstart[c + 1] - v.pstart[c]) : 1;
    v.key[c] = {ilog2ceil(m), ilog2ceil(n), ilog2ceil(std::max(1LL, kavg))};
  }
  return v;
}

// Work list: items (cblk, tile, shape), touched blocks sorted by cost (heaviest first), then
// untouched blocks (beta scaling only).
static void build_batched_work(sht_plan* p, const HostPlanView& v, const std::map<std::string, int>& shape_of,
                               cudaStream_t s, const std::vector<char>* subset = nullptr,
                               std::vector<int4>* out = nullptr) {
  const long long nc = p->ncblk;
  // order C blocks (not tiles) by cost, heaviest first; untouched blocks last
  struct Blk { double cost; int c, sh, tiles; bool has; };
  std::vector<Blk> blks;
  blks.reserve(nc);
  size_t ntouched = 0, nall = 0;
  for (long long c = 0; c < nc; ++c) {
    if (subset && !(*subset)[c]) continue;
    auto it = shape_of.find(v.key[c].str());
    const int sh = it != shape_of.end() ? it->second : model_shape(v.m[c], v.n[c]);
    const long long tm = kBTM[sh], tn = kBTN[sh];
    const int tiles = (int)(((v.m[c] + tm - 1) / tm) * ((v.n[c] + tn - 1) / tn));
    const bool has = v.pstart[c + 1] > v.pstart[c];
    blks.push_back({has ? (double)tm * tn * (double)v.ksum[c] : -1.0, (int)c, sh, tiles, has});
    nall += tiles;
    if (has) ntouched += tiles;
  }
  std::stable_sort(blks.begin(), blks.end(), [](const Blk& a, const Blk& b) { return a.cost > b.cost; });
  std::vector<int4> w;
  w.reserve(nall);
  for (const Blk& b : blks)
    for (int t = 0; t < b.tiles; ++t) w.push_back(make_int4(b.c, t, b.sh, 0));
  if (w.size() > (size_t)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "work list above 2^31 tiles");
  if (out) {
    *out = std::move(w);
    return;
  }
  p->bwork_touched = (long long)ntouched;
  p->bwork = (long long)w.size();
  p->d_bwork = PoolBuf(p->ctx->pool.get(), std::max<size_t>(w.size(), 1) * sizeof(int4), s);
  if (!w.empty()) {
    SHT_CUDA(cudaMemcpyAsync(p->d_bwork.ptr, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaStreamSynchronize(s));
  }
}

static void launch_batched(sht_plan* p, BatchedArgs& b, cudaStream_t s) {
  if (b.nwork <= 0) return;
  SHT_CUDA(cudaMemsetAsync(b.counter, 0, sizeof(int), s));
  const int grid = std::min<long long>(batched_grid(p->ctx), b.nwork);
  k_batched<false><<<grid, 128, kBatchedSmem, s>>>(b);
  SHT_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ device work list
struct ShapeSet {
  int n;
  int tm[kNumB], tn[kNumB];
};

__device__ __forceinline__ int ilog2ceil_dev(long long v) {
  int b = 0;
  while ((1LL << b) < v) ++b;
  return b;
}

__global__ void k_block_shapes(const int* __restrict__ cm, const int* __restrict__ cn,
                               const long long* __restrict__ cksum, const int* __restrict__ pstart, long long nc,
                               const unsigned char* __restrict__ table, int fixed_tm, int fixed_tn, ShapeSet ss,
                               int* __restrict__ shape, long long* __restrict__ tiles,
                               long long* __restrict__ touched_tiles, unsigned long long* __restrict__ key,
                               int* __restrict__ idx) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const long long m = cm[c], n = cn[c], ks = cksum[c];
    const int np = pstart[c + 1] - pstart[c];
    int sh = 0;
    long long tm = fixed_tm, tn = fixed_tn;
    if (fixed_tm <= 0) {
      int t = 255;
      if (table) {
        const int lm = min(ilog2ceil_dev(m), 31), ln = min(ilog2ceil_dev(n), 31);
        const int lk = min(ilog2ceil_dev(np > 0 ? (ks / np > 0 ? ks / np : 1) : 1), 31);
        t = table[(lm * 32 + ln) * 32 + lk];
      }
      if (t != 255) {
        sh = t;
      } else {  // padded-area model, as on the host
        double best = 1e300;
        for (int q = 0; q < ss.n; ++q) {
          const long long a = ss.tm[q], b = ss.tn[q];
          const long long nt = ((m + a - 1) / a) * ((n + b - 1) / b);
          const double cost = (double)nt * (double)(a * b) + 3072.0 * (double)nt;
          if (cost < best) { best = cost; sh = q; }
        }
      }
      tm = ss.tm[sh];
      tn = ss.tn[sh];
    }
    const long long nt = ((m + tm - 1) / tm) * ((n + tn - 1) / tn);
    shape[c] = sh;
    tiles[c] = nt;
    touched_tiles[c] = np > 0 ? nt : 0;
    // cost of one tile, coarsened to 16 bits (the float's exponent and 7 mantissa bits: the
    // order is for load balance only, and the stable sort keeps ties in block order)
    const float cost = np > 0 ? (float)((double)(tm * tn) * (double)ks + 1.0) : 0.0f;
    key[c] = (unsigned long long)(__float_as_uint(cost) >> 16);
    idx[c] = (int)c;
  }
}

__global__ void k_gather_tiles(const int* __restrict__ idx, const long long* __restrict__ tiles, long long nc,
                               long long* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x)
    out[i] = tiles[idx[i]];
}

__global__ void k_emit_items(const int* __restrict__ idx, const long long* __restrict__ tiles_sorted,
                             const long long* __restrict__ off, const int* __restrict__ shape, long long nc,
                             int4* __restrict__ work) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nc; i += (long long)gridDim.x * blockDim.x) {
    const int c = idx[i];
    const long long w0 = off[i];
    for (long long t = 0; t < tiles_sorted[i]; ++t) work[w0 + t] = make_int4(c, (int)t, shape[c], 0);
  }
}

// Up to eight device scalars (each a value or the sum of two) gathered into one buffer for a
// single read-back.
struct ScalarSrc {
  DevSum v[8];
  int n;
};
__global__ void k_collect(ScalarSrc src, long long* __restrict__ out) {
  const int i = threadIdx.x;
  if (i < src.n) out[i] = *src.v[i].a + (src.v[i].b ? *src.v[i].b : 0);
}

void device_work_list(sht_plan* p, int fixed_tm, int fixed_tn, bool per_class, cudaStream_t s, const DevSum* extra,
                      long long* extra_out, int nextra, const unsigned long long* order_key, int order_bits) {
  if (nextra > 3) fail(SHT_ERR_INVALID, "work list: at most three extra scalars");
  DevicePool* pool = p->ctx->pool.get();
  const long long nc = p->ncblk;
  p->bwork = p->bwork_touched = 0;
  if (nc == 0) {
    p->d_bwork = PoolBuf(pool, sizeof(int4), s);
    return;
  }
  ShapeSet ss{};
  ss.n = kNumB;
  for (int q = 0; q < kNumB; ++q) { ss.tm[q] = kBTM[q]; ss.tn[q] = kBTN[q]; }
  PoolBuf table;
  if (per_class && !p->ctx->tuned.empty()) {
    std::vector<unsigned char> h(32 * 32 * 32, 255);
    for (auto& kv : p->ctx->tuned) {
      int lm, ln, lk;
      if (std::sscanf(kv.first.c_str(), "%d,%d,%d", &lm, &ln, &lk) == 3 && lm < 32 && ln < 32 && lk < 32)
        h[(lm * 32 + ln) * 32 + lk] = (unsigned char)kv.second;
    }
    table = PoolBuf(pool, h.size(), s);
    SHT_CUDA(cudaMemcpyAsync(table.ptr, h.data(), h.size(), cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaStreamSynchronize(s));  // pageable source
  }
  PoolBuf shape(pool, nc * 4, s), tiles(pool, nc * 8, s), ttiles(pool, nc * 8, s), key(pool, nc * 8, s),
      idx(pool, nc * 4, s), key2(pool, nc * 8, s), idx2(pool, nc * 4, s), tsorted(pool, nc * 8, s),
      off(pool, nc * 8, s), sums(pool, 16, s);
  k_block_shapes<<<grid_for(nc, 256), 256, 0, s>>>(
      p->d_cm.as<int>(), p->d_cn.as<int>(), p->d_cksum.as<long long>(), p->d_pstart.as<int>(), nc,
      table.as<unsigned char>(), per_class ? 0 : fixed_tm, fixed_tn, ss, shape.as<int>(), tiles.as<long long>(),
      ttiles.as<long long>(), key.as<unsigned long long>(), idx.as<int>());
  SHT_CUDA(cudaGetLastError());
  // a caller's order (ascending keys, untouched blocks keyed last) replaces the cost order
  auto sort_blocks = [&](void* tmp_ptr, size_t& bytes) {
    if (order_key)
      cub::DeviceRadixSort::SortPairs(tmp_ptr, bytes, key.as<unsigned long long>(), key2.as<unsigned long long>(),
                                      idx.as<int>(), idx2.as<int>(), (int)nc, 0, order_bits, s);
    else
      cub::DeviceRadixSort::SortPairsDescending(tmp_ptr, bytes, key.as<unsigned long long>(),
                                                key2.as<unsigned long long>(), idx.as<int>(), idx2.as<int>(), (int)nc, 0,
                                                16, s);
  };
  if (order_key)
    SHT_CUDA(cudaMemcpyAsync(key.ptr, order_key, nc * 8, cudaMemcpyDeviceToDevice, s));
  size_t tb = 0, tb2 = 0, tb3 = 0;
  sort_blocks(nullptr, tb);
  cub::DeviceScan::ExclusiveSum(nullptr, tb2, tsorted.as<long long>(), off.as<long long>(), (int)nc, s);
  cub::DeviceReduce::Sum(nullptr, tb3, ttiles.as<long long>(), sums.as<long long>(), (int)nc, s);
  PoolBuf tmp(pool, std::max(tb, std::max(tb2, tb3)), s);
  sort_blocks(tmp.ptr, tb);
  k_gather_tiles<<<grid_for(nc, 256), 256, 0, s>>>(idx2.as<int>(), tiles.as<long long>(), nc, tsorted.as<long long>());
  cub::DeviceScan::ExclusiveSum(tmp.ptr, tb2, tsorted.as<long long>(), off.as<long long>(), (int)nc, s);
  cub::DeviceReduce::Sum(tmp.ptr, tb3, ttiles.as<long long>(), sums.as<long long>(), (int)nc, s);
  // one read-back: the list's length and touched count, the plan's flop count (while it is
  // still on the device) and the caller's extra scalars
  ScalarSrc src{};
  src.v[src.n++] = {off.as<long long>() + nc - 1, tsorted.as<long long>() + nc - 1};
  src.v[src.n++] = {sums.as<long long>(), nullptr};
  const bool fl = p->flops_pending;
  if (fl) src.v[src.n++] = {p->d_flops.as<long long>(), nullptr};  // the double's bits
  const bool npc = p->d_npairs.ptr != nullptr;
  const int inp = src.n;
  if (npc) src.v[src.n++] = {p->d_npairs.as<long long>(), nullptr};  // the device's pair count
  const bool msc = p->d_missing.ptr != nullptr;
  const int ims = src.n;
  if (msc) src.v[src.n++] = {p->d_missing.as<long long>(), nullptr};  // product blocks not in C
  for (int i = 0; i < nextra; ++i) src.v[src.n++] = extra[i];
  PoolBuf got(pool, 64, s);
  k_collect<<<1, 32, 0, s>>>(src, got.as<long long>());
  SHT_CUDA(cudaGetLastError());
  long long h[8];
  SHT_CUDA(cudaMemcpyAsync(h, got.ptr, src.n * 8, cudaMemcpyDeviceToHost, s));  // pageable: returns when done
  if (fl) {
    std::memcpy(&p->flops, &h[2], 8);
    p->flops_pending = false;
  }
  for (int i = 0; i < nextra; ++i) extra_out[i] = h[src.n - nextra + i];
  if (msc) {
    p->d_missing = PoolBuf();
    if (h[ims] != 0) throw PatternGrew{};  // the build assumed C's pattern: redo it
  }
  if (npc) {
    // the pair list was sized from the host patterns: the device must have found as many
    if (h[inp] != p->npairs) fail(SHT_ERR_STATE, "pair count of the host patterns differs from the device's");
    p->d_npairs = PoolBuf();
  }
  const long long total = h[0];
  if (total > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "work list above 2^31 tiles");
  p->bwork = total;
  p->bwork_touched = h[1];
  p->d_bwork = PoolBuf(pool, std::max(total, 1LL) * sizeof(int4), s);
  k_emit_items<<<grid_for(nc, 128), 128, 0, s>>>(idx2.as<int>(), tsorted.as<long long>(), off.as<long long>(),
                                                  shape.as<int>(), nc, p->d_bwork.as<int4>());
  SHT_CUDA(cudaGetLastError());
}

void batched_prepare(sht_plan* p, cudaStream_t s) {
  p->d_counter = PoolBuf(p->ctx->pool.get(), 256, s);
  matform_prepare(p, s);
  trace("batched: matform layout", s);
  device_work_list(p, 0, 0, true, s);
  trace("batched: work list", s);
}


static void fill_operands(sht_plan* p, BatchedArgs& b) {
  b.Am = p->mf_a.as<double>(); b.aoff = p->mf_aoff.as<long long>(); b.ald = p->mf_ald.as<int>();
  b.ak4 = p->mf_ak4.as<int>();
  b.Bm = p->mf_b.as<double>(); b.boff = p->mf_boff.as<long long>(); b.bld = p->mf_bld.as<int>();
}

// Descriptor of one batched plan's execute (also used by the serving loop).
static BatchedArgs batched_args(sht_plan* p, const SparseArgs& g) {
  BatchedArgs b{};
  b.mp = g.mp;
  b.sc = g.sc;
  fill_operands(p, b);
  b.C = g.C; b.offC = g.offC; b.dimsC = g.dimsC;
  b.pair_a = g.pair_a; b.pair_b = g.pair_b; b.pstart = g.pstart;
  b.work = p->d_bwork.as<int4>();
  uint64_t one, bb;
  const double d1 = 1.0;
  std::memcpy(&one, &d1, 8);
  std::memcpy(&bb, &g.sc.beta, 8);
  b.nwork = (int)((bb == one) ? p->bwork_touched : p->bwork);
  b.counter = p->d_counter.as<int>();
  return b;
}

size_t batched_desc_bytes() { return sizeof(BatchedArgs); }

// resident CTAs per SM of the persistent kernel
int batched_ctas_per_sm(sht_ctx* ctx) { return batched_grid(ctx) / ctx->num_sms; }

// One persistent launch over the work of several batched executes (the serving loop).  The
// operands must already be in matrix form (matform_execute).  host_descs: pinned host memory
// for plans.size() descriptors that the caller keeps unchanged until the launch completes (the
// upload reads it asynchronously); `descs` and `counter` are allocated on `s` and must be held
// as long.  ctas_per_sm (1..batched_ctas_per_sm) sets the persistent grid: fewer than the
// maximum leaves room on every SM for the planning kernels of requests that arrive meanwhile.
// Returns the number of launch items.
long long batched_multi_launch(sht_ctx* ctx, const std::vector<sht_plan*>& plans, const std::vector<SparseArgs>& args,
                               void* host_descs, PoolBuf& descs, PoolBuf& counter, int ctas_per_sm, cudaStream_t s) {
  DevicePool* pool = ctx->pool.get();
  BatchedArgs* h = static_cast<BatchedArgs*>(host_descs);
  long long total = 0;
  for (size_t i = 0; i < plans.size(); ++i) {
    h[i] = batched_args(plans[i], args[i]);
    h[i].first = (int)total;
    total += h[i].nwork;
    if (total > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "batched launch above 2^31 tiles");
  }
  if (total == 0) return 0;
  descs = PoolBuf(pool, plans.size() * sizeof(BatchedArgs), s);
  counter = PoolBuf(pool, 256, s);
  SHT_CUDA(cudaMemcpyAsync(descs.ptr, h, plans.size() * sizeof(BatchedArgs), cudaMemcpyHostToDevice, s));
  BatchedArgs b = h[0];
  b.nwork = (int)total;
  b.counter = counter.as<int>();
  b.multi = descs.as<BatchedArgs>();
  b.nmulti = (int)plans.size();
  SHT_CUDA(cudaMemsetAsync(b.counter, 0, sizeof(int), s));
  const int per_sm = std::max(1, std::min(ctas_per_sm, batched_ctas_per_sm(ctx)));
  const int grid = (int)std::min<long long>((long long)ctx->num_sms * per_sm, total);
  k_batched<true><<<grid, 128, kBatchedSmem, s>>>(b);
  SHT_CUDA(cudaGetLastError());
  return total;
}

void batched_launch(sht_plan* p, const SparseArgs& g, cudaStream_t s) {
  BatchedArgs b = batched_args(p, g);
  launch_batched(p, b, s);
}

void batched_execute(sht_plan* p, const SparseArgs& g, long long, cudaStream_t s) {
  BatchedArgs b = batched_args(p, g);
  if (!g.sc.alpha_zero) matform_execute(p, g.sc.alpha, s);
  trace("batched: matform kernels", s);
  launch_batched(p, b, s);
  trace("batched: tile kernel", s);
}

// ------------------------------------------------------------------ autotuner
// For every size class with work, time each tile shape on a sample of the class's C blocks
// (written to a scratch copy, never to C) and keep the fastest.  Choices persist in the
// context and, when a file is given, in a "key shape" text file keyed by GPU name.
void autotune(sht_plan* p, const char* cache_file, cudaStream_t s) {
  sht_ctx* ctx = p->ctx;
  cudaDeviceProp prop;
  SHT_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
  std::string gpu = prop.name;
  std::replace(gpu.begin(), gpu.end(), ' ', '_');
  if (cache_file) {
    std::ifstream in(cache_file);
    std::string g, k;
    int sh;
    while (in >> g >> k >> sh)
      if (g == gpu && sh >= 0 && sh < kNumB) ctx->tuned[k] = sh;
  }
  const HostPlanView v = host_view(p, s);
  matform_execute(p, 1.0, s);  // operands in matrix form for the timing runs
  std::map<std::string, std::vector<long long>> members;
  for (long long c = 0; c < p->ncblk; ++c)
    if (v.pstart[c + 1] > v.pstart[c]) members[v.key[c].str()].push_back(c);
  DevicePool* pool = ctx->pool.get();
  // scratch C: offsets remapped into a compact buffer for the sampled blocks
  std::vector<long long> offs(p->ncblk, 0);
  cudaEvent_t e0, e1;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  bool changed = false;
  for (auto& kv : members) {
    if (ctx->tuned.count(kv.first)) continue;
    std::vector<char> subset(p->ncblk, 0);
    long long elems = 0;
    size_t taken = 0;
    const size_t stride = std::max<size_t>(1, kv.second.size() / 256);
    for (size_t i = 0; i < kv.second.size() && taken < 256; i += stride, ++taken) {
      const long long c = kv.second[i];
      subset[c] = 1;
      offs[c] = elems;
      elems += v.m[c] * v.n[c];
    }
    PoolBuf scratch(pool, std::max(elems, 1LL) * 8, s), doffs(pool, p->ncblk * 8, s), work(pool, 1, s);
    SHT_CUDA(cudaMemcpyAsync(doffs.ptr, offs.data(), p->ncblk * 8, cudaMemcpyHostToDevice, s));
    double best = 1e300;
    int best_sh = model_shape(v.m[kv.second[0]], v.n[kv.second[0]]);
    for (int sh = 0; sh < kNumB; ++sh) {
      std::map<std::string, int> forced{{kv.first, sh}};
      std::vector<int4> items;
      build_batched_work(p, v, forced, s, &subset, &items);
      work = PoolBuf(pool, items.size() * sizeof(int4), s);
      SHT_CUDA(cudaMemcpyAsync(work.ptr, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
      BatchedArgs b{};
      b.mp = p->tmaps;
      b.sc = {1.0, 0.0, 1, 0};
      fill_operands(p, b);
      b.C = scratch.as<double>(); b.offC = doffs.as<long long>(); b.dimsC = p->C->d_dims.as<int>();
      b.pair_a = p->d_pair_a.as<int>(); b.pair_b = p->d_pair_b.as<int>(); b.pstart = p->d_pstart.as<int>();
      b.work = work.as<int4>();
      b.nwork = (int)items.size();
      b.counter = p->d_counter.as<int>();
      launch_batched(p, b, s);  // warm-up
      float ms = 0, tot = 0;
      for (int r = 0; r < 3; ++r) {
        SHT_CUDA(cudaEventRecord(e0, s));
        launch_batched(p, b, s);
        SHT_CUDA(cudaEventRecord(e1, s));
        SHT_CUDA(cudaEventSynchronize(e1));
        SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        tot += ms;
      }
      if (tot < best) { best = tot; best_sh = sh; }
    }
    ctx->tuned[kv.first] = best_sh;
    changed = true;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cache_file && changed) {
    std::ofstream out(cache_file, std::ios::app);
    for (auto& kv : ctx->tuned) out << gpu << " " << kv.first << " " << kv.second << "\n";
  }
  device_work_list(p, 0, 0, true, s);
}

}  // namespace sht
