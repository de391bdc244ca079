// contract.cu -- block-sparse contraction on one GPU: device plan + FP64 tile kernels.
//
// Plan (all on the device; the reference has no block-sparse contract, src/Tensor/Tensor.cpp
// is empty, so the rules below are this library's canonical ones, restated in the oracle):
//   1. keys: per A block the rolled block indices of its contracted modes, per B block the
//      same over B's contracted modes; the C id splits into an A part and a B part;
//   2. B is radix-sorted by key (stable, so equal keys keep id order); every A block finds
//      its equal-key range by binary search, counts surviving pairs (norm screening) and
//      emits (idC, a, b) in (a, b) order;
//   3. a stable radix sort by idC gives the canonical pair order (idC, idA, idB);
//   4. the distinct idC merged with C's stored ids is the result pattern; C is re-reserved
//      to it when it grows (old blocks copied, new blocks zero-filled);
//   5. per C block its pair range, and the work list of TM x TN tiles (tiles of C blocks
//      with pairs first, untouched C blocks after; the latter are skipped when beta == 1).
// Execute launches the output-stationary tile kernel (tile_core.cuh) over the work list.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "contract.h"
#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void trace(const char* what, cudaStream_t s) {
  // SHT_TRACE=1: synchronize at every point (device + host time per phase);
  // SHT_TRACE=2: host time only (what the host spends issuing each phase)
  static const int on = [] {
    const char* e = std::getenv("SHT_TRACE");
    return e && (e[0] == '1' || e[0] == '2') ? e[0] - '0' : 0;
  }();
  if (!on) return;
  static double last = 0;
  if (on == 1) cudaStreamSynchronize(s);
  const double t = now_ms();
  std::fprintf(stderr, "[sht] %-28s %8.3f ms\n", what, last > 0 ? t - last : 0.0);
  last = t;
}

// ---------------------------------------------------------------------------------------
// plan kernels
// ---------------------------------------------------------------------------------------
struct KeySpec {
  int nk;                   // contracted modes
  int kmode[kMaxOrder];     // mode index in this tensor
  long long kstride[kMaxOrder];
  int nf;                   // free modes
  int fmode[kMaxOrder];
  long long fstride[kMaxOrder];  // C block-grid stride of the matching C mode
};

__global__ void k_keys(TensorMeta m, KeySpec ks, const long long* __restrict__ ids, long long n,
                       unsigned long long* __restrict__ key, long long* __restrict__ part) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < n; b += (long long)gridDim.x * blockDim.x) {
    int c[kMaxOrder];
    unroll_block(m, ids[b], c);
    unsigned long long k = 0;
    long long p = 0;
    for (int t = 0; t < ks.nk; ++t) k += (unsigned long long)c[ks.kmode[t]] * (unsigned long long)ks.kstride[t];
    for (int t = 0; t < ks.nf; ++t) p += (long long)c[ks.fmode[t]] * ks.fstride[t];
    key[b] = k;
    part[b] = p;
  }
}

__global__ void k_iota(int* v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) v[i] = (int)i;
}

__device__ __forceinline__ long long lower_bound_u64(const unsigned long long* a, long long n, unsigned long long x) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ long long lower_bound_i64(const long long* a, long long n, long long x) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// per A block: equal-key range in sorted B keys and number of surviving pairs
__global__ void k_count(const unsigned long long* __restrict__ keyA, long long nA,
                        const unsigned long long* __restrict__ keyBs, const int* __restrict__ permB, long long nB,
                        const double* __restrict__ normA, const double* __restrict__ normB, double eps,
                        long long* __restrict__ lo_out, long long* __restrict__ cnt) {
  for (long long a = blockIdx.x * (long long)blockDim.x + threadIdx.x; a < nA; a += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = keyA[a];
    const long long lo = lower_bound_u64(keyBs, nB, k);
    long long hi = lo;
    while (hi < nB && keyBs[hi] == k) ++hi;
    long long c = hi - lo;
    if (normA) {
      c = 0;
      const double na = normA[a];
      for (long long j = lo; j < hi; ++j) c += (na * normB[permB[j]] >= eps) ? 1 : 0;
    }
    lo_out[a] = lo;
    cnt[a] = c;
  }
}

__global__ void k_emit(const unsigned long long* __restrict__ keyA, const long long* __restrict__ partA, long long nA,
                       const unsigned long long* __restrict__ keyBs, const int* __restrict__ permB,
                       const long long* __restrict__ partB, long long nB, const double* __restrict__ normA,
                       const double* __restrict__ normB, double eps, const long long* __restrict__ lo_in,
                       const long long* __restrict__ end, const long long* __restrict__ cnt, long long* __restrict__ pc,
                       int* __restrict__ pa, int* __restrict__ pb) {
  for (long long a = blockIdx.x * (long long)blockDim.x + threadIdx.x; a < nA; a += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = keyA[a];
    long long w = end[a] - cnt[a];  // inclusive prefix sum minus own count
    const long long pA = partA[a];
    const double na = normA ? normA[a] : 0.0;
    for (long long j = lo_in[a]; j < nB && keyBs[j] == k; ++j) {
      const int b = permB[j];
      if (normA && !(na * normB[b] >= eps)) continue;
      pc[w] = pA + partB[b];
      pa[w] = (int)a;
      pb[w] = b;
      ++w;
    }
  }
}

__global__ void k_gather_pairs(const int* __restrict__ order, const int* __restrict__ pa_in, const int* __restrict__ pb_in,
                               long long n, int* __restrict__ pa, int* __restrict__ pb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int o = order[i];
    pa[i] = pa_in[o];
    pb[i] = pb_in[o];
  }
}

// pair range of each C block
__global__ void k_pstart(const long long* __restrict__ cids, long long nc, const long long* __restrict__ pcs,
                         long long np, int* __restrict__ pstart) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= nc; c += (long long)gridDim.x * blockDim.x)
    pstart[c] = (c == nc) ? (int)np : (int)lower_bound_i64(pcs, np, cids[c]);
}

// copy surviving old C blocks into the re-reserved layout
template <typename T>
__global__ void k_move_blocks(const T* __restrict__ src, const long long* __restrict__ old_ids,
                              const long long* __restrict__ old_off, const int* __restrict__ old_dims, int order,
                              long long n_old, const long long* __restrict__ new_ids, long long n_new,
                              const long long* __restrict__ new_off, T* __restrict__ dst) {
  for (long long b = blockIdx.x; b < n_old; b += gridDim.x) {
    long long s = 1;
    for (int d = 0; d < order; ++d) s *= old_dims[b * order + d];
    const long long pos = lower_bound_i64(new_ids, n_new, old_ids[b]);
    const T* p = src + old_off[b];
    T* q = dst + new_off[pos];
    for (long long e = threadIdx.x; e < s; e += blockDim.x) q[e] = p[e];
  }
}

// tiles per C block for a given tile shape; touched / untouched counted separately
__global__ void k_tile_counts(const int* __restrict__ dimsC, int oC, ModeMap row, ModeMap col, long long nc,
                              const int* __restrict__ pstart, int TM, int TN, long long* __restrict__ nt_touched,
                              long long* __restrict__ nt_untouched) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    long long m = 1, n = 1;
    for (int t = 0; t < row.n; ++t) m *= dimsC[c * oC + row.y[t]];
    for (int t = 0; t < col.n; ++t) n *= dimsC[c * oC + col.y[t]];
    const long long tiles = ((m + TM - 1) / TM) * ((n + TN - 1) / TN);
    const bool touched = pstart[c + 1] > pstart[c];
    nt_touched[c] = touched ? tiles : 0;
    nt_untouched[c] = touched ? 0 : tiles;
  }
}

__global__ void k_tile_emit(long long nc, const long long* __restrict__ cnt_t, const long long* __restrict__ off_t,
                            const long long* __restrict__ cnt_u, const long long* __restrict__ off_u,
                            long long base_u, int2* __restrict__ work) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const long long nt = cnt_t[c] + cnt_u[c];
    const long long w0 = cnt_t[c] ? off_t[c] : base_u + off_u[c];
    for (long long t = 0; t < nt; ++t) work[w0 + t] = make_int2((int)c, (int)t);
  }
}

// ---------------------------------------------------------------------------------------
// execute kernels
// ---------------------------------------------------------------------------------------
template <class Cfg>
__global__ void __launch_bounds__(Cfg::kThreads) k_contract_tiles(SparseArgs g) {
  __shared__ TileSmem<double, Cfg> sm;
  const int2 w = g.work[blockIdx.x];
  const int c = w.x;
  auto getc = [&](double*& p, const int*& d) {
    p = g.C + g.offC[c];
    d = g.dimsC + (long long)c * g.mp.oC;
  };
  auto getpair = [&](int p, const double*& a, const int*& ad, const double*& b, const int*& bd) {
    const int ia = g.pair_a[p], ib = g.pair_b[p];
    a = g.A + g.offA[ia];
    ad = g.dimsA + (long long)ia * g.mp.oA;
    b = g.B + g.offB[ib];
    bd = g.dimsB + (long long)ib * g.mp.oB;
  };
  tile_run<double, Cfg>(g.mp, g.sc, w.y, getc, getpair, g.pstart[c], g.pstart[c + 1], sm);
}

// tile shapes of the plain path (256 or 128 threads)
using Cfg64x64 = TileCfg<64, 64, 16, 4, 4>;
using Cfg128x32 = TileCfg<128, 32, 16, 8, 2>;
using Cfg32x128 = TileCfg<32, 128, 16, 2, 8>;
using Cfg128x16 = TileCfg<128, 16, 16, 4, 4>;
using Cfg16x128 = TileCfg<16, 128, 16, 4, 4>;
using Cfg32x32 = TileCfg<32, 32, 16, 2, 2>;

struct TileShape { int tm, tn; };
static const TileShape kShapes[] = {{64, 64}, {128, 32}, {32, 128}, {128, 16}, {16, 128}, {32, 32}};
constexpr int kNumShapes = 6;

static void launch_tiles(int cfg, long long nwork, const SparseArgs& g, cudaStream_t s) {
  if (nwork <= 0) return;
  const unsigned grid = (unsigned)nwork;
  switch (cfg) {
    case 0: k_contract_tiles<Cfg64x64><<<grid, Cfg64x64::kThreads, 0, s>>>(g); break;
    case 1: k_contract_tiles<Cfg128x32><<<grid, Cfg128x32::kThreads, 0, s>>>(g); break;
    case 2: k_contract_tiles<Cfg32x128><<<grid, Cfg32x128::kThreads, 0, s>>>(g); break;
    case 3: k_contract_tiles<Cfg128x16><<<grid, Cfg128x16::kThreads, 0, s>>>(g); break;
    case 4: k_contract_tiles<Cfg16x128><<<grid, Cfg16x128::kThreads, 0, s>>>(g); break;
    default: k_contract_tiles<Cfg32x32><<<grid, Cfg32x32::kThreads, 0, s>>>(g); break;
  }
  SHT_CUDA(cudaGetLastError());
}

// The FP64 tiles of a split plan's work list, computed only when the device word *flag is set
// (an operand of the execute holds a non-finite value): persistent, one 128 x 32 tile per
// iteration, the same tiles and element order as the plain form.
__global__ void __launch_bounds__(Cfg128x32::kThreads) k_contract_tiles_if(SparseArgs g, const int4* __restrict__ work,
                                                                            int nwork, const int* __restrict__ flag) {
  if (*flag == 0) return;
  __shared__ TileSmem<double, Cfg128x32> sm;
  for (int i = blockIdx.x; i < nwork; i += gridDim.x) {
    const int4 w = work[i];
    const int c = w.x;
    auto getc = [&](double*& p, const int*& d) {
      p = g.C + g.offC[c];
      d = g.dimsC + (long long)c * g.mp.oC;
    };
    auto getpair = [&](int p, const double*& a, const int*& ad, const double*& b, const int*& bd) {
      const int ia = g.pair_a[p], ib = g.pair_b[p];
      a = g.A + g.offA[ia];
      ad = g.dimsA + (long long)ia * g.mp.oA;
      b = g.B + g.offB[ib];
      bd = g.dimsB + (long long)ib * g.mp.oB;
    };
    tile_run<double, Cfg128x32>(g.mp, g.sc, w.y, getc, getpair, g.pstart[c], g.pstart[c + 1], sm);
    __syncthreads();  // the next tile reuses the shared tables
  }
}

void fallback_tiles_if(const SparseArgs& g, const int4* work, long long nwork, const int* flag, int grid,
                       cudaStream_t s) {
  if (nwork <= 0) return;
  k_contract_tiles_if<<<(unsigned)std::min<long long>(grid, nwork), Cfg128x32::kThreads, 0, s>>>(g, work, (int)nwork,
                                                                                               flag);
  SHT_CUDA(cudaGetLastError());
}

// Count the product block ids (sorted, with repeats) that are absent from the stored C ids
// (sorted, unique): zero means the result pattern is C's pattern.
__global__ void k_count_missing(const long long* __restrict__ pc, long long np, const long long* __restrict__ cids,
                                long long nc, unsigned long long* __restrict__ missing) {
  unsigned long long n = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x) {
    if (i > 0 && pc[i] == pc[i - 1]) continue;  // one search per distinct id
    const long long id = pc[i];
    long long lo = 0, hi = nc;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (cids[mid] < id) lo = mid + 1; else hi = mid;
    }
    if (lo == nc || cids[lo] != id) ++n;
  }
  if (n) atomicAdd(missing, n);
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static int bits_for(unsigned long long v) {
  int b = 1;
  while (b < 64 && (v >> b)) ++b;
  return b;
}

template <typename T>
static T d2h_scalar(const void* p, cudaStream_t s) {
  T v{};
  SHT_CUDA(cudaMemcpyAsync(&v, p, sizeof(T), cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  return v;
}

static bool bytes_zero(double v) {
  uint64_t u;
  std::memcpy(&u, &v, 8);
  return u == 0;
}

static void check_block_sizes(const sht_tensor* X, const std::vector<int>& mx, const sht_tensor* Y,
                              const std::vector<int>& my, const char* nx, const char* ny) {
  for (size_t t = 0; t < mx.size(); ++t)
    if (X->bs[mx[t]] != Y->bs[my[t]])
      fail(SHT_ERR_SIZE, std::string("Block sizes of mode ") + std::to_string(mx[t]) + " of " + nx + " and mode " +
                             std::to_string(my[t]) + " of " + ny + " do not match");
}

static ModeMap make_modemap(const std::vector<int>& x, const std::vector<int>& y) {
  ModeMap m{};
  m.n = (int)x.size();
  for (size_t i = 0; i < x.size(); ++i) { m.x[i] = x[i]; m.y[i] = y[i]; }
  return m;
}

// median-ish tile choice for the plain path: the shape that wastes the least tile area
// over the C blocks' (m, n), sampled from the host index
static int choose_plain_shape(const sht_plan* p) {
  const sht_tensor* C = p->C;
  if (C->nblocks == 0) return 0;
  const int stride = std::max<int64_t>(1, C->nblocks / 512);
  double best = 1e300;
  int best_i = 0;
  for (int si = 0; si < kNumShapes; ++si) {
    double waste = 0;
    for (int64_t b = 0; b < C->nblocks; b += stride) {
      const int64_t id = C->ids[b];
      int64_t m = 1, n = 1;
      for (int ax : p->maps.rowC) m *= C->bs[ax][(id / C->gstride[ax]) % C->nblk[ax]];
      for (int ax : p->maps.colC) n *= C->bs[ax][(id / C->gstride[ax]) % C->nblk[ax]];
      const int64_t tm = kShapes[si].tm, tn = kShapes[si].tn;
      const double area = (double)((m + tm - 1) / tm * tm) * (double)((n + tn - 1) / tn * tn);
      // padded area plus a per-tile fixed cost of 2k elements
      waste += area + 2048.0 * (double)(((m + tm - 1) / tm) * ((n + tn - 1) / tn));
    }
    if (waste < best) { best = waste; best_i = si; }
  }
  return best_i;
}

// per C block: matrix extents m, n, the sum over its pairs of the contracted extent, flops
__global__ void k_cstats(const int* __restrict__ dimsC, int oC, ModeMap row, ModeMap col,
                         const int* __restrict__ pstart, const int* __restrict__ pair_a,
                         const int* __restrict__ dimsA, int oA, ModeMap kk, long long nc, int* __restrict__ m_out,
                         int* __restrict__ n_out, long long* __restrict__ ksum_out, double* __restrict__ flops_out) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    long long m = 1, n = 1, ks = 0;
    for (int t = 0; t < row.n; ++t) m *= dimsC[c * oC + row.y[t]];
    for (int t = 0; t < col.n; ++t) n *= dimsC[c * oC + col.y[t]];
    for (int p = pstart[c]; p < pstart[c + 1]; ++p) {
      const int* ad = dimsA + (long long)pair_a[p] * oA;
      long long k = 1;
      for (int t = 0; t < kk.n; ++t) k *= ad[kk.x[t]];
      ks += k;
    }
    m_out[c] = (int)m;
    n_out[c] = (int)n;
    ksum_out[c] = ks;
    flops_out[c] = 2.0 * (double)m * (double)n * (double)ks;
  }
}

void cblock_stats(sht_plan* p, cudaStream_t s) {
  DevicePool* pool = p->ctx->pool.get();
  const long long nc = p->ncblk;
  p->d_cm = PoolBuf(pool, std::max(nc, 1LL) * 4, s);
  p->d_cn = PoolBuf(pool, std::max(nc, 1LL) * 4, s);
  p->d_cksum = PoolBuf(pool, std::max(nc, 1LL) * 8, s);
  p->flops = 0.0;
  p->flops_pending = false;
  if (nc == 0) return;
  PoolBuf fl(pool, nc * 8, s);
  p->d_flops = PoolBuf(pool, 8, s);
  k_cstats<<<grid_for(nc, 256), 256, 0, s>>>(p->C->d_dims.as<int>(), p->C->order, p->tmaps.row, p->tmaps.col,
                                              p->d_pstart.as<int>(), p->d_pair_a.as<int>(), p->A->d_dims.as<int>(),
                                              p->A->order, p->tmaps.kk, nc, p->d_cm.as<int>(), p->d_cn.as<int>(),
                                              p->d_cksum.as<long long>(), fl.as<double>());
  SHT_CUDA(cudaGetLastError());
  size_t tb = 0;
  cub::DeviceReduce::Sum(nullptr, tb, fl.as<double>(), p->d_flops.as<double>(), (int)nc, s);
  PoolBuf tmp(pool, tb, s);
  cub::DeviceReduce::Sum(tmp.ptr, tb, fl.as<double>(), p->d_flops.as<double>(), (int)nc, s);
  p->flops_pending = true;  // read with the next synchronization (plan_flops)
  if (!p->flops_event) SHT_CUDA(cudaEventCreateWithFlags(&p->flops_event, cudaEventDisableTiming));
  SHT_CUDA(cudaEventRecord(p->flops_event, s));
}

double plan_flops(sht_plan* p, cudaStream_t s) {
  if (p->flops_pending) {
    // s need not be the stream that computed the count: order the read after it
    if (p->flops_event) SHT_CUDA(cudaStreamWaitEvent(s, p->flops_event, 0));
    p->flops = d2h_scalar<double>(p->d_flops.ptr, s);
    p->flops_pending = false;
  }
  return p->flops;
}

sht_plan* plan_create(sht_ctx* ctx, const std::string& expr, sht_tensor* A, sht_tensor* B, sht_tensor* C,
                      double eps, sht_norm norm, sht_mode mode, cudaStream_t s) {
  std::unique_ptr<sht_plan> p(plan_init(ctx, expr, A, B, C, eps, norm, mode, s));
  plan_build(p.get(), s);
  return p.release();
}

sht_plan* plan_init(sht_ctx* ctx, const std::string& expr, sht_tensor* A, sht_tensor* B, sht_tensor* C,
                    double eps, sht_norm norm, sht_mode mode, cudaStream_t s) {
  const double t0 = now_ms();
  trace("plan: start", s);
  if (!A || !B || !C) fail(SHT_ERR_INVALID, "null tensor");
  if (A->ctx != ctx || B->ctx != ctx || C->ctx != ctx) fail(SHT_ERR_INVALID, "tensors from another context");
  if (A->dtype != SHT_F64 || B->dtype != SHT_F64 || C->dtype != SHT_F64)
    fail(SHT_ERR_UNSUPPORTED, "block-sparse contraction runs on FP64 tensors");
  if (A == C || B == C) fail(SHT_ERR_INVALID, "C must not alias A or B");
  for (sht_tensor* t : {A, B, C}) {
    tensor_touch(t, s);
    tensor_sync_host(t, s);
    if (t->has_marked) fail(SHT_ERR_STATE, "tensor has filtered blocks that were not compressed");
  }
  auto p = std::make_unique<sht_plan>();
  p->keep = ctx->pool;
  p->ctx = ctx;
  p->mode = mode;
  p->A = A; p->B = B; p->C = C;
  parse_einsum(expr, A->order, nullptr, B->order, nullptr, C->order, nullptr, p->maps);
  const ShtMaps& mp = p->maps;
  check_block_sizes(A, mp.rowA, C, mp.rowC, "tensor A", "tensor C");
  check_block_sizes(B, mp.colB, C, mp.colC, "tensor B", "tensor C");
  check_block_sizes(A, mp.colA, B, mp.rowB, "tensor A", "tensor B");
  p->eps = eps;
  p->norm = norm;
  p->plan_ms = now_ms() - t0;
  return p.release();
}

void plan_build(sht_plan* p, cudaStream_t s, bool speculate) {
  const double t0 = now_ms();
  sht_ctx* ctx = p->ctx;
  sht_tensor *A = p->A, *B = p->B, *C = p->C;
  // buffers the build reads or replaces are released against this stream
  for (sht_tensor* t : {A, B, C}) tensor_touch(t, s);
  const double eps = p->eps;
  const sht_norm norm = p->norm;
  const sht_mode mode = p->mode;
  const ShtMaps& mp = p->maps;
  DevicePool* pool = ctx->pool.get();
  const long long nA = A->nblocks, nB = B->nblocks;

  // contracted key radices
  KeySpec ka{}, kb{};
  unsigned long long kspan = 1;
  ka.nk = kb.nk = (int)mp.colA.size();
  for (size_t t = 0; t < mp.colA.size(); ++t) {
    ka.kmode[t] = mp.colA[t];
    kb.kmode[t] = mp.rowB[t];
    ka.kstride[t] = kb.kstride[t] = (long long)kspan;
    const unsigned long long nb = (unsigned long long)A->nblk[mp.colA[t]];
    if (kspan > (1ULL << 62) / nb) fail(SHT_ERR_UNSUPPORTED, "contracted block grid too large");
    kspan *= nb;
  }
  ka.nf = (int)mp.rowA.size();
  for (size_t t = 0; t < mp.rowA.size(); ++t) { ka.fmode[t] = mp.rowA[t]; ka.fstride[t] = C->gstride[mp.rowC[t]]; }
  kb.nf = (int)mp.colB.size();
  for (size_t t = 0; t < mp.colB.size(); ++t) { kb.fmode[t] = mp.colB[t]; kb.fstride[t] = C->gstride[mp.colC[t]]; }
  long double cgrid = 1;
  for (int d = 0; d < C->order; ++d) cgrid *= C->nblk[d];
  if (cgrid > 9.0e18L) fail(SHT_ERR_UNSUPPORTED, "C block grid too large");

  // Without screening the pair count follows from the host patterns (per contracted key the
  // number of B blocks, summed over A's blocks), so the device count need not be read back.
  long long np_host = -1;
  if (!(eps > 0.0) && kspan <= (1ULL << 16) && nA > 0 && nB > 0) {
    const int* xa = tensor_host_coords(A);
    const int* xb = tensor_host_coords(B);
    std::vector<long long> nbk(kspan, 0);
    for (long long b = 0; b < nB; ++b) {
      long long k = 0;
      for (int t = 0; t < kb.nk; ++t) k += xb[b * B->order + kb.kmode[t]] * kb.kstride[t];
      nbk[k]++;
    }
    np_host = 0;
    for (long long a = 0; a < nA; ++a) {
      long long k = 0;
      for (int t = 0; t < ka.nk; ++t) k += xa[a * A->order + ka.kmode[t]] * ka.kstride[t];
      np_host += nbk[k];
    }
  }
  long long np = 0;
  PoolBuf pc_sorted;
  if (nA > 0 && nB > 0) {
    PoolBuf keyA(pool, nA * 8, s), partA(pool, nA * 8, s), keyB(pool, nB * 8, s), partB(pool, nB * 8, s);
    k_keys<<<grid_for(nA, 256), 256, 0, s>>>(make_meta(A), ka, A->d_ids.as<long long>(), nA,
                                              keyA.as<unsigned long long>(), partA.as<long long>());
    k_keys<<<grid_for(nB, 256), 256, 0, s>>>(make_meta(B), kb, B->d_ids.as<long long>(), nB,
                                              keyB.as<unsigned long long>(), partB.as<long long>());
    SHT_CUDA(cudaGetLastError());
    PoolBuf keyBs, iota(pool, nB * 4, s), permB;
    k_iota<<<grid_for(nB, 256), 256, 0, s>>>(iota.as<int>(), nB);
    // B's blocks are stored by id (column-major over the block grid): when the contracted
    // modes are B's last modes, in order, the keys already ascend in storage order
    bool b_sorted = true;
    for (size_t t = 0; t < mp.rowB.size(); ++t)
      b_sorted = b_sorted && mp.rowB[t] == B->order - (int)mp.rowB.size() + (int)t;
    const int kbits = bits_for(kspan);
    size_t tb = 0;
    if (b_sorted) {
      keyBs = std::move(keyB);
      permB = std::move(iota);
    } else {
      keyBs = PoolBuf(pool, nB * 8, s);
      permB = PoolBuf(pool, nB * 4, s);
      cub::DeviceRadixSort::SortPairs(nullptr, tb, keyB.as<unsigned long long>(), keyBs.as<unsigned long long>(),
                                      iota.as<int>(), permB.as<int>(), (int)nB, 0, kbits, s);
      PoolBuf tmp(pool, tb, s);
      cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, keyB.as<unsigned long long>(), keyBs.as<unsigned long long>(),
                                      iota.as<int>(), permB.as<int>(), (int)nB, 0, kbits, s);
    }
    PoolBuf normA, normB;
    if (eps > 0.0) {
      normA = PoolBuf(pool, nA * 8, s);
      normB = PoolBuf(pool, nB * 8, s);
      tensor_norms_device(A, norm, normA.as<double>(), s);
      tensor_norms_device(B, norm, normB.as<double>(), s);
    }
    PoolBuf lo(pool, nA * 8, s), cnt(pool, nA * 8, s), off(pool, nA * 8, s);
    k_count<<<grid_for(nA, 128), 128, 0, s>>>(keyA.as<unsigned long long>(), nA, keyBs.as<unsigned long long>(),
                                              permB.as<int>(), nB, normA.as<double>(), normB.as<double>(), eps,
                                              lo.as<long long>(), cnt.as<long long>());
    SHT_CUDA(cudaGetLastError());
    cub::DeviceScan::InclusiveSum(nullptr, tb, cnt.as<long long>(), off.as<long long>(), (int)nA, s);
    {
      PoolBuf tmp(pool, tb, s);
      cub::DeviceScan::InclusiveSum(tmp.ptr, tb, cnt.as<long long>(), off.as<long long>(), (int)nA, s);
    }
    if (np_host >= 0) {
      // checked against the device's count at the next read-back (work list)
      np = np_host;
      p->d_npairs = PoolBuf(pool, 8, s);
      SHT_CUDA(cudaMemcpyAsync(p->d_npairs.ptr, off.as<long long>() + nA - 1, 8, cudaMemcpyDeviceToDevice, s));
    } else {
      np = d2h_scalar<long long>(off.as<long long>() + nA - 1, s);
    }
    if (np > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "more than 2^31 block pairs");
    if (np > 0) {
      PoolBuf pc(pool, np * 8, s), pa(pool, np * 4, s), pb(pool, np * 4, s);
      k_emit<<<grid_for(nA, 128), 128, 0, s>>>(keyA.as<unsigned long long>(), partA.as<long long>(), nA,
                                               keyBs.as<unsigned long long>(), permB.as<int>(), partB.as<long long>(),
                                               nB, normA.as<double>(), normB.as<double>(), eps, lo.as<long long>(),
                                               off.as<long long>(), cnt.as<long long>(), pc.as<long long>(),
                                               pa.as<int>(), pb.as<int>());
      SHT_CUDA(cudaGetLastError());
      PoolBuf pidx(pool, np * 4, s), porder(pool, np * 4, s);
      pc_sorted = PoolBuf(pool, np * 8, s);
      k_iota<<<grid_for(np, 256), 256, 0, s>>>(pidx.as<int>(), np);
      const int cbits = bits_for((unsigned long long)(cgrid > 1 ? (long long)cgrid - 1 : 1));
      cub::DeviceRadixSort::SortPairs(nullptr, tb, pc.as<long long>(), pc_sorted.as<long long>(), pidx.as<int>(),
                                      porder.as<int>(), (int)np, 0, cbits, s);
      {
        PoolBuf tmp(pool, tb, s);
        cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, pc.as<long long>(), pc_sorted.as<long long>(), pidx.as<int>(),
                                        porder.as<int>(), (int)np, 0, cbits, s);
      }
      p->d_pair_a = PoolBuf(pool, np * 4, s);
      p->d_pair_b = PoolBuf(pool, np * 4, s);
      k_gather_pairs<<<grid_for(np, 256), 256, 0, s>>>(porder.as<int>(), pa.as<int>(), pb.as<int>(), np,
                                                        p->d_pair_a.as<int>(), p->d_pair_b.as<int>());
      SHT_CUDA(cudaGetLastError());
    }
  }
  p->npairs = np;
  trace("plan: match+sort pairs", s);

  // result pattern: unique idC ∪ stored C ids
  long long nu = 0;
  PoolBuf uids;
  bool grow = np > 0;
  if (np > 0 && C->nblocks > 0) {
    // the repeated case: every product block is stored already (one count, no sorts)
    PoolBuf miss(pool, 8, s);
    SHT_CUDA(cudaMemsetAsync(miss.ptr, 0, 8, s));
    k_count_missing<<<grid_for(np, 256), 256, 0, s>>>(pc_sorted.as<long long>(), np, C->d_ids.as<long long>(),
                                                       C->nblocks, miss.as<unsigned long long>());
    SHT_CUDA(cudaGetLastError());
    if (speculate) {
      p->d_missing = std::move(miss);
      grow = false;
    } else {
      grow = d2h_scalar<unsigned long long>(miss.ptr, s) > 0;
    }
  }
  if (grow) {
    uids = PoolBuf(pool, np * 8, s);
    PoolBuf counts(pool, np * 4, s), nruns(pool, 8, s);
    size_t tb = 0;
    cub::DeviceRunLengthEncode::Encode(nullptr, tb, pc_sorted.as<long long>(), uids.as<long long>(),
                                       counts.as<int>(), nruns.as<long long>(), (int)np, s);
    PoolBuf tmp(pool, tb, s);
    cub::DeviceRunLengthEncode::Encode(tmp.ptr, tb, pc_sorted.as<long long>(), uids.as<long long>(),
                                       counts.as<int>(), nruns.as<long long>(), (int)np, s);
    nu = d2h_scalar<long long>(nruns.ptr, s);
  }
  const long long nC_old = C->nblocks;
  PoolBuf union_ids;
  long long nunion = nC_old;
  if (nu > 0) {
    if (nC_old == 0) {
      union_ids = std::move(uids);
      nunion = nu;
    } else {
      PoolBuf cat(pool, (nu + nC_old) * 8, s), cats(pool, (nu + nC_old) * 8, s), nsel(pool, 8, s);
      SHT_CUDA(cudaMemcpyAsync(cat.ptr, uids.ptr, nu * 8, cudaMemcpyDeviceToDevice, s));
      SHT_CUDA(cudaMemcpyAsync(cat.as<long long>() + nu, C->d_ids.ptr, nC_old * 8, cudaMemcpyDeviceToDevice, s));
      size_t tb = 0;
      cub::DeviceRadixSort::SortKeys(nullptr, tb, cat.as<long long>(), cats.as<long long>(), (int)(nu + nC_old), 0, 63, s);
      {
        PoolBuf tmp(pool, tb, s);
        cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, cat.as<long long>(), cats.as<long long>(), (int)(nu + nC_old), 0, 63, s);
      }
      union_ids = PoolBuf(pool, (nu + nC_old) * 8, s);
      cub::DeviceSelect::Unique(nullptr, tb, cats.as<long long>(), union_ids.as<long long>(), nsel.as<long long>(),
                                (int)(nu + nC_old), s);
      {
        PoolBuf tmp(pool, tb, s);
        cub::DeviceSelect::Unique(tmp.ptr, tb, cats.as<long long>(), union_ids.as<long long>(), nsel.as<long long>(),
                                  (int)(nu + nC_old), s);
      }
      nunion = d2h_scalar<long long>(nsel.ptr, s);
    }
  }
  if (nunion != nC_old) {
    // re-reserve C to the union pattern
    PoolBuf ndims(pool, std::max(nunion, 1LL) * C->order * 4, s), nsizes(pool, nunion * 8, s),
        noff(pool, nunion * 8, s);
    block_dims_sizes(C, union_ids.as<long long>(), nunion, ndims.as<int>(), nsizes.as<long long>(), s);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, nsizes.as<long long>(), noff.as<long long>(), (int)nunion, s);
    {
      PoolBuf tmp(pool, tb, s);
      cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, nsizes.as<long long>(), noff.as<long long>(), (int)nunion, s);
    }
    const long long nnz = d2h_scalar<long long>(noff.as<long long>() + nunion - 1, s) +
                          d2h_scalar<long long>(nsizes.as<long long>() + nunion - 1, s);
    PoolBuf ndata(pool, std::max(nnz, 1LL) * 8, s);
    SHT_CUDA(cudaMemsetAsync(ndata.ptr, 0, std::max(nnz, 1LL) * 8, s));
    if (nC_old > 0) {
      const int grid = (int)std::min<long long>(nC_old, (long long)ctx->num_sms * 8);
      k_move_blocks<double><<<grid, 256, 0, s>>>(C->d_data.as<double>(), C->d_ids.as<long long>(),
                                                 C->d_offsets.as<long long>(), C->d_dims.as<int>(), C->order, nC_old,
                                                 union_ids.as<long long>(), nunion, noff.as<long long>(),
                                                 ndata.as<double>());
      SHT_CUDA(cudaGetLastError());
    }
    C->d_ids = std::move(union_ids);
    C->d_offsets = std::move(noff);
    C->d_dims = std::move(ndims);
    C->d_data = std::move(ndata);
    C->nblocks = nunion;
    C->nnz = nnz;
    C->host_stale = true;
    tensor_sync_host(C, s);
  }
  const long long nc = C->nblocks;
  p->ncblk = nc;
  trace("plan: result pattern", s);

  // pair ranges and work list
  p->d_pstart = PoolBuf(pool, (nc + 1) * 4, s);
  k_pstart<<<grid_for(nc + 1, 256), 256, 0, s>>>(C->d_ids.as<long long>(), nc, pc_sorted.as<long long>(), np,
                                                  p->d_pstart.as<int>());
  SHT_CUDA(cudaGetLastError());
  p->flops = 0;
  p->tmaps.row = make_modemap(mp.rowA, mp.rowC);
  p->tmaps.kk = make_modemap(mp.colA, mp.rowB);
  p->tmaps.col = make_modemap(mp.colB, mp.colC);
  p->tmaps.oA = A->order;
  p->tmaps.oB = B->order;
  p->tmaps.oC = C->order;
  // per C block m, n, sum of the pairs' k and flops; the total flop count
  cblock_stats(p, s);
  trace("plan: pstart+flops", s);
  if (mode == SHT_MODE_PLAIN_FP64) {
    p->shape = choose_plain_shape(p);
    build_work(p, kShapes[p->shape].tm, kShapes[p->shape].tn, s);
    trace("plan: plain work list", s);
  }
  p->plan_ms += now_ms() - t0;
}

void build_work(sht_plan* p, int TM, int TN, cudaStream_t s) {
  DevicePool* pool = p->ctx->pool.get();
  const long long nc = p->ncblk;
  p->nwork = p->nwork_touched = 0;
  if (nc == 0) return;
  PoolBuf ct(pool, nc * 8, s), cu(pool, nc * 8, s), ot(pool, nc * 8, s), ou(pool, nc * 8, s);
  k_tile_counts<<<grid_for(nc, 256), 256, 0, s>>>(p->C->d_dims.as<int>(), p->C->order, p->tmaps.row, p->tmaps.col, nc,
                                                   p->d_pstart.as<int>(), TM, TN, ct.as<long long>(), cu.as<long long>());
  SHT_CUDA(cudaGetLastError());
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, ct.as<long long>(), ot.as<long long>(), (int)nc, s);
  {
    PoolBuf tmp(pool, tb, s);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, ct.as<long long>(), ot.as<long long>(), (int)nc, s);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, cu.as<long long>(), ou.as<long long>(), (int)nc, s);
  }
  const long long nt = d2h_scalar<long long>(ot.as<long long>() + nc - 1, s) + d2h_scalar<long long>(ct.as<long long>() + nc - 1, s);
  const long long nu = d2h_scalar<long long>(ou.as<long long>() + nc - 1, s) + d2h_scalar<long long>(cu.as<long long>() + nc - 1, s);
  if (nt + nu > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "work list above 2^31 tiles");
  p->d_work = PoolBuf(pool, std::max(nt + nu, 1LL) * 8, s);
  k_tile_emit<<<grid_for(nc, 128), 128, 0, s>>>(nc, ct.as<long long>(), ot.as<long long>(), cu.as<long long>(),
                                                 ou.as<long long>(), nt, p->d_work.as<int2>());
  SHT_CUDA(cudaGetLastError());
  plan_flops(p, s);  // the stream is idle after the reads above
  if (p->d_npairs.ptr) {
    // the pair list was sized from the host patterns: the device must have found as many
    if (d2h_scalar<long long>(p->d_npairs.ptr, s) != p->npairs)
      fail(SHT_ERR_STATE, "pair count of the host patterns differs from the device's");
    p->d_npairs = PoolBuf();
  }
  p->nwork_touched = nt;
  p->nwork = nt + nu;
  p->work_tm = TM;
  p->work_tn = TN;
}

SparseArgs sparse_args(sht_plan* p, double alpha, double beta) {
  const sht_tensor *A = p->A, *B = p->B, *C = p->C;
  SparseArgs g{};
  g.mp = p->tmaps;
  g.sc.alpha = alpha;
  g.sc.beta = beta;
  g.sc.beta_zero = bytes_zero(beta);
  g.sc.alpha_zero = bytes_zero(alpha);
  g.A = A->d_data.as<double>(); g.offA = A->d_offsets.as<long long>(); g.dimsA = A->d_dims.as<int>();
  g.B = B->d_data.as<double>(); g.offB = B->d_offsets.as<long long>(); g.dimsB = B->d_dims.as<int>();
  g.C = C->d_data.as<double>(); g.offC = C->d_offsets.as<long long>(); g.dimsC = C->d_dims.as<int>();
  g.pair_a = p->d_pair_a.as<int>(); g.pair_b = p->d_pair_b.as<int>(); g.pstart = p->d_pstart.as<int>();
  g.work = p->d_work.as<int2>();
  return g;
}

void plan_touch(sht_plan* p, cudaStream_t s) {
  for (sht_tensor* t : {p->A, p->B, p->C}) tensor_touch(t, s);
  for (PoolBuf* b : {&p->d_pair_a, &p->d_pair_b, &p->d_pstart, &p->d_work, &p->d_bwork, &p->d_counter, &p->mf_a,
                     &p->mf_b, &p->mf_aoff, &p->mf_boff, &p->mf_ald, &p->mf_bld, &p->mf_ak4, &p->mf_aitems,
                     &p->mf_bitems})
    b->use_on(s);
  for (PoolBuf* b : {&p->sp_a, &p->sp_b, &p->sp_ae, &p->sp_be, &p->sp_bsc, &p->sp_meta, &p->sp_items, &p->sp_pairs,
                     &p->sp_rowtab, &p->sp_coltab})
    b->use_on(s);
}

void plan_execute(sht_plan* p, double alpha, double beta, cudaStream_t s) {
  plan_touch(p, s);
  const SparseArgs g = sparse_args(p, alpha, beta);
  uint64_t one;
  const double d1 = 1.0;
  std::memcpy(&one, &d1, 8);
  uint64_t bb;
  std::memcpy(&bb, &beta, 8);
  const long long nwork = (bb == one) ? p->nwork_touched : p->nwork;
  if (p->mode == SHT_MODE_BATCHED_FP64) {
    batched_execute(p, g, nwork, s);
  } else if (p->mode == SHT_MODE_SPLIT) {
    split_execute(p, g, s);
  } else {
    launch_tiles(p->shape, nwork, g, s);
  }
}

}  // namespace sht
