// split.cu -- split-precision (Ozaki scheme) contraction on the INT8 tensor cores (tcgen05).
//
// Every A row (of every A block, after alpha) and every B column is scaled by a power of two
// 2^-e so its entries lie in (-1, 1), then cut into S slices of 7 bits:
//     x = sum_{t=1..S} 2^(-7t) s_t,   s_t = trunc(128 * remainder) in [-127, 127]
// (exact up to the truncated tail, < 2^(-7S) of the row / column maximum).  A block pair's
// product is then  C(r,c) = 2^(e_r + f_c) * sum_g 2^(-7g) * P_g(r,c),  P_g = sum_{t+u=g} A_t B_u
// over g = 2..S+1 (the triangle t+u <= S+1; dropped terms are below the truncation error).
// Each P_g is an exact INT32 sum, accumulated by tcgen05.mma kind::i8 into its own TMEM
// columns; the epilogue reads the groups back (tcgen05.ld), combines them in FP64 by Horner's
// rule from the smallest group up, scales by 2^(e_r+f_c) and adds into FP64 accumulators
// held in registers, one pair after another in the canonical pair order.  FP64 is used only
// for the reassembly, the accumulation into C and the scaling exponents.
//
// Tile: 128 rows (one TMEM lane per row, M = 128) x 32 columns of one C block; TMEM holds up
// to 8 groups x 32 columns.  One elected thread issues the MMAs and commits them to an
// mbarrier; every wait on it is bounded and reports SHT_ERR_TIMEOUT through an error word.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "contract.h"
#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

constexpr int kSplitM = 128, kSplitN = 32, kSplitK = 32, kMaxSlices = 8;
constexpr int kSplitTmemCols = 256;  // kMaxSlices groups x 32 columns

// ------------------------------------------------------------------ slicing
constexpr int kSliceTab = 4096;

// One CTA per block: row maxima -> exponents, then S int8 slices in K-major rows
// (out[t][r][k], row length Kp = K rounded up to 32, zero in the K padding).
__global__ void __launch_bounds__(256) k_slice(const double* __restrict__ src, const long long* __restrict__ src_off,
                                               const int* __restrict__ dims, int order, ModeMap fm, ModeMap km,
                                               const long long* __restrict__ out_off,
                                               const long long* __restrict__ exp_off, signed char* __restrict__ out,
                                               short* __restrict__ expo, double scale, int S, long long nblocks,
                                               int* __restrict__ bad) {
  __shared__ int fo[kSliceTab], ko[kSliceTab];
  for (long long b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int* d = dims + b * order;
    int st[kMaxOrder];
    block_strides(d, order, st);
    int m = 1, K = 1;
    for (int t = 0; t < fm.n; ++t) m *= d[fm.x[t]];
    for (int t = 0; t < km.n; ++t) K *= d[km.x[t]];
    const int Kp = (K + kSplitK - 1) / kSplitK * kSplitK;
    const bool tab = m <= kSliceTab && K <= kSliceTab;
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
    signed char* o = out + out_off[b];
    short* ex = expo + exp_off[b];
    const long long slab = (long long)m * Kp;
    // pass 1: row exponents (|v| / 2^e < 1), threads over rows
    for (int r = threadIdx.x; r < m; r += blockDim.x) {
      const int fr = tab ? fo[r] : offset(fm, r);
      double mx = 0.0;
      for (int k = 0; k < K; ++k) {
        const double v = __dmul_rn(s[fr + (tab ? ko[k] : offset(km, k))], scale);
        if (!isfinite(v)) atomicExch(bad, 1);
        mx = fmax(mx, fabs(v));
      }
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);
      ex[r] = (short)e;
    }
    __syncthreads();
    // pass 2: one thread per (row, 16-wide k chunk), rows fastest across threads
    const int kq = Kp / 16;
    for (int it = threadIdx.x; it < m * kq; it += blockDim.x) {
      const int r = it % m, q = it / m;
      const int fr = tab ? fo[r] : offset(fm, r);
      const int e = ex[r];
      signed char pk[kMaxSlices][16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int k = q * 16 + j;
        double x = (k < K) ? scalbn(__dmul_rn(s[fr + (tab ? ko[k] : offset(km, k))], scale), -e) : 0.0;
#pragma unroll
        for (int t = 0; t < kMaxSlices; ++t) {
          const double y = x * 128.0;
          const double tr = trunc(y);
          pk[t][j] = (signed char)(int)tr;
          x = y - tr;
        }
      }
      for (int t = 0; t < S; ++t)
        *reinterpret_cast<int4*>(o + t * slab + (long long)r * Kp + q * 16) = *reinterpret_cast<const int4*>(pk[t]);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ unsigned smem_u32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

// K-major, no swizzle: core matrices of 8 rows x 16 bytes; LBO = 128 (the two 16-byte halves
// of a 32-byte K step), SBO = 256 (next 8 rows).
__device__ __forceinline__ unsigned long long umma_desc(const void* smem) {
  const unsigned long long a = (smem_u32(smem) >> 4) & 0x3FFFu;
  return a | (8ull << 16) | (16ull << 32) | (1ull << 46);
}

// kind::i8, signed A and B, S32 accumulate, K-major operands, M = 128, N = 32
constexpr unsigned kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(kSplitN >> 3) << 17) |
                              ((unsigned)(kSplitM >> 4) << 24);

__device__ __forceinline__ void umma_i8(unsigned tmem_d, unsigned long long da, unsigned long long db, int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdescI8), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(void* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(void* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// bounded wait on an mbarrier phase; returns false on timeout
__device__ __forceinline__ bool mbar_wait(void* mbar, unsigned parity, long long limit) {
  const unsigned a = smem_u32(mbar);
  for (long long i = 0; i < limit; ++i) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void cp16(void* smem, const void* gmem, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(bytes)
               : "memory");
}

// int32 -> double with one integer add and one FP64 add: the bits of 1.5*2^52 plus the
// sign-extended x are the double 1.5*2^52 + x (unit spacing in that binade)
__device__ __forceinline__ double i2d(unsigned x) {
  return __longlong_as_double(0x4338000000000000LL + (long long)(int)x) - 6755399441055744.0;
}

// ------------------------------------------------------------------ main kernel
struct SplitArgs {
  TileMaps mp;
  double beta;
  int beta_zero, alpha_zero, S;
  const signed char* As; const long long* as_off; const long long* ae_off; const short* Ae;  // A slices
  const signed char* Bs; const long long* bs_off; const long long* be_off; const short* Be;  // B slices
  const int* dimsA; const int* dimsB;
  double* C; const long long* offC; const int* dimsC;
  const int* pair_a; const int* pair_b; const int* pstart;
  const int4* work;
  int nwork;
  int* counter;
  int* err;
  long long wait_limit;
};

struct SplitSmem {
  union {
    struct {
      alignas(128) signed char a[kMaxSlices][kSplitM * kSplitK];  // per slice one 128 x 32 K-major slab
      alignas(128) signed char b[kMaxSlices][kSplitN * kSplitK];
    } op;
    double c[kSplitN][kSplitM + 2];
  } u;
  int rowC[kSplitM], colC[kSplitN];
  short fexp[kSplitN];
  alignas(8) unsigned long long mbar;
  unsigned tmem_base;
  int item;
};

__global__ void __launch_bounds__(128, 1) k_split(SplitArgs g) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  SplitSmem& sm = *reinterpret_cast<SplitSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int S = g.S;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(kSplitTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&sm.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = sm.tmem_base;
  unsigned phase = 0;
  bool failed = false;

  for (;;) {
    if (tid == 0) sm.item = atomicAdd(g.counter, 1);
    __syncthreads();
    const int item = sm.item;
    __syncthreads();
    if (item >= g.nwork || failed) break;
    const int4 w = g.work[item];
    const int c = w.x;
    double* cptr = g.C + g.offC[c];
    const int* cd = g.dimsC + (long long)c * g.mp.oC;
    int stC[kMaxOrder];
    block_strides(cd, g.mp.oC, stC);
    int m = 1, n = 1;
    for (int t = 0; t < g.mp.row.n; ++t) m *= cd[g.mp.row.y[t]];
    for (int t = 0; t < g.mp.col.n; ++t) n *= cd[g.mp.col.y[t]];
    const int ntr = (m + kSplitM - 1) / kSplitM;
    const int r0 = (w.y % ntr) * kSplitM, c0 = (w.y / ntr) * kSplitN;
    const int mt = min(kSplitM, m - r0), nt = min(kSplitN, n - c0);
    for (int i = tid; i < kSplitM + kSplitN; i += 128) {
      if (i < kSplitM) {
        int r = r0 + i, off = 0;
        for (int t = 0; t < g.mp.row.n; ++t) {
          const int e = cd[g.mp.row.y[t]];
          off += (r % e) * stC[g.mp.row.y[t]];
          r /= e;
        }
        sm.rowC[i] = (i < mt) ? off : 0;
      } else {
        const int j = i - kSplitM;
        int cc = c0 + j, off = 0;
        for (int t = 0; t < g.mp.col.n; ++t) {
          const int e = cd[g.mp.col.y[t]];
          off += (cc % e) * stC[g.mp.col.y[t]];
          cc /= e;
        }
        sm.colC[j] = (j < nt) ? off : 0;
      }
    }
    __syncthreads();
    // this thread owns tile row `tid` (TMEM lane tid) and all 32 columns
    double acc[kSplitN];
    if (g.beta_zero) {
#pragma unroll
      for (int j = 0; j < kSplitN; ++j) acc[j] = 0.0;
    } else {
      for (int e = tid; e < kSplitM * kSplitN; e += 128) {
        const int i = e % kSplitM, j = e / kSplitM;
        sm.u.c[j][i] = (i < mt && j < nt) ? cptr[sm.rowC[i] + sm.colC[j]] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kSplitN; ++j) acc[j] = __dmul_rn(g.beta, sm.u.c[j][tid]);
      __syncthreads();
    }

    const int pb = g.pstart[c], pe = g.pstart[c + 1];
    for (int p = pb; p < pe && !g.alpha_zero; ++p) {
      const int ia = g.pair_a[p], ib = g.pair_b[p];
      const int* ad = g.dimsA + (long long)ia * g.mp.oA;
      const int* bdm = g.dimsB + (long long)ib * g.mp.oB;
      int ma = 1, nb = 1, K = 1;
      for (int t = 0; t < g.mp.row.n; ++t) ma *= ad[g.mp.row.x[t]];
      for (int t = 0; t < g.mp.col.n; ++t) nb *= bdm[g.mp.col.x[t]];
      for (int t = 0; t < g.mp.kk.n; ++t) K *= ad[g.mp.kk.x[t]];
      const int Kp = (K + kSplitK - 1) / kSplitK * kSplitK;
      const signed char* abase = g.As + g.as_off[ia];
      const signed char* bbase = g.Bs + g.bs_off[ib];
      const long long aslab = (long long)ma * Kp, bslab = (long long)nb * Kp;
      for (int j = tid; j < kSplitN; j += 128) sm.fexp[j] = (j < nt) ? g.Be[g.be_off[ib] + c0 + j] : 0;
      const int er = (tid < mt) ? g.Ae[g.ae_off[ia] + r0 + tid] : 0;
      for (int ks = 0; ks < Kp; ks += kSplitK) {
        // operand slabs: A rows r0.. (zero past m), B columns c0.. (zero past n)
        for (int e = tid; e < S * kSplitM * 2; e += 128) {
          const int t = e / (kSplitM * 2), rem = e % (kSplitM * 2), r = rem >> 1, h = rem & 1;
          const bool ok = r < mt;
          const signed char* src = abase + t * aslab + (long long)(ok ? r0 + r : 0) * Kp + ks + h * 16;
          cp16(&sm.u.op.a[t][(r >> 3) * 256 + h * 128 + (r & 7) * 16], src, ok ? 16 : 0);
        }
        for (int e = tid; e < S * kSplitN * 2; e += 128) {
          const int t = e / (kSplitN * 2), rem = e % (kSplitN * 2), r = rem >> 1, h = rem & 1;
          const bool ok = r < nt;
          const signed char* src = bbase + t * bslab + (long long)(ok ? c0 + r : 0) * Kp + ks + h * 16;
          cp16(&sm.u.op.b[t][(r >> 3) * 256 + h * 128 + (r & 7) * 16], src, ok ? 16 : 0);
        }
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
          for (int gi = 2; gi <= S + 1; ++gi) {
            const unsigned dcol = tmem + (unsigned)((gi - 2) * kSplitN);
            bool first = (ks == 0);
            for (int t = 1; t <= S; ++t) {
              const int u = gi - t;
              if (u < 1 || u > S) continue;
              umma_i8(dcol, umma_desc(sm.u.op.a[t - 1]), umma_desc(sm.u.op.b[u - 1]), first ? 0 : 1);
              first = false;
            }
          }
          umma_commit(&sm.mbar);
        }
        // every thread waits for the MMAs (operands are rewritten next step, TMEM read below)
        const bool ok = mbar_wait(&sm.mbar, phase, g.wait_limit);
        phase ^= 1;
        tc_fence_after();
        failed = __syncthreads_or(!ok);
        if (failed) {
          if (tid == 0) atomicExch(g.err, (int)SHT_ERR_TIMEOUT);
          // let the tensor core finish before TMEM is released (bounded as well)
          mbar_wait(&sm.mbar, phase ^ 1, g.wait_limit);
          break;
        }
      }
      if (failed) break;
      // epilogue for the pair: Horner over groups from the smallest weight up, then scale
#pragma unroll
      for (int h = 0; h < kSplitN / 16; ++h) {
        double part[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) part[j] = 0.0;
        for (int gi = S + 1; gi >= 2; --gi) {
          unsigned v[16];
          tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)((gi - 2) * kSplitN + h * 16), v);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) part[j] = fma(part[j], 0.0078125, i2d(v[j]));
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          acc[h * 16 + j] += scalbn(part[j], er + sm.fexp[h * 16 + j] - 14);
        }
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
    }
    if (failed) break;
    // stage and store the tile along C's memory order
#pragma unroll
    for (int j = 0; j < kSplitN; ++j) sm.u.c[j][tid] = acc[j];
    __syncthreads();
    for (int e = tid; e < kSplitM * kSplitN; e += 128) {
      const int i = e % kSplitM, j = e / kSplitM;
      if (i < mt && j < nt) cptr[sm.rowC[i] + sm.colC[j]] = sm.u.c[j][i];
    }
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kSplitTmemCols) : "memory");
}

// ------------------------------------------------------------------ host side
static ModeMap modes_of(const std::vector<int>& v) {
  ModeMap m{};
  m.n = (int)v.size();
  for (size_t i = 0; i < v.size(); ++i) m.x[i] = m.y[i] = v[i];
  return m;
}

static void slice_layout(const sht_tensor* T, const std::vector<int>& free_modes, const std::vector<int>& k_modes,
                         int S, std::vector<long long>& off, std::vector<long long>& eoff, long long& total,
                         long long& etotal) {
  const long long n = T->nblocks;
  off.resize(n);
  eoff.resize(n);
  total = etotal = 0;
  for (long long b = 0; b < n; ++b) {
    const int64_t id = T->ids[b];
    long long m = 1, K = 1;
    for (int ax : free_modes) m *= T->bs[ax][(id / T->gstride[ax]) % T->nblk[ax]];
    for (int ax : k_modes) K *= T->bs[ax][(id / T->gstride[ax]) % T->nblk[ax]];
    const long long Kp = (K + kSplitK - 1) / kSplitK * kSplitK;
    if ((long long)S * m * Kp >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "block slices above 2^31 bytes");
    off[b] = total;
    eoff[b] = etotal;
    total += (long long)S * m * Kp;  // multiple of 32: every block stays 16-byte aligned
    etotal += m;
  }
}

int split_slices_default() { return 7; }

void split_prepare(sht_plan* p, int S, cudaStream_t s) {
  if (S < 1 || S > kMaxSlices) fail(SHT_ERR_INVALID, "split slices must be 1..8");
  DevicePool* pool = p->ctx->pool.get();
  p->split_slices = S;
  std::vector<long long> ao, ae, bo, be;
  long long at, aet, bt, bet;
  slice_layout(p->A, p->maps.rowA, p->maps.colA, S, ao, ae, at, aet);
  slice_layout(p->B, p->maps.colB, p->maps.rowB, S, bo, be, bt, bet);
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  p->sp_a = PoolBuf(pool, std::max(at, 16LL), s);
  p->sp_b = PoolBuf(pool, std::max(bt, 16LL), s);
  p->sp_ae = PoolBuf(pool, std::max(aet, 1LL) * 2, s);
  p->sp_be = PoolBuf(pool, std::max(bet, 1LL) * 2, s);
  p->sp_aoff = PoolBuf(pool, std::max(nA, 1LL) * 8, s);
  p->sp_aeoff = PoolBuf(pool, std::max(nA, 1LL) * 8, s);
  p->sp_boff = PoolBuf(pool, std::max(nB, 1LL) * 8, s);
  p->sp_beoff = PoolBuf(pool, std::max(nB, 1LL) * 8, s);
  p->sp_err = PoolBuf(pool, 256, s);
  if (nA) {
    SHT_CUDA(cudaMemcpyAsync(p->sp_aoff.ptr, ao.data(), nA * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->sp_aeoff.ptr, ae.data(), nA * 8, cudaMemcpyHostToDevice, s));
  }
  if (nB) {
    SHT_CUDA(cudaMemcpyAsync(p->sp_boff.ptr, bo.data(), nB * 8, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaMemcpyAsync(p->sp_beoff.ptr, be.data(), nB * 8, cudaMemcpyHostToDevice, s));
  }
  SHT_CUDA(cudaMemsetAsync(p->sp_err.ptr, 0, 256, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  // work list: 128 x 32 tiles of every C block, heaviest blocks first
  device_work_list(p, kSplitM, kSplitN, false, s);
  p->d_counter = PoolBuf(pool, 256, s);
  SHT_CUDA(cudaStreamSynchronize(s));
}

// Each CTA holds kSplitTmemCols of the SM's 512 TMEM columns for its lifetime, so at most two
// may be resident on an SM: the launch reserves enough shared memory that a third cannot fit.
constexpr size_t kSplitSmemLaunch = std::max<size_t>(sizeof(SplitSmem), 100 * 1024);

static int split_grid(sht_ctx* ctx) {
  static int per_sm = -1;
  if (per_sm < 0) {
    SHT_CUDA(cudaFuncSetAttribute(k_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmemLaunch));
    SHT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_split, 128, kSplitSmemLaunch));
    if (per_sm > 512 / kSplitTmemCols) fail(SHT_ERR_STATE, "split kernel occupancy exceeds the TMEM budget");
    per_sm = std::max(per_sm, 1);
  }
  return ctx->num_sms * per_sm;
}

void split_execute(sht_plan* p, const SparseArgs& sa, cudaStream_t s) {
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  const int S = p->split_slices;
  const int cap = p->ctx->num_sms * 8;
  if (!sa.sc.alpha_zero) {
    if (nA)
      k_slice<<<(int)std::min<long long>(nA, cap), 256, 0, s>>>(
          p->A->d_data.as<double>(), p->A->d_offsets.as<long long>(), p->A->d_dims.as<int>(), p->A->order,
          modes_of(p->maps.rowA), modes_of(p->maps.colA), p->sp_aoff.as<long long>(), p->sp_aeoff.as<long long>(),
          p->sp_a.as<signed char>(), p->sp_ae.as<short>(), sa.sc.alpha, S, nA, p->sp_err.as<int>() + 1);
    if (nB)
      k_slice<<<(int)std::min<long long>(nB, cap), 256, 0, s>>>(
          p->B->d_data.as<double>(), p->B->d_offsets.as<long long>(), p->B->d_dims.as<int>(), p->B->order,
          modes_of(p->maps.colB), modes_of(p->maps.rowB), p->sp_boff.as<long long>(), p->sp_beoff.as<long long>(),
          p->sp_b.as<signed char>(), p->sp_be.as<short>(), 1.0, S, nB, p->sp_err.as<int>() + 1);
    SHT_CUDA(cudaGetLastError());
  }
  uint64_t one, bb;
  const double d1 = 1.0;
  std::memcpy(&one, &d1, 8);
  std::memcpy(&bb, &sa.sc.beta, 8);
  SplitArgs g{};
  g.mp = sa.mp;
  g.beta = sa.sc.beta;
  g.beta_zero = sa.sc.beta_zero;
  g.alpha_zero = sa.sc.alpha_zero;
  g.S = S;
  g.As = p->sp_a.as<signed char>(); g.as_off = p->sp_aoff.as<long long>(); g.ae_off = p->sp_aeoff.as<long long>();
  g.Ae = p->sp_ae.as<short>();
  g.Bs = p->sp_b.as<signed char>(); g.bs_off = p->sp_boff.as<long long>(); g.be_off = p->sp_beoff.as<long long>();
  g.Be = p->sp_be.as<short>();
  g.dimsA = p->A->d_dims.as<int>(); g.dimsB = p->B->d_dims.as<int>();
  g.C = sa.C; g.offC = sa.offC; g.dimsC = sa.dimsC;
  g.pair_a = sa.pair_a; g.pair_b = sa.pair_b; g.pstart = sa.pstart;
  g.work = p->d_bwork.as<int4>();
  g.nwork = (int)((bb == one) ? p->bwork_touched : p->bwork);
  g.counter = p->d_counter.as<int>();
  g.err = p->sp_err.as<int>();
  g.wait_limit = 1LL << 20;
  if (g.nwork <= 0) return;
  SHT_CUDA(cudaMemsetAsync(g.counter, 0, sizeof(int), s));
  const int grid = (int)std::min<long long>(split_grid(p->ctx), g.nwork);
  k_split<<<grid, 128, kSplitSmemLaunch, s>>>(g);
  SHT_CUDA(cudaGetLastError());
}

// error words of the last split execute: [0] status from bounded waits, [1] non-finite input
void split_check(sht_plan* p, cudaStream_t s) {
  int e[2] = {0, 0};
  SHT_CUDA(cudaMemcpyAsync(e, p->sp_err.ptr, 8, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  if (e[0]) fail((sht_status)e[0], "split-precision kernel: a bounded wait on the tensor cores expired");
  if (e[1]) fail(SHT_ERR_UNSUPPORTED, "split-precision mode needs finite inputs");
}

}  // namespace sht
