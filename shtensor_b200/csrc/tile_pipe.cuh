// tile_pipe.cuh -- software-pipelined output-stationary FP64 tile (batched form).
//
// Same arithmetic as tile_core.cuh (per element: c = beta*c or 0, then for every pair in
// order and k ascending c = fma(alpha*a, b, c): bit-identical results), reorganised for
// throughput:
//   * the (pair, k-chunk) sequence of a tile is one stream of chunks; chunk c+1 is copied
//     from global to shared memory with cp.async while chunk c is multiplied;
//   * operand offset tables are built two chunks ahead into a double-buffered table, so each
//     chunk costs one __syncthreads();
//   * 128 threads, RM x RN accumulators per thread.
#pragma once

#include "tile_core.cuh"

namespace sht {

template <int TM_, int TN_, int RM_, int RN_>
struct PipeCfg {
  static constexpr int TM = TM_, TN = TN_, TK = 16, RM = RM_, RN = RN_;
  static constexpr int NT = (TM / RM) * (TN / RN);
  static constexpr int P = 8;  // row pitch = TM+8 doubles: staging stores hit 2 wavefronts
  static constexpr int LA = TM * TK / NT;  // A elements loaded per thread per chunk
  static constexpr int LB = TN * TK / NT;
  static_assert(NT == 128, "pipelined tiles run 128 threads");
  static_assert((TM * TK) % NT == 0 && (TN * TK) % NT == 0, "load split");
};

template <class Cfg>
struct PipeSmem {
  static constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, P = Cfg::P;
  union {
    struct {
      double a[2][TK][TM + P];
      double b[2][TK][TN + P];
    } ab;
    double c[TN][TM + P];
  } u;
  int rowC[TM], colC[TN];
  int rowA[2][TM], colB[2][TN];
  int kA[2][TK], kB[2][TK];
  short rdig[kMaxOrder][TM];
  short cdig[kMaxOrder][TN];
};

// Walks the (pair, k-chunk) sequence of one tile.  Every thread holds an identical copy.
struct ChunkIter {
  int p, pe, k0, K;
  const double* a;
  const double* b;
  const int* ad;
  const int* bd;
};

template <class GetPair>
__device__ __forceinline__ void chunk_open(ChunkIter& it, const TileMaps& mp, GetPair& getpair) {
  if (it.p < it.pe) {
    getpair(it.p, it.a, it.ad, it.b, it.bd);
    int K = 1;
    for (int t = 0; t < mp.kk.n; ++t) K *= it.ad[mp.kk.x[t]];
    it.K = K;
  }
}

template <class GetPair>
__device__ __forceinline__ void chunk_next(ChunkIter& it, int TK, const TileMaps& mp, GetPair& getpair) {
  it.k0 += TK;
  if (it.k0 >= it.K) {
    it.k0 = 0;
    ++it.p;
    chunk_open(it, mp, getpair);
  }
}

// Offset tables of chunk `it` into table slot s (rows/cols of A/B for the pair, k offsets).
template <class Cfg>
__device__ __forceinline__ void chunk_tables(const ChunkIter& it, const TileMaps& mp, PipeSmem<Cfg>& sm, int s,
                                             int mt, int nt) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, NT = Cfg::NT;
  if (it.p >= it.pe) return;
  int stA[kMaxOrder], stB[kMaxOrder];
  block_strides(it.ad, mp.oA, stA);
  block_strides(it.bd, mp.oB, stB);
  const int kc = min(TK, it.K - it.k0);
  for (int i = threadIdx.x; i < TM + TN + TK; i += NT) {
    if (i < TM) {
      int off = 0;
      for (int t = 0; t < mp.row.n; ++t) off += sm.rdig[t][i] * stA[mp.row.x[t]];
      sm.rowA[s][i] = off;
    } else if (i < TM + TN) {
      const int j = i - TM;
      int off = 0;
      for (int t = 0; t < mp.col.n; ++t) off += sm.cdig[t][j] * stB[mp.col.x[t]];
      sm.colB[s][j] = off;
    } else {
      const int k = i - TM - TN;
      int q = it.k0 + k, oa = 0, ob = 0;
      if (k < kc) {
        for (int t = 0; t < mp.kk.n; ++t) {
          const int e = it.ad[mp.kk.x[t]];
          const int dgt = q % e;
          q /= e;
          oa += dgt * stA[mp.kk.x[t]];
          ob += dgt * stB[mp.kk.y[t]];
        }
      }
      sm.kA[s][k] = oa;
      sm.kB[s][k] = ob;
    }
  }
  (void)mt; (void)nt;
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Global -> shared (asynchronous) for chunk `it` with table slot s into operand buffer buf.
// A element e of this thread is (row i, k) with i fastest when a_kfast == 0, k fastest
// otherwise (likewise B with columns).  Out-of-range elements are zero-filled (source size 0,
// the source address then points at the operand base, which is never read).
template <class Cfg>
__device__ __forceinline__ void chunk_issue(const ChunkIter& it, PipeSmem<Cfg>& sm, int s, int buf, int mt, int nt,
                                            int a_kfast, int b_kfast, const double* dummy) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, NT = Cfg::NT;
  const int kc = (it.p < it.pe) ? min(TK, it.K - it.k0) : 0;
  const double* abase = kc ? it.a : dummy;
  const double* bbase = kc ? it.b : dummy;
#pragma unroll
  for (int q = 0; q < Cfg::LA; ++q) {
    const int e = threadIdx.x + q * NT;
    const int i = a_kfast ? e / TK : e % TM;
    const int k = a_kfast ? e % TK : e / TM;
    const bool ok = i < mt && k < kc;
    cp_async8(&sm.u.ab.a[buf][k][i], ok ? abase + sm.rowA[s][i] + sm.kA[s][k] : abase, ok ? 8 : 0);
  }
#pragma unroll
  for (int q = 0; q < Cfg::LB; ++q) {
    const int e = threadIdx.x + q * NT;
    const int j = b_kfast ? e / TK : e % TN;
    const int k = b_kfast ? e % TK : e / TN;
    const bool ok = j < nt && k < kc;
    cp_async8(&sm.u.ab.b[buf][k][j], ok ? bbase + sm.kB[s][k] + sm.colB[s][j] : bbase, ok ? 8 : 0);
  }
  cp_async_commit();
}

// After the copies of this thread landed: a = alpha*a on the A elements it copied (the XMM
// kernel scales a before the fma).  Skipped for alpha == 1, where the product is exact.
template <class Cfg>
__device__ __forceinline__ void chunk_scale(PipeSmem<Cfg>& sm, int buf, int a_kfast, double alpha) {
  constexpr int TM = Cfg::TM, TK = Cfg::TK, NT = Cfg::NT;
#pragma unroll
  for (int q = 0; q < Cfg::LA; ++q) {
    const int e = threadIdx.x + q * NT;
    const int i = a_kfast ? e / TK : e % TM;
    const int k = a_kfast ? e % TK : e / TM;
    sm.u.ab.a[buf][k][i] = mul_rn(alpha, sm.u.ab.a[buf][k][i]);
  }
}

// Thread (tx, ty) owns rows tx + i*XT and columns ty + j*YT: a warp's operand reads are
// consecutive doubles (one wavefront per load, no bank conflicts).
template <class Cfg>
__device__ __forceinline__ void chunk_mma(const PipeSmem<Cfg>& sm, int buf, int kc, int tx, int ty,
                                          double (&acc)[Cfg::RM][Cfg::RN]) {
  constexpr int RM = Cfg::RM, RN = Cfg::RN, XT = Cfg::TM / RM, YT = Cfg::TN / RN;
#pragma unroll 4
  for (int k = 0; k < kc; ++k) {
    double a[RM], b[RN];
#pragma unroll
    for (int i = 0; i < RM; ++i) a[i] = sm.u.ab.a[buf][k][tx + i * XT];
#pragma unroll
    for (int j = 0; j < RN; ++j) b[j] = sm.u.ab.b[buf][k][ty + j * YT];
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
}

// One tile of one C block; pairs pb..pe-1.
template <class Cfg, class GetC, class GetPair>
__device__ __forceinline__ void tile_run_pipe(const TileMaps& mp, const TileScalars<double>& sc, int tile,
                                              GetC getc, GetPair getpair, int pb, int pe, int a_kfast,
                                              int b_kfast, PipeSmem<Cfg>& sm) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, RM = Cfg::RM, RN = Cfg::RN, NT = Cfg::NT;
  constexpr int XT = TM / RM, YT = TN / RN;
  const int tid = threadIdx.x;
  const int tx = tid % XT, ty = tid / XT;

  double* cptr;
  const int* cd;
  getc(cptr, cd);
  int stC[kMaxOrder];
  block_strides(cd, mp.oC, stC);
  int m = 1, n = 1;
  for (int t = 0; t < mp.row.n; ++t) m *= cd[mp.row.y[t]];
  for (int t = 0; t < mp.col.n; ++t) n *= cd[mp.col.y[t]];
  const int ntr = (m + TM - 1) / TM;
  const int r0 = (tile % ntr) * TM, c0 = (tile / ntr) * TN;
  const int mt = min(TM, m - r0), nt = min(TN, n - c0);

  for (int i = tid; i < TM + TN; i += NT) {
    if (i < TM) {
      int r = r0 + i, off = 0;
      for (int t = 0; t < mp.row.n; ++t) {
        const int e = cd[mp.row.y[t]];
        const int dgt = (i < mt) ? r % e : 0;
        r /= e;
        sm.rdig[t][i] = (short)dgt;
        off += dgt * stC[mp.row.y[t]];
      }
      sm.rowC[i] = (i < mt) ? off : 0;
    } else {
      const int j = i - TM;
      int c = c0 + j, off = 0;
      for (int t = 0; t < mp.col.n; ++t) {
        const int e = cd[mp.col.y[t]];
        const int dgt = (j < nt) ? c % e : 0;
        c /= e;
        sm.cdig[t][j] = (short)dgt;
        off += dgt * stC[mp.col.y[t]];
      }
      sm.colC[j] = (j < nt) ? off : 0;
    }
  }
  __syncthreads();

  double acc[RM][RN];
  if (sc.beta_zero) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = 0.0;
  } else {
    for (int e = tid; e < TM * TN; e += NT) {
      const int i = e % TM, j = e / TM;
      sm.u.c[j][i] = (i < mt && j < nt) ? cptr[sm.rowC[i] + sm.colC[j]] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = mul_rn(sc.beta, sm.u.c[ty + j * YT][tx + i * XT]);
    __syncthreads();
  }

  if (!sc.alpha_zero && pb < pe) {
    const bool scale = sc.alpha != 1.0;
    // chunk iterators for c (cur), c+1 (nxt) and c+2 (far)
    ChunkIter cur{pb, pe, 0, 0, nullptr, nullptr, nullptr, nullptr};
    chunk_open(cur, mp, getpair);
    const double* dummy = cur.a;
    ChunkIter nxt = cur;
    chunk_next(nxt, TK, mp, getpair);
    chunk_tables<Cfg>(cur, mp, sm, 0, mt, nt);
    chunk_tables<Cfg>(nxt, mp, sm, 1, mt, nt);
    __syncthreads();
    chunk_issue<Cfg>(cur, sm, 0, 0, mt, nt, a_kfast, b_kfast, dummy);
    cp_async_wait_all();
    if (scale) chunk_scale<Cfg>(sm, 0, a_kfast, sc.alpha);
    __syncthreads();
    ChunkIter far = nxt;
    chunk_next(far, TK, mp, getpair);
    int slot = 0;
    while (cur.p < pe) {
      // 1. chunk c+1 into the other operand buffer, asynchronously (tables in slot^1)
      chunk_issue<Cfg>(nxt, sm, slot ^ 1, slot ^ 1, mt, nt, a_kfast, b_kfast, dummy);
      // 2. multiply chunk c
      chunk_mma<Cfg>(sm, slot, min(TK, cur.K - cur.k0), tx, ty, acc);
      // 3. tables of chunk c+2 into slot (free: chunk c's copies were issued last iteration)
      chunk_tables<Cfg>(far, mp, sm, slot, mt, nt);
      // 4. wait for chunk c+1, scale its A by alpha
      cp_async_wait_all();
      if (scale) chunk_scale<Cfg>(sm, slot ^ 1, a_kfast, sc.alpha);
      __syncthreads();
      cur = nxt;
      nxt = far;
      if (far.p < pe) chunk_next(far, TK, mp, getpair);
      slot ^= 1;
    }
  }

#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < RN; ++j) sm.u.c[ty + j * YT][tx + i * XT] = acc[i][j];
  __syncthreads();
  for (int e = tid; e < TM * TN; e += NT) {
    const int i = e % TM, j = e / TM;
    if (i < mt && j < nt) cptr[sm.rowC[i] + sm.colC[j]] = sm.u.c[j][i];
  }
  __syncthreads();
}

}  // namespace sht
