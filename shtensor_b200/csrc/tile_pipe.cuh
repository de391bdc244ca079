// tile_pipe.cuh -- pipelined output-stationary FP64 tile on the FP64 tensor cores (batched form).
//
// Arithmetic per output element is the reference XMM kernel's (src/Kernel/KernelImpl.cpp:
// 594-619, 661-683): c = beta*c (0 when beta is +0.0), then for every pair in order and every
// contracted index k ascending, c = fma(alpha*a_ik, b_kj, c).  The products run on
// mma.sync.m8n8k4.f64: on sm_100a one m8n8k4 step accumulates its four k in ascending order
// with one rounding each (measured bit-identical to the fma chain over 1.28M outputs), so
// feeding k ascending keeps the results bit-identical to the CPU restatement.  A k-chunk whose
// length is not a multiple of 4 is padded with a = -0.0, b = +0.0: fma(-0, +0, c) == c for
// every c, signed zeros included.
//
// Organisation:
//   * a tile's (pair, k-chunk) sequence is one stream of 16-deep chunks; chunk c+1 is copied
//     global -> shared with cp.async while chunk c is multiplied;
//   * operand offset tables are built two chunks ahead into double-buffered slots, so each
//     chunk costs one __syncthreads();
//   * 128 threads = 4 warps, each warp a WM x WN block of 8x8 accumulator fragments.
#pragma once

#include "tile_core.cuh"

namespace sht {

template <int TM_, int TN_, int WARPS_M_>
struct PipeCfg {
  static constexpr int TM = TM_, TN = TN_, TK = 16;
  static constexpr int NT = 128;
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = 4 / WARPS_M_;
  static constexpr int WM = TM / WARPS_M, WN = TN / WARPS_N;  // warp tile
  static constexpr int FM = WM / 8, FN = WN / 8;              // 8x8 fragments per warp
  static constexpr int PO = 8;  // operand pitch TM+8 doubles: fragment loads hit 2 wavefronts
  static constexpr int PC = 2;  // staging pitch TM+2 doubles: fragment stores hit 2 wavefronts
  static constexpr int LA = TM * TK / NT;  // A elements copied per thread per chunk
  static constexpr int LB = TN * TK / NT;
  static_assert(WM % 8 == 0 && WN % 8 == 0, "warp tile in 8x8 fragments");
  static_assert((TM * TK) % NT == 0 && (TN * TK) % NT == 0, "copy split");
};

template <class Cfg>
struct PipeSmem {
  static constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK;
  union {
    struct {
      double a[2][TK][TM + Cfg::PO];
      double b[2][TK][TN + Cfg::PO];
    } ab;
    double c[TN][TM + Cfg::PC];
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

// Offset tables of chunk `it` into table slot s (A rows and B columns for the pair, k offsets).
template <class Cfg>
__device__ __forceinline__ void chunk_tables(const ChunkIter& it, const TileMaps& mp, PipeSmem<Cfg>& sm, int s) {
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
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Element q of this thread's share of a chunk: (row or column index, k).  Rows/columns run
// fastest (coalesced when the operand's mode 0 is a free mode) unless kfast.
template <int TX>
__device__ __forceinline__ void chunk_elem(int q, int kfast, int TK, int& x, int& k) {
  const int e = threadIdx.x + q * 128;
  x = kfast ? e / TK : e % TX;
  k = kfast ? e % TK : e / TX;
}

// Global -> shared (asynchronous) for chunk `it` with table slot s into operand buffer buf.
// Out-of-range elements are zero-filled (source size 0; the source address is then a valid
// operand base that is never read).
template <class Cfg>
__device__ __forceinline__ void chunk_issue(const ChunkIter& it, PipeSmem<Cfg>& sm, int s, int buf, int mt, int nt,
                                            int a_kfast, int b_kfast, const double* dummy) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK;
  const int kc = (it.p < it.pe) ? min(TK, it.K - it.k0) : 0;
  const double* abase = kc ? it.a : dummy;
  const double* bbase = kc ? it.b : dummy;
#pragma unroll
  for (int q = 0; q < Cfg::LA; ++q) {
    int i, k;
    chunk_elem<TM>(q, a_kfast, TK, i, k);
    const bool ok = i < mt && k < kc;
    cp_async8(&sm.u.ab.a[buf][k][i], ok ? abase + sm.rowA[s][i] + sm.kA[s][k] : abase, ok ? 8 : 0);
  }
#pragma unroll
  for (int q = 0; q < Cfg::LB; ++q) {
    int j, k;
    chunk_elem<TN>(q, b_kfast, TK, j, k);
    const bool ok = j < nt && k < kc;
    cp_async8(&sm.u.ab.b[buf][k][j], ok ? bbase + sm.kB[s][k] + sm.colB[s][j] : bbase, ok ? 8 : 0);
  }
  cp_async_commit();
}

// After this thread's copies landed: a = alpha*a on the A elements it copied (the XMM kernel
// scales a before the fma; skipped when alpha == 1 where the product is exact), and a = -0.0
// in the k padding up to the next multiple of 4.
template <class Cfg>
__device__ __forceinline__ void chunk_fix(PipeSmem<Cfg>& sm, int buf, int a_kfast, double alpha, bool scale, int kc) {
  constexpr int TM = Cfg::TM, TK = Cfg::TK;
  const int kc4 = (kc + 3) & ~3;
  if (!scale && kc == kc4) return;
#pragma unroll
  for (int q = 0; q < Cfg::LA; ++q) {
    int i, k;
    chunk_elem<TM>(q, a_kfast, TK, i, k);
    double& v = sm.u.ab.a[buf][k][i];
    if (k < kc) {
      if (scale) v = mul_rn(alpha, v);
    } else if (k < kc4) {
      v = -0.0;
    }
  }
}

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Multiply one chunk (kc4 = k count rounded up to 4) into the warp's fragments.
template <class Cfg>
__device__ __forceinline__ void chunk_mma(const PipeSmem<Cfg>& sm, int buf, int kc4, int wm0, int wn0, int lane,
                                          double (&acc)[Cfg::FM][Cfg::FN][2]) {
  const int r = lane >> 2, q = lane & 3;
#pragma unroll 2
  for (int k = 0; k < kc4; k += 4) {
    double af[Cfg::FM], bf[Cfg::FN];
#pragma unroll
    for (int f = 0; f < Cfg::FM; ++f) af[f] = sm.u.ab.a[buf][k + q][wm0 + f * 8 + r];
#pragma unroll
    for (int f = 0; f < Cfg::FN; ++f) bf[f] = sm.u.ab.b[buf][k + q][wn0 + f * 8 + r];
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn) dmma884(acc[fm][fn], af[fm], bf[fn]);
  }
}

// One tile of one C block; pairs pb..pe-1.
template <class Cfg, class GetC, class GetPair>
__device__ __forceinline__ void tile_run_pipe(const TileMaps& mp, const TileScalars<double>& sc, int tile,
                                              GetC getc, GetPair getpair, int pb, int pe, int a_kfast,
                                              int b_kfast, PipeSmem<Cfg>& sm) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, NT = Cfg::NT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % Cfg::WARPS_M) * Cfg::WM, wn0 = (warp / Cfg::WARPS_M) * Cfg::WN;
  const int fr = lane >> 2, fc = 2 * (lane & 3);  // fragment element (row, column pair)

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

  double acc[Cfg::FM][Cfg::FN][2];
  if (sc.beta_zero) {
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn) acc[fm][fn][0] = acc[fm][fn][1] = 0.0;
  } else {
    for (int e = tid; e < TM * TN; e += NT) {
      const int i = e % TM, j = e / TM;
      sm.u.c[j][i] = (i < mt && j < nt) ? cptr[sm.rowC[i] + sm.colC[j]] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
      for (int fn = 0; fn < Cfg::FN; ++fn)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          acc[fm][fn][h] = mul_rn(sc.beta, sm.u.c[wn0 + fn * 8 + fc + h][wm0 + fm * 8 + fr]);
    __syncthreads();
  }

  if (!sc.alpha_zero && pb < pe) {
    const bool scale = sc.alpha != 1.0;
    ChunkIter cur{pb, pe, 0, 0, nullptr, nullptr, nullptr, nullptr};
    chunk_open(cur, mp, getpair);
    const double* dummy = cur.a;
    ChunkIter nxt = cur;
    chunk_next(nxt, TK, mp, getpair);
    chunk_tables<Cfg>(cur, mp, sm, 0);
    chunk_tables<Cfg>(nxt, mp, sm, 1);
    __syncthreads();
    chunk_issue<Cfg>(cur, sm, 0, 0, mt, nt, a_kfast, b_kfast, dummy);
    cp_async_wait_all();
    chunk_fix<Cfg>(sm, 0, a_kfast, sc.alpha, scale, min(TK, cur.K - cur.k0));
    __syncthreads();
    ChunkIter far = nxt;
    chunk_next(far, TK, mp, getpair);
    int slot = 0;
    while (cur.p < pe) {
      // 1. chunk c+1 into the other operand buffer, asynchronously (tables in slot^1)
      chunk_issue<Cfg>(nxt, sm, slot ^ 1, slot ^ 1, mt, nt, a_kfast, b_kfast, dummy);
      // 2. multiply chunk c
      chunk_mma<Cfg>(sm, slot, (min(TK, cur.K - cur.k0) + 3) & ~3, wm0, wn0, lane, acc);
      // 3. tables of chunk c+2 into slot (its last reader, chunk c's copy issue, is done)
      chunk_tables<Cfg>(far, mp, sm, slot);
      // 4. wait for chunk c+1; alpha scaling and k padding of its A elements
      cp_async_wait_all();
      if (nxt.p < pe) chunk_fix<Cfg>(sm, slot ^ 1, a_kfast, sc.alpha, scale, min(TK, nxt.K - nxt.k0));
      __syncthreads();
      cur = nxt;
      nxt = far;
      if (far.p < pe) chunk_next(far, TK, mp, getpair);
      slot ^= 1;
    }
  }

  // stage the fragments, then store along C's memory order (rows fastest)
#pragma unroll
  for (int fm = 0; fm < Cfg::FM; ++fm)
#pragma unroll
    for (int fn = 0; fn < Cfg::FN; ++fn)
#pragma unroll
      for (int h = 0; h < 2; ++h) sm.u.c[wn0 + fn * 8 + fc + h][wm0 + fm * 8 + fr] = acc[fm][fn][h];
  __syncthreads();
  for (int e = tid; e < TM * TN; e += NT) {
    const int i = e % TM, j = e / TM;
    if (i < mt && j < nt) cptr[sm.rowC[i] + sm.colC[j]] = sm.u.c[j][i];
  }
  __syncthreads();
}

}  // namespace sht
