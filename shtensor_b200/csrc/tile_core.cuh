// tile_core.cuh -- output-stationary contraction tile for block-sparse and stacked blocks.
//
// One CTA owns a TM x TN tile of one C block (rows = A's free modes, columns = B's free
// modes, the matrix view of src/Basics/ContractInfo.h:284-291).  It runs over every block
// pair feeding that C block in pair order and over each pair's contracted index in
// ascending order, and writes the tile once.  Per output element the arithmetic is the
// reference XMM kernel's (src/Kernel/KernelImpl.cpp:594-619, 661-683):
//     c = beta*c  (c = 0 when beta is +0.0);   per k:  c = fma(alpha*a_ik, b_kj, c)
// so results are bit-identical to the CPU restatement.  Operands are gathered straight from
// the blocks' own column-major layouts through per-tile offset tables (the permute of the
// LAPACK path, Utils::reshape, never materialises); the C tile is staged through shared
// memory so its loads and stores run along C's fastest modes.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sht_internal.h"
#include "tile_types.h"

namespace sht {

template <int TM, int TN, int TK, int RM, int RN>
struct TileCfg {
  static constexpr int kTM = TM, kTN = TN, kTK = TK, kRM = RM, kRN = RN;
  static constexpr int kThreads = (TM / RM) * (TN / RN);
  static constexpr int kPad = 8;
};

template <typename T, class Cfg>
struct TileSmem {
  static constexpr int TM = Cfg::kTM, TN = Cfg::kTN, TK = Cfg::kTK, P = Cfg::kPad;
  union {
    struct {
      T a[TK][TM + P];
      T b[TK][TN + P];
    } ab;
    T c[TN][TM + P];
  } u;
  int rowC[TM], rowA[TM], colC[TN], colB[TN], kA[TK], kB[TK];
  short rdig[kMaxOrder][TM];
  short cdig[kMaxOrder][TN];
};

__device__ __forceinline__ void block_strides(const int* dims, int order, int* st) {
  int s = 1;
#pragma unroll
  for (int d = 0; d < kMaxOrder; ++d) {
    if (d < order) { st[d] = s; s *= dims[d]; }
  }
}

// Products that must round on their own (never contracted into a neighbouring fma).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// Core: compute tile `tile` of one C block.  getc(ptr, dims) gives the C block, pairs
// pb..pe-1 are visited in order, getpair(p, a, adims, b, bdims) gives each pair's operands.
template <typename T, class Cfg, class GetC, class GetPair>
__device__ __forceinline__ void tile_run(const TileMaps& mp, const TileScalars<T>& sc, int tile,
                                         GetC getc, GetPair getpair, int pb, int pe,
                                         TileSmem<T, Cfg>& sm) {
  constexpr int TM = Cfg::kTM, TN = Cfg::kTN, TK = Cfg::kTK, RM = Cfg::kRM, RN = Cfg::kRN;
  constexpr int NT = Cfg::kThreads;
  constexpr int XT = TM / RM, YT = TN / RN;  // threads along rows / columns
  const int tid = threadIdx.x;
  const int tx = tid % XT, ty = tid / XT;

  T* cptr;
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

  // row / column digits and C offsets for this tile
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

  T acc[RM][RN];
  if (sc.beta_zero) {
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = T(0);
  } else {
    for (int e = tid; e < TM * TN; e += NT) {
      const int i = e % TM, j = e / TM;
      sm.u.c[j][i] = (i < mt && j < nt) ? cptr[sm.rowC[i] + sm.colC[j]] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RM; ++i)
#pragma unroll
      for (int j = 0; j < RN; ++j) acc[i][j] = mul_rn(sc.beta, sm.u.c[ty + j * YT][tx + i * XT]);
    __syncthreads();
  }

  if (!sc.alpha_zero) {
    for (int p = pb; p < pe; ++p) {
      const T* ap;
      const T* bp;
      const int* ad;
      const int* bd;
      getpair(p, ap, ad, bp, bd);
      int stA[kMaxOrder], stB[kMaxOrder];
      block_strides(ad, mp.oA, stA);
      block_strides(bd, mp.oB, stB);
      int K = 1;
      for (int t = 0; t < mp.kk.n; ++t) K *= ad[mp.kk.x[t]];
      for (int i = tid; i < TM + TN; i += NT) {
        if (i < TM) {
          int off = 0;
          for (int t = 0; t < mp.row.n; ++t) off += sm.rdig[t][i] * stA[mp.row.x[t]];
          sm.rowA[i] = off;
        } else {
          const int j = i - TM;
          int off = 0;
          for (int t = 0; t < mp.col.n; ++t) off += sm.cdig[t][j] * stB[mp.col.x[t]];
          sm.colB[j] = off;
        }
      }
      for (int k0 = 0; k0 < K; k0 += TK) {
        const int kc = min(TK, K - k0);
        for (int k = tid; k < TK; k += NT) {
          int q = k0 + k, oa = 0, ob = 0;
          if (k < kc) {
            for (int t = 0; t < mp.kk.n; ++t) {
              const int e = ad[mp.kk.x[t]];
              const int dgt = q % e;
              q /= e;
              oa += dgt * stA[mp.kk.x[t]];
              ob += dgt * stB[mp.kk.y[t]];
            }
          }
          sm.kA[k] = oa;
          sm.kB[k] = ob;
        }
        __syncthreads();
        // gather A (alpha applied here, as the XMM kernel scales a before the fma) and B
        for (int e = tid; e < TM * TK; e += NT) {
          const int i = e % TM, k = e / TM;
          sm.u.ab.a[k][i] = (i < mt && k < kc) ? mul_rn(sc.alpha, ap[sm.rowA[i] + sm.kA[k]]) : T(0);
        }
        for (int e = tid; e < TN * TK; e += NT) {
          const int j = e % TN, k = e / TN;
          sm.u.ab.b[k][j] = (j < nt && k < kc) ? bp[sm.kB[k] + sm.colB[j]] : T(0);
        }
        __syncthreads();
        if (kc == TK) {
#pragma unroll 4
          for (int k = 0; k < TK; ++k) {
            T a[RM], b[RN];
#pragma unroll
            for (int i = 0; i < RM; ++i) a[i] = sm.u.ab.a[k][tx + i * XT];
#pragma unroll
            for (int j = 0; j < RN; ++j) b[j] = sm.u.ab.b[k][ty + j * YT];
#pragma unroll
            for (int i = 0; i < RM; ++i)
#pragma unroll
              for (int j = 0; j < RN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
          }
        } else {
          for (int k = 0; k < kc; ++k) {
            T a[RM], b[RN];
#pragma unroll
            for (int i = 0; i < RM; ++i) a[i] = sm.u.ab.a[k][tx + i * XT];
#pragma unroll
            for (int j = 0; j < RN; ++j) b[j] = sm.u.ab.b[k][ty + j * YT];
#pragma unroll
            for (int i = 0; i < RM; ++i)
#pragma unroll
              for (int j = 0; j < RN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
          }
        }
        __syncthreads();
      }
    }
  }

  // stage and store the tile along C's memory order (rows fastest)
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
