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
// Operands come in matrix form (matform.cu): every A block as an m_pad x K4 column-major
// matrix with alpha applied and the K padding set to -0.0, every B block as an n_pad x K4
// matrix (columns fastest) with +0.0 padding, m_pad/n_pad even and each block 16-byte
// aligned.  So:
//   * a tile's (pair, k-chunk) sequence is one stream of 16-deep chunks; chunk c+1 is copied
//     global -> shared with 16-byte cp.async while chunk c is multiplied (one __syncthreads()
//     per chunk, no operand index tables);
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
  static_assert(WM % 8 == 0 && WN % 8 == 0, "warp tile in 8x8 fragments");
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
};

// Operand views of one pair: matrix-form bases, leading dimensions and K rounded up to 4.
struct PairView {
  const double* a;  // A_mat: element (row r, k) at a[k*lda + r]
  const double* b;  // B_mat: element (k, col c) at b[k*ldb + c]
  int lda, ldb, K4;
};

// Walks the (pair, k-chunk) sequence of one tile.  Every thread holds an identical copy.
struct ChunkIter {
  int p, pe, k0;
  PairView v;
};

template <class GetPair>
__device__ __forceinline__ void chunk_open(ChunkIter& it, GetPair& getpair) {
  if (it.p < it.pe) getpair(it.p, it.v);
}

template <class GetPair>
__device__ __forceinline__ void chunk_next(ChunkIter& it, int TK, GetPair& getpair) {
  it.k0 += TK;
  if (it.k0 >= it.v.K4) {
    it.k0 = 0;
    ++it.p;
    chunk_open(it, getpair);
  }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Global -> shared (asynchronous) of chunk `it` into operand buffer buf: kc4 k-rows of TM
// A rows and TN B columns, as 16-byte pairs; pairs past the block's padded extent are
// zero-filled (source size 0, source address the valid block base, never read).
template <class Cfg>
__device__ __forceinline__ void chunk_issue(const ChunkIter& it, PipeSmem<Cfg>& sm, int buf, int r0, int c0) {
  constexpr int TM = Cfg::TM, TN = Cfg::TN, TK = Cfg::TK, NT = Cfg::NT;
  if (it.p >= it.pe) return;
  const int kc4 = min(TK, it.v.K4 - it.k0);
  constexpr int HA = TM / 2, HB = TN / 2;
  for (int e = threadIdx.x; e < kc4 * HA; e += NT) {
    const int k = e / HA, r = 2 * (e % HA);
    const bool ok = r0 + r < it.v.lda;
    const double* src = it.v.a + (long long)(it.k0 + k) * it.v.lda + (ok ? r0 + r : 0);
    cp_async16(&sm.u.ab.a[buf][k][r], src, ok ? 16 : 0);
  }
  for (int e = threadIdx.x; e < kc4 * HB; e += NT) {
    const int k = e / HB, c = 2 * (e % HB);
    const bool ok = c0 + c < it.v.ldb;
    const double* src = it.v.b + (long long)(it.k0 + k) * it.v.ldb + (ok ? c0 + c : 0);
    cp_async16(&sm.u.ab.b[buf][k][c], src, ok ? 16 : 0);
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
                                              GetC getc, GetPair getpair, int pb, int pe, PipeSmem<Cfg>& sm) {
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
        off += (r % e) * stC[mp.row.y[t]];
        r /= e;
      }
      sm.rowC[i] = (i < mt) ? off : 0;
    } else {
      const int j = i - TM;
      int c = c0 + j, off = 0;
      for (int t = 0; t < mp.col.n; ++t) {
        const int e = cd[mp.col.y[t]];
        off += (c % e) * stC[mp.col.y[t]];
        c /= e;
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
    ChunkIter cur{pb, pe, 0, {}};
    chunk_open(cur, getpair);
    ChunkIter nxt = cur;
    chunk_next(nxt, TK, getpair);
    chunk_issue<Cfg>(cur, sm, 0, r0, c0);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    int slot = 0;
    while (cur.p < pe) {
      // 1. chunk c+1 into the other operand buffer, asynchronously
      chunk_issue<Cfg>(nxt, sm, slot ^ 1, r0, c0);
      cp_async_commit();
      // 2. multiply chunk c
      chunk_mma<Cfg>(sm, slot, min(TK, cur.v.K4 - cur.k0), wm0, wn0, lane, acc);
      // 3. chunk c+1 landed for every thread
      cp_async_wait_all();
      __syncthreads();
      cur = nxt;
      if (nxt.p < pe) chunk_next(nxt, TK, getpair);
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
