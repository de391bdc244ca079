// split.cu -- split-precision (Ozaki scheme) contraction on the INT8 tensor cores (tcgen05).
//
// Every A row (of every A block, after alpha) and every B column is scaled by a power of two
// 2^-e so its entries lie in (-1, 1), then cut into S slices of 7 bits:
//     x = sum_{t=1..S} 2^(-7t) s_t,   s_t = trunc(128 * remainder) in [-127, 127]
// (exact up to the truncated tail, < 2^(-7S) of the row / column maximum).  A block pair's
// product is then  C(r,c) = 2^(e_r + f_c) * sum_g 2^(-7g) * P_g(r,c),  P_g = sum_{t+u=g} A_t B_u
// over g = 2..S+1 (the triangle t+u <= S+1; dropped terms are below the truncation error).
// Each P_g is an exact INT32 sum, accumulated by tcgen05.mma kind::i8 into its own TMEM
// columns; the epilogue reads the groups back (tcgen05.ld), combines them, scales by
// 2^(e_r+f_c) and adds into FP64 accumulators held in registers, one pair after another in
// the canonical pair order.  FP64 is used only for the reassembly, the accumulation into C
// and the scaling exponents.
//
// Layout.  k_slice writes the slices of every block already in the order the tensor cores
// read them from shared memory: for A, per 128-row tile and 32-wide k-step, the S slices'
// 128 x 32-byte slabs one after another, each slab in K-major core matrices (8 rows x 16
// bytes); B likewise with 32-row (column) tiles.  One k-step of one pair is therefore two
// contiguous ranges, S*4 KB of A and S*1 KB of B, fetched with two bulk copies
// (cp.async.bulk, completion counted on an mbarrier).  The B slabs of one k-step lie one
// after another, so slices u = 1..n together form one operand of 32*n columns.
//
// Kernel (k_split, one 384-thread CTA per SM, persistent over 128 x 32 tiles of C):
//   warp 0      producer: for every (tile, pair, k-step) waits for a free stage of the
//               shared-memory ring (split_stages(S) deep) and issues its two bulk copies;
//   warp 1      MMA issuer: waits for the stage and issues S MMAs, A slice t times B slices
//               1..S+1-t (N = 32*(S+1-t)) into TMEM groups t+1..S+1 of one of two
//               accumulator sets; frees the stage with tcgen05.commit and, at the end of a
//               pair, commits the accumulator set to the epilogue;
//   warps 2-9   epilogue: 4 TMEM lane quarters x 2 column halves of 16 columns; reassemble a
//               pair's groups while the tensor cores already work on the next pair (second
//               TMEM set), accumulate in registers, store the tile at the end;
//   warp 10     record warp: resolves each pair's copy sources and exponent rows into a
//               shared ring that the producer, the MMA issuer and the slot warp read;
//   warp 11     slot warp: loads each tile's record and row / column offsets, and each
//               pair's row exponents, column exponents and column scales, into the tile and
//               exponent rings with ordinary loads and stores.  The bulk copies of one SM
//               run one after another, each taking hundreds of cycles however small, so
//               only the operand slabs (two large copies per k-step) go through them.
// Per-tile and per-pair records are built at plan time so that each role reads one record
// per tile and per pair.  Every wait is bounded: a role that gives up raises a CTA-wide abort
// flag and the error word (SHT_ERR_TIMEOUT); the others leave their waits on the flag, the
// MMA issuer drains the tensor core (bounded), the producer waits for its copies in flight
// (bounded), and TMEM is freed before the CTA exits.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "contract.h"
#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

constexpr int kSplitM = 128, kSplitN = 32, kSplitK = 32, kMaxSlices = 8;
// Operand stages of the shared-memory ring: as many as fit beside the slots in the 227 KB of
// one CTA (6 at S = 7).  A stage holds one k-step of one pair, S * 5 KB; the copies of a stage
// take longer than the tensor core needs for one, so depth hides their latency.
constexpr int kSplitSmemBudget = 227 * 1024;
constexpr int kSplitSlotBytes = 8 * 1024;  // tile and exponent rings, barriers (upper bound)
__host__ __device__ constexpr int split_stages(int S) {
  return (kSplitSmemBudget - kSplitSlotBytes) / (S * 5 * 1024) > 8 ? 8
                                                                  : (kSplitSmemBudget - kSplitSlotBytes) / (S * 5 * 1024);
}
constexpr int kAChunk = kSplitM * kSplitK;      // bytes of one A slab (128 rows x 32 k)
constexpr int kBChunk = kSplitN * kSplitK;      // bytes of one B slab (32 columns x 32 k)
constexpr int kBufCols = kMaxSlices * kSplitN;  // TMEM columns of one accumulator set (8 groups)
constexpr int kSplitTmemCols = 2 * kBufCols;    // two sets: 512 columns, the whole TMEM of an SM
constexpr int kEpiWarps = 8;                    // 4 TMEM lane quarters x (kEpiWarps / 4) column parts
constexpr int kEpiCols = kSplitN / (kEpiWarps / 4);  // tile columns per epilogue thread
constexpr int kTileSlots = 4, kExpSlots = 4;    // depth of the tile-record and exponent rings
constexpr int kRecSlots = 16;                   // depth of the record ring (power of two)
constexpr int kRecWarp = 2 + kEpiWarps;         // the record warp, after the epilogue warps
constexpr int kSlotWarp = kRecWarp + 1;         // the slot warp, last
// 12 warps: producer, MMA issuer, 8 epilogue warps, record warp, slot warp.  Twelve warps
// put three on each SM sub-partition, whose 16K registers then allow 168 per thread (eleven
// would allow only 160 per thread under the launch bound's rounding).
constexpr int kSplitThreads = 64 + kEpiWarps * 32 + 64;

// ------------------------------------------------------------------ slicing

// byte offset of (row r, k) inside one K-major slab of 32-byte rows: core matrices of 8 rows
// x 16 bytes, 128 bytes apart along k (LBO) and 256 bytes apart along rows (SBO)
__host__ __device__ __forceinline__ int slab_offset(int r, int k) {
  return (r >> 3) * 256 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

// Flag words of one split execute (device, zeroed before the slicer runs):
//   [0] set by the slicer when an operand holds a non-finite value: the tensor-core kernel
//       then writes nothing and the FP64 tile kernel computes the contraction instead;
//   [1] set when a row or column exponent lies outside the range of the scale-folded
//       reassembly (A rows: 2^e with -900 <= e <= 960; B columns: 2^e a normal double): the
//       kernel then scales every element on its own.
constexpr int kFlagNonFinite = 0, kFlagGeneralExp = 1;
constexpr int kExpLoA = -900, kExpHiA = 960, kExpLoB = -1022, kExpHiB = 1023;

// One operand of the slicer: A (rows = A's free modes, tiles of 128 rows, alpha folded into the
// values) or B (rows = B's free modes, i.e. C columns, tiles of 32 rows, column scales written).
struct SliceOperand {
  const double* src;           // the operand's block data
  const long long* src_off;    // element offset of every block
  const int* dims;             // block extents, order per block
  const long long* out_off;    // byte offset of every block's slices
  const long long* exp_off;    // offset of every block's row exponents
  const long long* istart;     // first slicer item of every block (items of 32 rows)
  signed char* out;
  short* expo;
  double* pscale;              // B: 2^e per column (0 when e is outside [elo, ehi]); A: null
  double scale;
  long long nblocks, nitems;
  ModeMap fm, km;              // the row modes and the contracted modes
  int order, R, elo, ehi;
};
struct SliceArgs {
  SliceOperand op[2];          // A, then B: items of A first, then items of B
  int* flags;
};

// The block holding item it: the last b with istart[b] <= it (istart[0] = 0, non-decreasing),
// found by the warp 32 ways at a time (two dependent loads for up to 1024 blocks).
__device__ __forceinline__ long long item_block(const long long* __restrict__ istart, long long nblocks, long long it,
                                                int lane) {
  long long lo = 0, n = nblocks;  // invariant: istart[lo] <= it, and lo + n == nblocks or istart[lo + n] > it
  while (n > 1) {
    const long long step = (n + 31) >> 5;
    const long long off = (long long)lane * step;
    const bool le = off < n && __ldg(istart + lo + off) <= it;
    const int last = 31 - __clz(__ballot_sync(0xffffffffu, le));  // lane 0 (off 0) always holds
    lo += (long long)last * step;
    n = min(step, n - (long long)last * step);
  }
  return lo;
}

// d = bytes of {b, a} chosen by the selector nibbles of c; a nibble with bit 3 set gives the
// sign of its byte replicated over 8 bits
__device__ __forceinline__ unsigned prmt(unsigned a, unsigned b, unsigned c) {
  unsigned d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// 8-byte global -> shared copy (cp.async), zero-filled when bytes is 0
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit8() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait8() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// offset of index idx of the modes mm within a block of extents d and strides st
__device__ __forceinline__ int mode_offset(const int* d, const int* st, const ModeMap& mm, int idx) {
  int off = 0;
  for (int t = 0; t < mm.n; ++t) {
    const int e = d[mm.x[t]];
    off += (idx % e) * st[mm.x[t]];
    idx /= e;
  }
  return off;
}

// True when the modes mm are consecutive and ascending (x[t+1] = x[t] + 1): the column-major
// strides then compose, and combined index idx lies at idx * st[x[0]] in every block.
__device__ __forceinline__ bool linear_modes(const ModeMap& mm) {
  bool lin = true;
  for (int t = 1; t < mm.n; ++t) lin = lin && mm.x[t] == mm.x[t - 1] + 1;
  return lin;
}

// Where one slicer item lies: its operand, its block (and the block's item range), the block's
// extents, and this lane's row in the block.
struct SliceLoc {
  long long b, bstart, bend;
  int opb, m, K, r;
};

// The location of item `item` (items of A first, then of B).  A CTA walks a contiguous range of
// items, so the block of the previous item (prev) is reused while the item stays inside it.
__device__ __forceinline__ SliceLoc slice_locate(const SliceArgs& g, long long item, const SliceLoc& prev, int lane) {
  const long long na = g.op[0].nitems;
  const int opb = item >= na ? 1 : 0;
  const SliceOperand& o = g.op[opb];
  const long long it = opb ? item - na : item;
  SliceLoc L;
  if (prev.opb == opb && it >= prev.bstart && it < prev.bend) {
    L = prev;
  } else {
    L.opb = opb;
    L.b = item_block(o.istart, o.nblocks, it, lane);
    L.bstart = o.istart[L.b];
    L.bend = L.b + 1 < o.nblocks ? o.istart[L.b + 1] : o.nitems;
    const int* d = o.dims + L.b * o.order;
    int m = 1, K = 1;
    for (int t = 0; t < o.fm.n; ++t) m *= d[o.fm.x[t]];
    for (int t = 0; t < o.km.n; ++t) K *= d[o.km.x[t]];
    L.m = m;
    L.K = K;
  }
  L.r = (int)(it - L.bstart) * 32 + lane;
  return L;
}

// Slices t = 1..S of the 8 values v (|v| * 2^-e < 1) of one row and one 8-wide k-chunk,
// stored as one 8-byte word per slice at out + base + (t - 1) * slab.  z = 1 + |y|, y = v 2^-e,
// rounded toward zero holds |y|'s first 52 bits in its mantissa, so slice t (t <= 7) is the
// 7-bit field of fraction bits 7t-6 .. 7t, negated when v is negative: exactly the digits of
// repeated s_t = trunc(128 * remainder).  Slice 8 takes fraction bits 50..52 from z and
// 53..56 from the exact tail |y| - (z - 1).  Four slices are packed into a register by byte
// permutes and negated four bytes at once ((0x80 - b) ^ 0x80 = -b mod 256 for 0 <= b <= 127,
// with no carry between bytes).
template <int S>
__device__ __forceinline__ void slice_chunk(const double (&v)[8], int e, signed char* out, long long base,
                                            long long slab) {
  // |v| * 2^-e is exact when 2^-e is a normal double and the product is normal; a product
  // below 2^-1022 has only zero slices either way.  Other exponents scale with scalbn.
  const bool mul = e >= -1022 && e <= 1022;
  const double inv = mul ? __longlong_as_double((long long)(1023 - e) << 52) : 0.0;
  unsigned w[S][2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    // byte masks of the four values' signs: 0xff where negative
    const unsigned sm = prmt(prmt((unsigned)__double2hiint(v[4 * q]), (unsigned)__double2hiint(v[4 * q + 1]), 0x00fbu),
                             prmt((unsigned)__double2hiint(v[4 * q + 2]), (unsigned)__double2hiint(v[4 * q + 3]), 0x00fbu),
                             0x5410u);
    const unsigned s1 = sm & 0x01010101u;
    unsigned zh[4], zl[4], d8[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double y = mul ? fabs(v[4 * q + i]) * inv : fabs(scalbn(v[4 * q + i], -e));
      const double z = __dadd_rz(y, 1.0);
      zh[i] = (unsigned)__double2hiint(z);
      zl[i] = (unsigned)__double2loint(z);
      if constexpr (S == 8) {
        const double tail = y - (z - 1.0);  // exact: the bits of |y| below 2^-52
        d8[i] = ((zl[i] & 7u) << 4) | (unsigned)__double2int_rz(tail * 72057594037927936.0);
      }
    }
#pragma unroll
    for (int t = 1; t <= S; ++t) {
      unsigned x[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        // fraction bits 7t-6 .. 7t of z sit at mantissa bits 58-7t .. 52-7t
        if (t == 1) x[i] = zh[i] >> 13;
        else if (t == 2) x[i] = zh[i] >> 6;
        else if (t == 3) x[i] = __funnelshift_r(zl[i], zh[i], 31);
        else if (t == 4) x[i] = zl[i];  // already byte-aligned: byte 3
        else if (t == 5) x[i] = zl[i] >> 17;
        else if (t == 6) x[i] = zl[i] >> 10;
        else if (t == 7) x[i] = zl[i] >> 3;
        else x[i] = d8[i];
      }
      const unsigned sel = t == 4 ? 0x73u : 0x40u;  // byte 0 (or 3) of the first and second word
      const unsigned pk = prmt(prmt(x[0], x[1], sel), prmt(x[2], x[3], sel), 0x5410u);
      w[t - 1][q] = (((pk ^ sm) & 0x7f7f7f7fu) + s1) ^ (sm & 0x80808080u);
    }
  }
#pragma unroll
  for (int t = 0; t < S; ++t)
    *reinterpret_cast<int2*>(out + base + t * slab) = make_int2((int)w[t][0], (int)w[t][1]);
}

// Items of 32 rows of one block; a 256-thread CTA walks a contiguous range of them.  Lane = row;
// warp w takes the 8-wide k-chunks w, w+8, ... of the row (a warp's load of one k is 32
// consecutive rows of a column-major block).  An item with K <= 64 (every row one chunk per
// warp at most) is copied into shared memory (8-byte cp.async, zero-filled past the block)
// while the CTA slices the previous one: two buffers, one item ahead.  Rows with K > 64 read
// their values from global memory twice (maximum, then slices).  The row maximum is reduced
// over the eight warps in shared memory and gives the row's exponent e (rows padded up to the
// tile height R get 0); the slices are stored in tile order:
//   out[((tile * ksteps + ks) * S + t) * R * 32 + slab_offset(row % R, k)].
// Rows past the block and k past K are zero.  With pscale set (B columns), the row's scale 2^e
// is also written as a double (0 when e is outside [elo, ehi]).
constexpr int kSliceWarps = 8, kSliceHoldK = 64, kSliceCtas = 4;  // CTAs per SM
template <int S>
__global__ void __launch_bounds__(kSliceWarps * 32, kSliceCtas) k_slice(const __grid_constant__ SliceArgs g) {
  __shared__ __align__(16) double buf[2][kSliceHoldK][32];
  __shared__ double wmax[kSliceWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long nitems = g.op[0].nitems + g.op[1].nitems;
  const long long per = (nitems + gridDim.x - 1) / gridDim.x;
  const long long i0 = blockIdx.x * per, i1 = min(nitems, i0 + per);
  if (i0 >= i1) return;

  // copies of item L into buffer bi (nothing for an item with K > 64)
  auto prefetch = [&](const SliceLoc& L, int bi) {
    if (L.K > kSliceHoldK || L.r - lane >= L.m) return;  // read directly, or rows all past the block
    const SliceOperand& o = g.op[L.opb];
    const int* d = o.dims + L.b * o.order;
    int st[kMaxOrder];
    block_strides(d, o.order, st);
    const bool live = L.r < L.m;
    const double* src = o.src + o.src_off[L.b];
    const double* row = live ? src + mode_offset(d, st, o.fm, L.r) : src;
    const int Kp = (L.K + kSplitK - 1) / kSplitK * kSplitK;
    if (linear_modes(o.km)) {
      const int kst = st[o.km.x[0]];
#pragma unroll
      for (int i = 0; i < kSliceHoldK / kSliceWarps; ++i) {
        const int k = warp + i * kSliceWarps;
        const bool in = live && k < L.K;
        if (k < Kp) cp_async8(&buf[bi][k][lane], in ? row + k * kst : src, in ? 8 : 0);
      }
    } else {
      for (int k = warp; k < Kp; k += kSliceWarps) {
        const bool in = live && k < L.K;
        cp_async8(&buf[bi][k][lane], in ? row + mode_offset(d, st, o.km, k) : src, in ? 8 : 0);
      }
    }
  };

  SliceLoc none;
  none.opb = -1;
  SliceLoc cur = slice_locate(g, i0, none, lane);
  prefetch(cur, 0);
  cp_async_commit8();
  for (long long item = i0; item < i1; ++item) {
    const int bi = (int)((item - i0) & 1);
    SliceLoc nxt = cur;
    if (item + 1 < i1) {
      nxt = slice_locate(g, item + 1, cur, lane);
      prefetch(nxt, bi ^ 1);  // that buffer was last read by the previous item (barrier below)
    }
    cp_async_commit8();
    cp_async_wait8<1>();  // this thread's copies of the current item have landed
    __syncthreads();      // and every thread's

    const SliceOperand& o = g.op[cur.opb];
    const int* d = o.dims + cur.b * o.order;
    const int R = o.R, K = cur.K, r = cur.r;
    const int Kp = (K + kSplitK - 1) / kSplitK * kSplitK;
    const int ksteps = Kp / kSplitK, nchunks = Kp / 8;
    const bool hold = K <= kSliceHoldK, live = r < cur.m;
    // chunks holding a value: none when the item's rows all lie past the block (padding up to
    // the tile height), and none past K; the others are stored as zero slices
    const int nvalued = r - lane >= cur.m ? 0 : (K + 7) / 8;
    const double scale = o.scale;
    // the direct path's addressing (K > 64)
    int st[kMaxOrder];
    const bool k1 = linear_modes(o.km);  // k at k * kst (no per-element index division)
    int kst = 0;
    const double* row = nullptr;
    if (!hold) {
      block_strides(d, o.order, st);
      kst = k1 ? st[o.km.x[0]] : 0;
      row = o.src + o.src_off[cur.b] + (live ? mode_offset(d, st, o.fm, r) : 0);
    }
    auto load_chunk = [&](int c, double (&v)[8]) {
      if (!hold && k1) {
        // eight loads from always-valid addresses (k clamped, rows past the block read the
        // block's start), issued together; the values outside the block are zeroed after
        double x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = row[min(c * 8 + j, K - 1) * kst];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = live && c * 8 + j < K ? __dmul_rn(x[j], scale) : 0.0;
        return;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = c * 8 + j;
        const bool in = live && k < K;
        if (hold) v[j] = in ? __dmul_rn(buf[bi][k][lane], scale) : 0.0;
        else v[j] = in ? __dmul_rn(row[k1 ? k * kst : mode_offset(d, st, o.km, k)], scale) : 0.0;
      }
    };
    double v[8];
    double mx = 0.0;
    bool finite = true;
    int c0 = warp;
    // two chunks per step: sixteen loads in flight per thread on the direct path
    for (; c0 + kSliceWarps < nvalued; c0 += 2 * kSliceWarps) {
      double v2[8];
      load_chunk(c0, v);
      load_chunk(c0 + kSliceWarps, v2);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        finite = finite && isfinite(v[j]) && isfinite(v2[j]);
        mx = fmax(mx, fmax(fabs(v[j]), fabs(v2[j])));
      }
    }
    if (c0 < nvalued) {
      load_chunk(c0, v);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        finite = finite && isfinite(v[j]);
        mx = fmax(mx, fabs(v[j]));
      }
    }
    if (!finite) atomicExch(&g.flags[kFlagNonFinite], 1);
    wmax[warp][lane] = mx;
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kSliceWarps; ++w) mx = fmax(mx, wmax[w][lane]);
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    const long long eo = o.exp_off[cur.b];
    if (warp == 0) {
      o.expo[eo + r] = (short)e;
      const bool in_range = e >= o.elo && e <= o.ehi;
      if (!in_range) atomicExch(&g.flags[kFlagGeneralExp], 1);
      if (o.pscale) o.pscale[eo + r] = in_range ? ldexp(1.0, e) : 0.0;
    }
    signed char* out = o.out + o.out_off[cur.b] + (long long)(r / R) * ksteps * S * R * kSplitK;
    const long long slab = (long long)R * kSplitK;
    for (int c = warp; c < nchunks; c += kSliceWarps) {
      const long long base = (long long)(c / 4) * S * slab + slab_offset(r % R, (c & 3) * 8);
      if (c < nvalued) {
        if (!hold) load_chunk(c, v);
        slice_chunk<S>(v, e, out, base, slab);
      } else {
#pragma unroll
        for (int t = 0; t < S; ++t) *reinterpret_cast<int2*>(out + base + t * slab) = make_int2(0, 0);
      }
    }
    __syncthreads();  // wmax and this item's buffer are rewritten from the next item on
    cur = nxt;
  }
  cp_async_wait8<0>();
}
using SliceKernel = void (*)(SliceArgs);
static const SliceKernel kSliceKernels[kMaxSlices] = {k_slice<1>, k_slice<2>, k_slice<3>, k_slice<4>,
                                                      k_slice<5>, k_slice<6>, k_slice<7>, k_slice<8>};

// ------------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ unsigned smem_u32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }

// K-major, no swizzle: core matrices of 8 rows x 16 bytes; LBO = 128 (the two 16-byte halves
// of a 32-byte K step), SBO = 256 (next 8 rows).
__device__ __forceinline__ unsigned long long umma_desc(const void* smem) {
  const unsigned long long a = (smem_u32(smem) >> 4) & 0x3FFFu;
  return a | (8ull << 16) | (16ull << 32) | (1ull << 46);
}

// kind::i8, signed A and B, S32 accumulate, K-major operands, M = 128, N = n (16..256, % 16)
__host__ __device__ constexpr unsigned idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(kSplitM >> 4) << 24);
}

__device__ __forceinline__ void umma_i8(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc,
                                        int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(void* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void mbar_init(void* mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tmem_ld16(unsigned taddr, unsigned* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld8(unsigned taddr, unsigned* v);
// kEpiCols consecutive TMEM columns of this warp's 32 lanes into v
__device__ __forceinline__ void tmem_ldc(unsigned taddr, unsigned* v) {
  if constexpr (kEpiCols == 16) tmem_ld16(taddr, v);
  else tmem_ld8(taddr, v);
}
__device__ __forceinline__ void tmem_ld8(unsigned taddr, unsigned* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ------------------------------------------------------------------ mbarrier / bulk copies
__device__ __forceinline__ bool mbar_try(void* mbar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(void* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(void* mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16) completing on mbar
__device__ __forceinline__ void bulk_g2s(void* smem, const void* gmem, unsigned bytes, void* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(smem)),
               "l"(gmem), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// L2 policy that keeps lines resident (evict last): the operand slices, read by many tiles
__device__ __forceinline__ unsigned long long l2_keep_policy() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

// bulk_g2s with an L2 cache policy for the source lines
__device__ __forceinline__ void bulk_g2s_hint(void* smem, const void* gmem, unsigned bytes, void* mbar,
                                              unsigned long long pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(smem)),
      "l"(gmem), "r"(bytes), "r"(smem_u32(mbar)), "l"(pol)
      : "memory");
}

// int64 -> double for |x| < 2^51 with one integer add and one FP64 add: the bits of
// 1.5*2^52 plus x are the double 1.5*2^52 + x (unit spacing in that binade), exact
__device__ __forceinline__ double i2d(long long x) {
  return __longlong_as_double(0x4338000000000000LL + x) - 6755399441055744.0;
}

// int32 -> double exactly: the double with high word 0x43300000 and low word x + 2^31 (as
// unsigned) is 2^52 + x + 2^31; one integer operation and one FP64 add
__device__ __forceinline__ double i32_to_d(int x) {
  return __hiloint2double(0x43300000, x ^ (int)0x80000000) - 4503601774854144.0;
}

// 2^k as a double for -1022 <= k <= 1023 (exact)
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// ------------------------------------------------------------------ records
// The work of one tile (built at plan time): the C block's element offset, where the tile's
// rows and columns start in the offset tables, its first row and column within the block,
// its pair range and its extents.
struct SplitItem {
  long long cbase;
  int rtab, ctab, r0, c0, pb, pe, mt, nt, pad;
};
static_assert(sizeof(SplitItem) == 48, "tile records are bulk-copied in 16-byte units");

// One block pair (built at plan time): where its slices and exponents start, its k-steps.
struct SplitPair {
  long long a_off, b_off, ae_off, be_off;
  int ksteps, pad;
};

// Element offsets, within their C block, of every row and every column of every C block
// (rows of block c at rowtab[rowbase[c] ..], columns at coltab[colbase[c] ..]).  One warp per
// C block.
__global__ void k_split_offsets(const int* __restrict__ dimsC, long long nc, TileMaps mp,
                                const long long* __restrict__ rowbase, const long long* __restrict__ colbase,
                                int* __restrict__ rowtab, int* __restrict__ coltab) {
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (long long c = (long long)blockIdx.x * wpb + (threadIdx.x >> 5); c < nc; c += (long long)gridDim.x * wpb) {
    const int* cd = dimsC + c * mp.oC;
    int st[kMaxOrder];
    block_strides(cd, mp.oC, st);
    int m = 1, n = 1;
    for (int q = 0; q < mp.row.n; ++q) m *= cd[mp.row.y[q]];
    for (int q = 0; q < mp.col.n; ++q) n *= cd[mp.col.y[q]];
    for (int r = lane; r < m; r += 32) {
      int x = r, off = 0;
      for (int q = 0; q < mp.row.n; ++q) {
        const int e = cd[mp.row.y[q]];
        off += (x % e) * st[mp.row.y[q]];
        x /= e;
      }
      rowtab[rowbase[c] + r] = off;
    }
    for (int j = lane; j < n; j += 32) {
      int x = j, off = 0;
      for (int q = 0; q < mp.col.n; ++q) {
        const int e = cd[mp.col.y[q]];
        off += (x % e) * st[mp.col.y[q]];
        x /= e;
      }
      coltab[colbase[c] + j] = off;
    }
  }
}

// per C block: rows and columns rounded up to 4 (16-byte aligned table starts)
__global__ void k_round4(const int* __restrict__ cm, const int* __restrict__ cn, long long nc,
                         long long* __restrict__ rm, long long* __restrict__ rn) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    rm[c] = (cm[c] + 3) & ~3;
    rn[c] = (cn[c] + 3) & ~3;
  }
}

// Work order of a split plan with many C blocks: by the block coordinates of C's row modes (the
// modes A contributes), so that tiles reading the same A row slabs run close together in time
// and find them in L2; blocks without pairs key last (flag bit `rbits`).
__global__ void k_split_order_keys(const long long* __restrict__ ids, long long nc, TensorMeta mC, ModeMap row,
                                   const int* __restrict__ pstart, int rbits, unsigned long long* __restrict__ key) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x) {
    const long long id = ids[c];
    unsigned long long k = 0, mul = 1;
    for (int t = 0; t < row.n; ++t) {
      const int y = row.y[t];
      k += (unsigned long long)((id / mC.gstride[y]) % mC.nblk[y]) * mul;
      mul *= (unsigned long long)mC.nblk[y];
    }
    key[c] = k | (pstart[c + 1] > pstart[c] ? 0ull : 1ull << rbits);
  }
}

__global__ void k_split_items(const int4* __restrict__ work, int nwork, const int* __restrict__ pstart,
                              const long long* __restrict__ offC, const int* __restrict__ dimsC, TileMaps mp,
                              const long long* __restrict__ rowbase, const long long* __restrict__ colbase,
                              SplitItem* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nwork; i += gridDim.x * blockDim.x) {
    const int4 w = work[i];
    const int* cd = dimsC + (long long)w.x * mp.oC;
    int m = 1, n = 1;
    for (int q = 0; q < mp.row.n; ++q) m *= cd[mp.row.y[q]];
    for (int q = 0; q < mp.col.n; ++q) n *= cd[mp.col.y[q]];
    const int ntc = (n + kSplitN - 1) / kSplitN;
    SplitItem t;
    t.cbase = offC[w.x];
    // column tiles of one row tile one after another: they read the same A slabs
    t.r0 = (w.y / ntc) * kSplitM;
    t.c0 = (w.y % ntc) * kSplitN;
    t.rtab = (int)(rowbase[w.x] + t.r0);
    t.ctab = (int)(colbase[w.x] + t.c0);
    t.pb = pstart[w.x];
    t.pe = pstart[w.x + 1];
    t.mt = min(kSplitM, m - t.r0);
    t.nt = min(kSplitN, n - t.c0);
    t.pad = 0;
    out[i] = t;
  }
}

__global__ void k_split_pairs(const int* __restrict__ pair_a, const int* __restrict__ pair_b, long long npairs,
                              const long long* __restrict__ as_off, const long long* __restrict__ bs_off,
                              const long long* __restrict__ ae_off, const long long* __restrict__ be_off,
                              const int* __restrict__ dimsA, TileMaps mp, SplitPair* __restrict__ out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npairs;
       p += (long long)gridDim.x * blockDim.x) {
    const int ia = pair_a[p], ib = pair_b[p];
    const int* ad = dimsA + (long long)ia * mp.oA;
    int K = 1;
    for (int q = 0; q < mp.kk.n; ++q) K *= ad[mp.kk.x[q]];
    SplitPair r;
    r.a_off = as_off[ia];
    r.b_off = bs_off[ib];
    r.ae_off = ae_off[ia];
    r.be_off = be_off[ib];
    r.ksteps = (K + kSplitK - 1) / kSplitK;
    r.pad = 0;
    out[p] = r;
  }
}

// ------------------------------------------------------------------ main kernel
struct SplitArgs {
  double beta;
  int beta_zero, alpha_zero, S;
  const signed char* As; const short* Ae;  // A slices and row exponents
  const signed char* Bs; const short* Be;  // B slices and column exponents
  const double* Bsc;                       // B column scales 2^f (0 outside the normal range)
  double* C;
  const int* rowtab; const int* coltab;  // element offsets of C rows / columns
  const SplitItem* items;  // per work item (tile)
  const SplitPair* prs;    // per block pair
  int nwork;
  const int* flags;        // the execute's flag words (kFlag*)
  // several requests in one launch (serving): their arguments, and the first global item of
  // each (ascending); nwork is then the total.  0 for a launch of this plan alone.
  const SplitArgs* multi;
  const int* mfirst;
  int nmulti;
  volatile int* err;       // the context's error word (host-mapped): SHT_ERR_TIMEOUT
  long long wait_limit;    // polls of one pipeline wait before the launch gives up
  long long drain_limit;   // polls of the waits for work already issued (copies, MMAs)
};

// Per tile, the slot warp loads the tile's record and its row / column offsets into a ring of
// tile slots, and per pair the A row exponents, the B column exponents and the B column
// scales into a ring of exponent slots, so the epilogue reads nothing from global memory but
// the C values it scales by beta.
// One record of the producer's, the MMA issuer's and the slot warp's work stream: one pair of one tile (or a
// tile without pairs), its copy sources resolved by the record warp.
struct SplitRec {
  const signed char* a_src;  // A slabs of the pair's k-steps for the tile's rows
  const signed char* b_src;  // B slabs for the tile's columns
  const short* ae_src;
  const short* be_src;
  const double* bsc_src;
  const SplitItem* rec_src;  // the tile record, its row and column offsets (first record of a tile)
  const int* rowtab_src;
  const int* coltab_src;
  int ksteps;                // 0: a tile without pairs
  int kind;                  // kRecFirst: first record of its tile; kRecEnd: end of the stream
};
constexpr int kRecFirst = 1, kRecEnd = 4;

struct SplitTileSlot {
  SplitItem rec;
  int rowoff[kSplitM];
  int coloff[kSplitN];
};
struct SplitExpSlot {
  short ea[kSplitM];
  short eb[kSplitN];
  double sc[kSplitN];
};
constexpr unsigned kTileSlotBytes = sizeof(SplitTileSlot);
constexpr unsigned kExpSlotBytes = sizeof(SplitExpSlot);
static_assert(sizeof(SplitItem) % 16 == 0 && kTileSlotBytes == 48 + 4 * (kSplitM + kSplitN) &&
                  kExpSlotBytes == 2 * (kSplitM + kSplitN) + 8 * kSplitN && offsetof(SplitExpSlot, sc) % 16 == 0,
              "slot members are filled by 16-byte stores at 16-byte offsets");

template <int S>
struct SplitSmem {
  static constexpr int kStages = split_stages(S);
  alignas(1024) signed char stage[kStages][S * (kAChunk + kBChunk)];
  alignas(16) SplitTileSlot tile[kTileSlots];
  alignas(16) SplitExpSlot ex[kExpSlots];
  alignas(8) unsigned long long full[kStages], empty[kStages], tfull[2], tempty[2], drain;
  unsigned long long ifull[kTileSlots], iempty[kTileSlots], efull[kExpSlots], eempty[kExpSlots];
  unsigned long long rfull[kRecSlots], rempty[kRecSlots];
  SplitRec rec[kRecSlots];
  unsigned tmem_base;
  int abort;
};

// The fields of one request that the roles use, copied into registers once per item: in a
// launch of one plan they come from the kernel parameters; in a launch of several requests
// from the request's entry of the device array (read once, not after every memory-clobbering
// mbarrier or bulk-copy instruction).
struct SplitReq {
  const signed char* As; const short* Ae;
  const signed char* Bs; const short* Be; const double* Bsc;
  double* C;
  const int* rowtab; const int* coltab;
  const SplitItem* items; const SplitPair* prs;
  double beta;
  int beta_zero, alpha_zero, flags_nonfinite, flags_general;
};

__device__ __forceinline__ SplitReq req_fields(const SplitArgs& a, bool read_flags) {
  SplitReq r;
  r.As = a.As; r.Ae = a.Ae; r.Bs = a.Bs; r.Be = a.Be; r.Bsc = a.Bsc; r.C = a.C;
  r.rowtab = a.rowtab; r.coltab = a.coltab; r.items = a.items; r.prs = a.prs;
  r.beta = a.beta; r.beta_zero = a.beta_zero; r.alpha_zero = a.alpha_zero;
  r.flags_nonfinite = read_flags ? a.flags[kFlagNonFinite] : 0;
  r.flags_general = read_flags ? a.flags[kFlagGeneralExp] : 0;
  return r;
}

// The request that global item `item` belongs to (Multi: binary search over the requests'
// first items) and its item index there.
template <bool Multi>
__device__ __forceinline__ SplitReq split_req(const SplitArgs& g, int item, int& li) {
  if constexpr (!Multi) {
    li = item;
    return req_fields(g, false);
  } else {
    int lo = 0, hi = g.nmulti;  // the last request whose first item is <= item
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (g.mfirst[mid] <= item) lo = mid; else hi = mid;
    }
    li = item - g.mfirst[lo];
    return req_fields(g.multi[lo], true);
  }
}

// bounded wait that also gives up when another role raised the abort flag
__device__ __forceinline__ bool split_wait(void* mbar, unsigned parity, volatile int* abort, const SplitArgs& g) {
  for (long long i = 0; i < g.wait_limit; ++i) {
    if (mbar_try(mbar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  *g.err = (int)SHT_ERR_TIMEOUT;  // every writer stores the same value
  __threadfence_system();
  return false;
}

// bounded wait for work this CTA issued already (bulk copies, MMAs): it always completes, so
// the bound is generous and no abort flag applies
__device__ __forceinline__ void split_settle(void* mbar, unsigned parity, const SplitArgs& g) {
  for (long long i = 0; i < g.drain_limit; ++i)
    if (mbar_try(mbar, parity)) return;
}

// Reassembly weights.  Groups are numbered gi = 0..S-1 (group g = gi + 2 of the triangle); the
// value of one element of one pair is 2^(e_r + f_c) * sum_gi 2^(-7(gi + 2)) P_gi.
// Narrow launches (every |P_gi| < 2^23) combine the groups two by two in 32 bits,
// X_k = P_2k * 128 + P_2k+1, with weight 2^(-14k - 21); for odd S >= 3 the last group is
// folded into the last pair rounded to its weight, X += (P_S-1 + 64) >> 7, an error of at most
// 2^(-7S - 1) of the row / column scales, below the slicing's own truncation (2^(-7S) per term
// of the contracted sum); S = 1 keeps X_0 = P_0 with weight 2^-14.
__host__ __device__ constexpr int narrow_nx(int S) { return S == 1 ? 1 : S / 2; }
__host__ __device__ constexpr int narrow_wexp(int S, int k) { return S == 1 ? -14 : -14 * k - 21; }

// Loads groups [g0, g1) of this thread's 8 columns from TMEM and folds them into the narrow
// sums X (groups 2k and 2k+1 into X_k; the odd last group rounded into X_(nx-1)).
template <int S, int g0, int g1>
__device__ __forceinline__ void narrow_load(unsigned tb, int (&X)[narrow_nx(S)][kEpiCols]) {
  unsigned v[g1 - g0][kEpiCols];
#pragma unroll
  for (int i = 0; i < g1 - g0; ++i) tmem_ldc(tb + (unsigned)((g0 + i) * kSplitN), v[i]);
  tmem_wait_ld();
#pragma unroll
  for (int gi = g0; gi < g1; ++gi) {
#pragma unroll
    for (int j = 0; j < kEpiCols; ++j) {
      const int p = (int)v[gi - g0][j];
      if (S == 1) {
        X[0][j] = p;
      } else if ((S & 1) && gi == S - 1) {
        X[narrow_nx(S) - 1][j] += (p + 64) >> 7;  // the odd last group, rounded
      } else if ((gi & 1) == 0) {
        X[gi >> 1][j] = p * 128;
      } else {
        X[gi >> 1][j] += p;
      }
    }
  }
}

// S (slices per operand) is a template parameter so that the group loops of the MMA issuer
// and of the reassembly unroll completely; one instance per S = 1..8.  Narrow: every group sum
// is below 2^23 in magnitude (the host checks S * 127^2 * K), so groups combine two by two in
// 32 bits and each pair converts with one integer operation and one FP64 add.
template <int S, bool Narrow, bool Multi>
__global__ void __launch_bounds__(kSplitThreads, 1) k_split(const __grid_constant__ SplitArgs g) {
  // an operand holds a non-finite value: the FP64 tile kernel computes this execute (in a
  // launch of several requests every role skips such a request's tiles alike)
  if (!Multi && g.flags[kFlagNonFinite]) return;
  // one plan: some row or column exponent lies outside the scale-folded range (uniform)
  const bool general1 = !Multi && g.flags[kFlagGeneralExp] != 0;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  using Smem = SplitSmem<S>;
  constexpr int kSplitStages = Smem::kStages;
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int* abort = &sm.abort;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem_base)),
                 "r"(kSplitTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    for (int i = 0; i < kSplitStages; ++i) {
      mbar_init(&sm.full[i], 1);
      mbar_init(&sm.empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&sm.tfull[i], 1);
      mbar_init(&sm.tempty[i], kEpiWarps);
    }
    for (int i = 0; i < kTileSlots; ++i) {
      mbar_init(&sm.ifull[i], 32);  // every lane of the slot warp, after its own stores
      mbar_init(&sm.iempty[i], kEpiWarps);
    }
    for (int i = 0; i < kExpSlots; ++i) {
      mbar_init(&sm.efull[i], 32);
      mbar_init(&sm.eempty[i], kEpiWarps);
    }
    for (int i = 0; i < kRecSlots; ++i) {
      mbar_init(&sm.rfull[i], 1);
      mbar_init(&sm.rempty[i], 3);  // the producer, the MMA issuer and the slot warp
    }
    mbar_init(&sm.drain, 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = sm.tmem_base;
  const unsigned a_bytes = (unsigned)(S * kAChunk), b_bytes = (unsigned)(S * kBChunk);

  if (warp == 0) {
    // ---------------------------------------------------------------- producer
    if (lane == 0) {
      long long n = 0;
      int st = 0;         // stage of k-step n (n % kSplitStages) and its ring phase
      unsigned sph = 0;
      bool ok = true;
      // the slices are read by every tile of their rows / columns: keep them in L2 against the
      // stream of C stores (which the epilogue marks evict-first)
      const unsigned long long keep = l2_keep_policy();
      for (long long r = 0; ok; ++r) {
        const int rs = (int)(r & (kRecSlots - 1));
        if (!split_wait(&sm.rfull[rs], (unsigned)((r / kRecSlots) & 1), abort, g)) { ok = false; break; }
        const SplitRec v = sm.rec[rs];
        mbar_arrive(&sm.rempty[rs]);
        if (v.kind & kRecEnd) break;
        if (v.ksteps == 0) continue;
        const signed char* asrc = v.a_src;
        const signed char* bsrc = v.b_src;
        for (int ks = 0; ks < v.ksteps; ++ks, ++n) {
          if (!split_wait(&sm.empty[st], sph ^ 1u, abort, g)) { ok = false; break; }
          mbar_expect_tx(&sm.full[st], a_bytes + b_bytes);
          bulk_g2s_hint(sm.stage[st], asrc, a_bytes, &sm.full[st], keep);
          bulk_g2s_hint(sm.stage[st] + a_bytes, bsrc, b_bytes, &sm.full[st], keep);
          asrc += a_bytes;
          bsrc += b_bytes;
          if (++st == kSplitStages) {
            st = 0;
            sph ^= 1u;
          }
        }
      }
      if (!ok) {
        // copies still in flight write into this CTA's shared memory: wait for them (bounded)
        auto settle = [&](unsigned long long* bars, int nbars, long long issued) {
          for (long long j = issued > nbars ? issued - nbars : 0; j < issued; ++j)
            split_settle(&bars[j % nbars], (unsigned)((j / nbars) & 1), g);
        };
        settle(sm.full, kSplitStages, n);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      long long n = 0, q = 0;
      int st = 0;  // stage of k-step n and its ring phase, as the producer's
      unsigned sph = 0;
      bool ok = true;
      for (long long r = 0; ok; ++r) {
        const int rs = (int)(r & (kRecSlots - 1));
        if (!split_wait(&sm.rfull[rs], (unsigned)((r / kRecSlots) & 1), abort, g)) { ok = false; break; }
        const int ksteps = sm.rec[rs].ksteps, kind = sm.rec[rs].kind;
        mbar_arrive(&sm.rempty[rs]);
        if (kind & kRecEnd) break;
        if (ksteps == 0) continue;
        const int buf = (int)(q & 1);
        if (!split_wait(&sm.tempty[buf], (unsigned)(((q >> 1) & 1) ^ 1), abort, g)) { ok = false; break; }
        ++q;
        tc_fence_after();
        const unsigned dbase = tmem + (unsigned)(buf * kBufCols);
        for (int ks = 0; ks < ksteps; ++ks, ++n) {
          if (!split_wait(&sm.full[st], sph, abort, g)) { ok = false; break; }
          tc_fence_after();
          const signed char* a = sm.stage[st];
          const signed char* b = sm.stage[st] + a_bytes;
          // A slice t times B slices 1..S+1-t in one MMA: the products land in TMEM groups
          // g = t+1 .. S+1, i.e. columns from (t-1)*32 on; t = 1 writes every group first.
#pragma unroll
          for (int t = 1; t <= S; ++t) {
            const int nn = kSplitN * (S + 1 - t);
            umma_i8(dbase + (unsigned)((t - 1) * kSplitN), umma_desc(a + (t - 1) * kAChunk), umma_desc(b),
                    idesc_i8(nn), (t == 1 && ks == 0) ? 0 : 1);
          }
          umma_commit(&sm.empty[st]);  // the stage is free once these MMAs have read it
          if (++st == kSplitStages) {
            st = 0;
            sph ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(&sm.tfull[buf]);  // the pair's groups are complete
      }
      // drain: every MMA issued above has finished before TMEM is released (bounded)
      umma_commit(&sm.drain);
      split_settle(&sm.drain, 0, g);
    }
    __syncwarp();
  } else if (warp == kRecWarp) {
    // ---------------------------------------------------------------- record warp
    // Walks the CTA's tiles 32 at a time, one tile per lane: the lanes load their tile records
    // and first pair records in parallel, then write their records into the ring in stream order
    // (lane after lane), resolving every copy source, so that the producer and the MMA issuer
    // read their work from shared memory.  Ends the stream with a kRecEnd record.
    long long r = 0;  // records written
    bool ok = true;
    for (int base = blockIdx.x; ok && base < g.nwork; base += 32 * gridDim.x) {
      const int item = base + lane * gridDim.x;
      int li = 0;
      SplitItem t{};
      SplitReq a{};
      int np = 0, cnt = 0;
      if (item < g.nwork) {
        a = split_req<Multi>(g, item, li);
        if (!a.flags_nonfinite) {
          t = a.items[li];
          np = a.alpha_zero ? 0 : t.pe - t.pb;
          cnt = np > 0 ? np : 1;
        }
      }
      SplitPair pr{};
      if (np > 0) pr = a.prs[t.pb];
      for (int l = 0; ok && l < 32; ++l) {
        const int c = __shfl_sync(0xffffffffu, cnt, l);
        if (lane == l) {
          for (int j = 0; ok && j < c; ++j, ++r) {
            if (j > 0) pr = a.prs[t.pb + j];
            const int rs = (int)(r & (kRecSlots - 1));
            if (!split_wait(&sm.rempty[rs], (unsigned)(((r / kRecSlots) & 1) ^ 1), abort, g)) { ok = false; break; }
            SplitRec v;
            v.kind = j == 0 ? kRecFirst : 0;
            v.rec_src = a.items + li;
            v.rowtab_src = a.rowtab + t.rtab;
            v.coltab_src = a.coltab + t.ctab;
            if (np > 0) {
              v.ksteps = pr.ksteps;
              v.a_src = a.As + pr.a_off + (long long)(t.r0 / kSplitM) * pr.ksteps * a_bytes;
              v.b_src = a.Bs + pr.b_off + (long long)(t.c0 / kSplitN) * pr.ksteps * b_bytes;
              v.ae_src = a.Ae + pr.ae_off + t.r0;
              v.be_src = a.Be + pr.be_off + t.c0;
              v.bsc_src = a.Bsc + pr.be_off + t.c0;
            } else {
              v.ksteps = 0;
              v.a_src = v.b_src = nullptr;
              v.ae_src = v.be_src = nullptr;
              v.bsc_src = nullptr;
            }
            sm.rec[rs] = v;
            mbar_arrive(&sm.rfull[rs]);  // release: the record's stores come first
          }
        }
        r = __shfl_sync(0xffffffffu, r, l);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, l) != 0;
      }
    }
    if (ok && lane == 0) {
      const int rs = (int)(r & (kRecSlots - 1));
      if (split_wait(&sm.rempty[rs], (unsigned)(((r / kRecSlots) & 1) ^ 1), abort, g)) {
        sm.rec[rs].kind = kRecEnd;
        sm.rec[rs].ksteps = 0;
        mbar_arrive(&sm.rfull[rs]);
      }
    }
    __syncwarp();
  } else if (warp == kSlotWarp) {
    // ---------------------------------------------------------------- slot warp
    // Follows the record stream: per tile record it fills a tile slot (the tile's record and
    // its row / column offsets), per pair an exponent slot (row exponents, column exponents,
    // column scales), 16 bytes per lane.  Two records are in hand at a time: the loads of the
    // next record are issued before the current one waits for its slots and is stored, so
    // their latency overlaps.  Every lane arrives on a slot's barrier after its own stores.
    struct SlotLoad {
      int4 t4, ro, co, x0, x1;
      bool first, pair;
    };
    auto issue = [&](const SplitRec& v) {
      SlotLoad d;
      d.first = (v.kind & kRecFirst) != 0;
      d.pair = v.ksteps > 0;
      d.t4 = d.ro = d.co = d.x0 = d.x1 = make_int4(0, 0, 0, 0);
      if (d.first) {
        if (lane < 3) d.t4 = reinterpret_cast<const int4*>(v.rec_src)[lane];    // 48-byte record
        d.ro = reinterpret_cast<const int4*>(v.rowtab_src)[lane];                // 128 row offsets
        if (lane < 8) d.co = reinterpret_cast<const int4*>(v.coltab_src)[lane];  // 32 column offsets
      }
      if (d.pair) {
        if (lane < 16) d.x0 = reinterpret_cast<const int4*>(v.ae_src)[lane];           // 128 row exponents
        else if (lane < 20) d.x0 = reinterpret_cast<const int4*>(v.be_src)[lane - 16];  // 32 column exponents
        if (lane < 16) d.x1 = reinterpret_cast<const int4*>(v.bsc_src)[lane];          // 32 column scales
      }
      return d;
    };
    long long q = 0, ni = 0;
    auto commit = [&](const SlotLoad& d) {
      if (d.first) {
        const int is = (int)(ni % kTileSlots);
        if (!__all_sync(0xffffffffu, split_wait(&sm.iempty[is], (unsigned)(((ni / kTileSlots) & 1) ^ 1), abort, g)))
          return false;
        ++ni;
        SplitTileSlot& ts = sm.tile[is];
        if (lane < 3) reinterpret_cast<int4*>(&ts.rec)[lane] = d.t4;
        reinterpret_cast<int4*>(ts.rowoff)[lane] = d.ro;
        if (lane < 8) reinterpret_cast<int4*>(ts.coloff)[lane] = d.co;
        mbar_arrive(&sm.ifull[is]);  // release: this lane's stores come first
      }
      if (d.pair) {
        const int es = (int)(q % kExpSlots);
        if (!__all_sync(0xffffffffu, split_wait(&sm.eempty[es], (unsigned)(((q / kExpSlots) & 1) ^ 1), abort, g)))
          return false;
        ++q;
        SplitExpSlot& ex = sm.ex[es];
        if (lane < 16) reinterpret_cast<int4*>(ex.ea)[lane] = d.x0;
        else if (lane < 20) reinterpret_cast<int4*>(ex.eb)[lane - 16] = d.x0;
        if (lane < 16) reinterpret_cast<int4*>(ex.sc)[lane] = d.x1;
        mbar_arrive(&sm.efull[es]);
      }
      return true;
    };
    SlotLoad cur{};
    bool have = false, ok = true;
    for (long long r = 0; ok; ++r) {
      const int rs = (int)(r & (kRecSlots - 1));
      if (!__all_sync(0xffffffffu, split_wait(&sm.rfull[rs], (unsigned)((r / kRecSlots) & 1), abort, g))) {
        ok = false;
        break;
      }
      const SplitRec v = sm.rec[rs];
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.rempty[rs]);
      if (v.kind & kRecEnd) break;
      const SlotLoad nxt = issue(v);
      if (have) ok = commit(cur);
      cur = nxt;
      have = true;
    }
    if (ok && have) commit(cur);
  } else if (warp < 2 + kEpiWarps) {
    // ---------------------------------------------------------------- epilogue
    const int quarter = warp & 3, cq = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;  // the TMEM lane this warp may read
    const unsigned tlane = (unsigned)(quarter * 32) << 16;
    long long q = 0, ni = 0;
    bool ok = true;
    for (int item = blockIdx.x; ok && item < g.nwork; item += gridDim.x) {
      int li;
      const SplitReq a = split_req<Multi>(g, item, li);
      if (a.flags_nonfinite) continue;
      // some row or column exponent of this request lies outside the scale-folded range
      const bool general = Multi ? a.flags_general != 0 : general1;
      const int is = (int)(ni % kTileSlots);
      if (!split_wait(&sm.ifull[is], (unsigned)((ni / kTileSlots) & 1), abort, g)) { ok = false; break; }
      ++ni;
      const SplitTileSlot& ts = sm.tile[is];
      const SplitItem t = ts.rec;
      const bool row_in = row < t.mt;
      // a warp whose rows or columns all lie outside a partial tile skips the reassembly
      const bool warp_live = quarter * 32 < t.mt && cq * kEpiCols < t.nt;
      const int roff = ts.rowoff[row];
      int coff[kEpiCols];
#pragma unroll
      for (int j = 0; j < kEpiCols; ++j) coff[j] = ts.coloff[cq * kEpiCols + j];
      // the slot warp refills the slot with ordinary stores after it sees this release
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.iempty[is]);
      double* cptr = a.C + t.cbase;
      double acc[kEpiCols];
#pragma unroll
      for (int j = 0; j < kEpiCols; ++j) {
        const bool in = row_in && cq * kEpiCols + j < t.nt;
        acc[j] = (a.beta_zero || !in) ? 0.0 : __dmul_rn(a.beta, __ldcs(cptr + roff + coff[j]));
      }
      const int pe = a.alpha_zero ? t.pb : t.pe;
      for (int p = t.pb; p < pe; ++p, ++q) {
        const int buf = (int)(q & 1);
        const int es = (int)(q % kExpSlots);
        // warp-uniform: the TMEM loads below are .sync.aligned
        if (!__all_sync(0xffffffffu, split_wait(&sm.efull[es], (unsigned)((q / kExpSlots) & 1), abort, g) &&
                                         split_wait(&sm.tfull[buf], (unsigned)((q >> 1) & 1), abort, g))) {
          ok = false;
          break;
        }
        // the slot's exponents and column scales are read where they are used; the slot is
        // released after the pair's arithmetic (the ring is four deep)
        const SplitExpSlot& ex = sm.ex[es];
        const double* sc = &ex.sc[cq * kEpiCols];
        const short* fe = &ex.eb[cq * kEpiCols];
        const int er = ex.ea[row];
        auto release_exp = [&]() {
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.eempty[es]);
        };
        tc_fence_after();
        const unsigned tb = tmem + tlane + (unsigned)(buf * kBufCols + cq * kEpiCols);
        auto release_set = [&]() {
          // the groups are in registers: the accumulator set may be overwritten
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.tempty[buf]);
        };
        if (!warp_live) {
          release_set();
          release_exp();
          continue;
        }
        if constexpr (Narrow) {
          // ---- narrow: NX 32-bit sums, one conversion each
          constexpr int NX = narrow_nx(S);
          int X[NX][kEpiCols];
          narrow_load<S, 0, (S < 4 ? S : 4)>(tb, X);
          if constexpr (S > 4) narrow_load<S, 4, S>(tb, X);
          release_set();
          constexpr double kM = 4503601774854144.0;  // 2^52 + 2^31: the conversion's offset
          if (!general) {
            // the row scale folded into the weights: W_k = 2^(e_r - 14k - 21) (exact, normal)
            double W[NX];
#pragma unroll
            for (int k = 0; k < NX; ++k) W[k] = pow2(er + narrow_wexp(S, k));
            const double mlast = -kM * W[NX - 1];
#pragma unroll
            for (int j = 0; j < kEpiCols; ++j) {
              // smallest weight first; the first product is exact: (2^52 + 2^31 + X) W - (2^52 + 2^31) W
              double part = fma(__hiloint2double(0x43300000, X[NX - 1][j] ^ (int)0x80000000), W[NX - 1], mlast);
#pragma unroll
              for (int k = NX - 2; k >= 0; --k)
                part = fma(__hiloint2double(0x43300000, X[k][j] ^ (int)0x80000000) - kM, W[k], part);
              acc[j] = fma(part, sc[j], acc[j]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < kEpiCols; ++j) {
              double part = 0.0;
#pragma unroll
              for (int k = NX - 1; k >= 0; --k)
                part = fma(__hiloint2double(0x43300000, X[k][j] ^ (int)0x80000000) - kM, pow2(narrow_wexp(S, k)),
                           part);
              const int e = er + fe[j];
              acc[j] = (e >= -1022 && e <= 1023) ? fma(part, pow2(e), acc[j]) : acc[j] + scalbn(part, e);
            }
          }
        } else {
          // ---- wide: the INT32 groups are combined exactly in int64 three at a time
          // (P_g 2^14 + P_g+1 2^7 + P_g+2 < 2^46), each triple converted once and weighted by
          // an exact power of two (smallest weights first)
          double part[kEpiCols];
#pragma unroll
          for (int j = 0; j < kEpiCols; ++j) part[j] = 0.0;
#pragma unroll
          for (int c = (kMaxSlices - 1) / 3; c >= 0; --c) {
            const int g0 = 3 * c;
            if (g0 >= S) continue;
            const int len = min(3, S - g0);
            unsigned v[3][kEpiCols];
#pragma unroll
            for (int i = 0; i < 3; ++i)
              if (i < len) tmem_ldc(tb + (unsigned)((g0 + i) * kSplitN), v[i]);
            tmem_wait_ld();
            if (c == 0) release_set();
            // the triple's lowest group has weight 2^(-7(g0 + len - 1)) relative to group 2
            const double w = pow2(-7 * (g0 + len - 1));
#pragma unroll
            for (int j = 0; j < kEpiCols; ++j) {
              long long x = (int)v[0][j];
              if (len > 1) x = x * 128 + (int)v[1][j];
              if (len > 2) x = x * 128 + (int)v[2][j];
              part[j] = fma(i2d(x), w, part[j]);
            }
          }
          if (!general) {
            // part * 2^(e_r - 14) is exact (normal) and sc[j] = 2^(f_c): one rounding
            const double sr = pow2(er - 14);
#pragma unroll
            for (int j = 0; j < kEpiCols; ++j) acc[j] = fma(part[j] * sr, sc[j], acc[j]);
          } else {
#pragma unroll
            for (int j = 0; j < kEpiCols; ++j) {
              const int e = er + fe[j] - 14;
              acc[j] = (e >= -1022 && e <= 1023) ? fma(part[j], pow2(e), acc[j]) : acc[j] + scalbn(part[j], e);
            }
          }
        }
        release_exp();
      }
      if (!ok) break;
      if (row_in) {
#pragma unroll
        for (int j = 0; j < kEpiCols; ++j)
          if (cq * kEpiCols + j < t.nt) __stcs(cptr + roff + coff[j], acc[j]);  // streaming: keeps the slices in L2
      }
    }
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

// Per block: byte offset of its slices (tiles of R rows) and offset of its exponents (rows
// padded to a multiple of R), plus the slicer's items of 32 rows.  Groups hold exact INT32
// sums of up to S products of |s| <= 127 per k, so K is limited to keep them below 2^31.
template <int R>
static void slice_layout(sht_tensor* T, const std::vector<int>& free_modes, const std::vector<int>& k_modes, int S,
                         long long* off, long long* eoff, long long* istart, long long& total, long long& etotal,
                         long long& nitems) {
  const long long n = T->nblocks;
  const int* dims = tensor_host_dims(T);
  total = etotal = nitems = 0;
  for (long long b = 0; b < n; ++b) {
    const int* d = dims + b * T->order;
    long long m = 1, K = 1;
    for (int ax : free_modes) m *= d[ax];
    for (int ax : k_modes) K *= d[ax];
    if (K > 16384) fail(SHT_ERR_UNSUPPORTED, "split mode: contracted block extent above 16384");
    const long long Kp = (K + kSplitK - 1) / kSplitK * kSplitK;
    const long long mp = (m + R - 1) / R * R;
    if ((long long)S * mp * Kp >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "block slices above 2^31 bytes");
    off[b] = total;
    eoff[b] = etotal;
    istart[b] = nitems;
    total += (long long)S * mp * Kp;  // a multiple of 1 KB: every block stays aligned for bulk copies
    etotal += mp;
    nitems += mp / 32;  // the slicer's items: 32 rows each
  }
}

int split_slices_default() { return 7; }

void split_prepare(sht_plan* p, int S, cudaStream_t s) {
  split_layout(p, S, s);
  split_records(p, s);
}

void split_layout(sht_plan* p, int S, cudaStream_t s) {
  if (S < 1 || S > kMaxSlices) fail(SHT_ERR_INVALID, "split slices must be 1..8");
  DevicePool* pool = p->ctx->pool.get();
  p->split_slices = S;
  const long long nA = p->A->nblocks, nB = p->B->nblocks;
  // host image of sp_meta, 8-byte words: per A block its slice offset, exponent offset and
  // first slicer item, the same per B block, then the error words (32 x 8 bytes, zero)
  std::vector<long long> meta((size_t)(3 * nA + 3 * nB + 32));
  long long at, aet, bt, bet, nia, nib;
  slice_layout<kSplitM>(p->A, p->maps.rowA, p->maps.colA, S, meta.data(), meta.data() + nA, meta.data() + 2 * nA, at,
                        aet, nia);
  long long* mb = meta.data() + 3 * nA;
  slice_layout<kSplitN>(p->B, p->maps.colB, p->maps.rowB, S, mb, mb + nB, mb + 2 * nB, bt, bet, nib);
  trace("split: slice layout (host)", s);
  p->sp_a = PoolBuf(pool, std::max(at, 16LL), s);
  p->sp_b = PoolBuf(pool, std::max(bt, 16LL), s);
  p->sp_ae = PoolBuf(pool, std::max(aet, 1LL) * 2, s);
  p->sp_be = PoolBuf(pool, std::max(bet, 1LL) * 2, s);
  p->sp_bsc = PoolBuf(pool, std::max(bet, 1LL) * 8, s);
  p->sp_meta = PoolBuf(pool, meta.size() * 8, s);
  long long* dm = p->sp_meta.as<long long>();
  p->sp_aoff = dm;
  p->sp_aeoff = dm + nA;
  p->sp_aistart = dm + 2 * nA;
  p->sp_boff = dm + 3 * nA;
  p->sp_beoff = dm + 3 * nA + nB;
  p->sp_bistart = dm + 3 * nA + 2 * nB;
  p->sp_err = reinterpret_cast<int*>(dm + 3 * nA + 3 * nB);
  p->sp_naitems = nia;
  p->sp_nbitems = nib;
  trace("split: slice buffers", s);
  // one copy (from pageable memory it has consumed its source when it returns)
  SHT_CUDA(cudaMemcpyAsync(dm, meta.data(), meta.size() * 8, cudaMemcpyHostToDevice, s));
  trace("split: slice layout", s);
}

void split_records(sht_plan* p, cudaStream_t s) {
  DevicePool* pool = p->ctx->pool.get();
  // row / column offset tables of the C blocks: starts from a scan of the blocks' row and
  // column counts (rounded up to 4 so that every tile's slice of a table is 16-byte aligned);
  // the totals come back with the work list's counts
  const sht_tensor* C = p->C;
  const long long nc = C->nblocks;
  PoolBuf drb(pool, std::max(nc, 1LL) * 8, s), dcb(pool, std::max(nc, 1LL) * 8, s);
  PoolBuf rm(pool, std::max(nc, 1LL) * 8, s), rn(pool, std::max(nc, 1LL) * 8, s);
  long long rtot = 0, ctot = 0;
  if (nc > 0) {
    k_round4<<<grid_for(nc, 256), 256, 0, s>>>(p->d_cm.as<int>(), p->d_cn.as<int>(), nc, rm.as<long long>(),
                                               rn.as<long long>());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, rm.as<long long>(), drb.as<long long>(), (int)nc, s);
    PoolBuf tmp(pool, tb, s);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, rm.as<long long>(), drb.as<long long>(), (int)nc, s);
    cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, rn.as<long long>(), dcb.as<long long>(), (int)nc, s);
  }
  // work list: 128 x 32 tiles of every C block, heaviest blocks first, with per-tile and
  // per-pair records so that the kernel reads each with one load
  const DevSum extra[2] = {{drb.as<long long>() + nc - 1, rm.as<long long>() + nc - 1},
                           {dcb.as<long long>() + nc - 1, rn.as<long long>() + nc - 1}};
  long long h[2] = {0, 0};
  // Many C blocks: order them by A row block (L2 reuse of the A slabs); the tiles are many per
  // CTA, so the static striding stays balanced.  Few C blocks: heaviest first, for balance.
  PoolBuf okey;
  int obits = 0;
  if (nc >= 16LL * p->ctx->num_sms) {
    unsigned long long span = 1;
    for (int t = 0; t < p->tmaps.row.n; ++t) span *= (unsigned long long)C->nblk[p->tmaps.row.y[t]];
    int rbits = 0;
    while (rbits < 62 && (1ull << rbits) < span) ++rbits;
    obits = rbits + 1;
    okey = PoolBuf(pool, nc * 8, s);
    k_split_order_keys<<<grid_for(nc, 256), 256, 0, s>>>(C->d_ids.as<long long>(), nc, make_meta(C), p->tmaps.row,
                                                         p->d_pstart.as<int>(), rbits, okey.as<unsigned long long>());
    SHT_CUDA(cudaGetLastError());
  }
  device_work_list(p, kSplitM, kSplitN, false, s, extra, h, nc > 0 ? 2 : 0, okey.as<unsigned long long>(), obits);
  rtot = h[0];
  ctot = h[1];
  trace("split: work list", s);
  if (rtot >= (1LL << 31) || ctot >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "split mode: C row / column tables above 2^31");
  // a tile reads a full 128 rows / 32 columns: slack past the last block
  p->sp_rowtab = PoolBuf(pool, (rtot + kSplitM) * 4, s);
  p->sp_coltab = PoolBuf(pool, (ctot + kSplitN) * 4, s);
  SHT_CUDA(cudaMemsetAsync(p->sp_rowtab.ptr, 0, (rtot + kSplitM) * 4, s));
  SHT_CUDA(cudaMemsetAsync(p->sp_coltab.ptr, 0, (ctot + kSplitN) * 4, s));
  if (nc > 0)
    k_split_offsets<<<(int)std::min<long long>((nc + 7) / 8, (long long)p->ctx->num_sms * 8), 256, 0, s>>>(
        C->d_dims.as<int>(), nc, p->tmaps, drb.as<long long>(), dcb.as<long long>(), p->sp_rowtab.as<int>(),
        p->sp_coltab.as<int>());
  trace("split: C offset tables", s);
  p->sp_items = PoolBuf(pool, std::max(p->bwork, 1LL) * sizeof(SplitItem), s);
  p->sp_pairs = PoolBuf(pool, std::max(p->npairs, 1LL) * sizeof(SplitPair), s);
  if (p->bwork > 0)
    k_split_items<<<grid_for(p->bwork, 256), 256, 0, s>>>(p->d_bwork.as<int4>(), (int)p->bwork, p->d_pstart.as<int>(),
                                                          p->C->d_offsets.as<long long>(), p->C->d_dims.as<int>(),
                                                          p->tmaps, drb.as<long long>(), dcb.as<long long>(),
                                                          p->sp_items.as<SplitItem>());
  if (p->npairs > 0)
    k_split_pairs<<<grid_for(p->npairs, 256), 256, 0, s>>>(
        p->d_pair_a.as<int>(), p->d_pair_b.as<int>(), p->npairs, p->sp_aoff,
        p->sp_boff, p->sp_aeoff, p->sp_beoff,
        p->A->d_dims.as<int>(), p->tmaps, p->sp_pairs.as<SplitPair>());
  SHT_CUDA(cudaGetLastError());
  trace("split: tile / pair records", s);
}

// One CTA per SM: it holds all 512 TMEM columns, and its shared memory (at least 116 KB, more
// than half an SM's) keeps a second CTA off.
template <int S>
constexpr size_t split_smem_bytes() {
  return sizeof(SplitSmem<S>) > 116 * 1024 ? sizeof(SplitSmem<S>) : 116 * 1024;
}
static_assert(sizeof(SplitSmem<1>) <= kSplitSmemBudget && sizeof(SplitSmem<7>) <= kSplitSmemBudget &&
                  sizeof(SplitSmem<8>) <= kSplitSmemBudget && split_stages(7) == 6,
              "the split CTA's shared memory fits one SM");
static const size_t kSplitSmemBytes[kMaxSlices] = {split_smem_bytes<1>(), split_smem_bytes<2>(), split_smem_bytes<3>(),
                                                   split_smem_bytes<4>(), split_smem_bytes<5>(), split_smem_bytes<6>(),
                                                   split_smem_bytes<7>(), split_smem_bytes<8>()};

using SplitKernel = void (*)(SplitArgs);
static const SplitKernel kSplitKernels[2][2][kMaxSlices] = {  // [multi][narrow][S - 1]
    {{k_split<1, false, false>, k_split<2, false, false>, k_split<3, false, false>, k_split<4, false, false>,
      k_split<5, false, false>, k_split<6, false, false>, k_split<7, false, false>, k_split<8, false, false>},
     {k_split<1, true, false>, k_split<2, true, false>, k_split<3, true, false>, k_split<4, true, false>,
      k_split<5, true, false>, k_split<6, true, false>, k_split<7, true, false>, k_split<8, true, false>}},
    {{k_split<1, false, true>, k_split<2, false, true>, k_split<3, false, true>, k_split<4, false, true>,
      k_split<5, false, true>, k_split<6, false, true>, k_split<7, false, true>, k_split<8, false, true>},
     {k_split<1, true, true>, k_split<2, true, true>, k_split<3, true, true>, k_split<4, true, true>,
      k_split<5, true, true>, k_split<6, true, true>, k_split<7, true, true>, k_split<8, true, true>}}};

// every group sum below 2^23: S * 127^2 * K for the largest padded contracted extent K (the
// product of the largest block extents of the contracted modes)
static bool split_narrow(const sht_plan* p, int S) {
  long double kmax = 1;
  for (int ax : p->maps.colA) {
    int mx = 0;
    for (int v : p->A->bs[ax]) mx = std::max(mx, v);
    kmax *= mx;
  }
  const long double kp = std::ceil(kmax / kSplitK) * kSplitK;
  return (long double)S * 16129.0L * kp < 8388608.0L;
}

static int split_grid(sht_ctx* ctx) {
  static std::once_flag once;
  std::call_once(once, [] {
    for (const auto& plane : kSplitKernels)
      for (const auto& row : plane)
        for (int si = 0; si < kMaxSlices; ++si) {
          const SplitKernel k = row[si];
          SHT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmemBytes[si]));
          int n = 0;
          SHT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kSplitThreads, kSplitSmemBytes[si]));
          if (n != 1) fail(SHT_ERR_STATE, "split kernel must run one CTA per SM (TMEM budget)");
        }
  });
  return ctx->num_sms;
}

void split_execute(sht_plan* p, const SparseArgs& sa, cudaStream_t s) {
  split_slice(p, sa.sc.alpha, s);
  split_launch(p, sa, s);
}

void split_slice(sht_plan* p, double alpha, cudaStream_t s) {
  const int S = p->split_slices;
  uint64_t ab;
  std::memcpy(&ab, &alpha, 8);
  // the execute's flag words start clear (the slicer sets them)
  SHT_CUDA(cudaMemsetAsync(p->sp_err, 0, 8, s));
  if (ab != 0 && p->sp_naitems + p->sp_nbitems > 0) {
    SliceArgs g{};
    SliceOperand& a = g.op[0];
    a.src = p->A->d_data.as<double>();
    a.src_off = p->A->d_offsets.as<long long>();
    a.dims = p->A->d_dims.as<int>();
    a.out_off = p->sp_aoff;
    a.exp_off = p->sp_aeoff;
    a.istart = p->sp_aistart;
    a.out = p->sp_a.as<signed char>();
    a.expo = p->sp_ae.as<short>();
    a.pscale = nullptr;
    a.scale = alpha;
    a.nblocks = p->A->nblocks;
    a.nitems = p->sp_naitems;
    a.fm = modes_of(p->maps.rowA);
    a.km = modes_of(p->maps.colA);
    a.order = p->A->order;
    a.R = kSplitM;
    a.elo = kExpLoA;
    a.ehi = kExpHiA;
    SliceOperand& bo = g.op[1];
    bo.src = p->B->d_data.as<double>();
    bo.src_off = p->B->d_offsets.as<long long>();
    bo.dims = p->B->d_dims.as<int>();
    bo.out_off = p->sp_boff;
    bo.exp_off = p->sp_beoff;
    bo.istart = p->sp_bistart;
    bo.out = p->sp_b.as<signed char>();
    bo.expo = p->sp_be.as<short>();
    bo.pscale = p->sp_bsc.as<double>();
    bo.scale = 1.0;
    bo.nblocks = p->B->nblocks;
    bo.nitems = p->sp_nbitems;
    bo.fm = modes_of(p->maps.colB);
    bo.km = modes_of(p->maps.rowB);
    bo.order = p->B->order;
    bo.R = kSplitN;
    bo.elo = kExpLoB;
    bo.ehi = kExpHiB;
    g.flags = p->sp_err;
    // one wave of resident CTAs, each over a contiguous range of items
    const long long cap = (long long)p->ctx->num_sms * kSliceCtas;
    kSliceKernels[S - 1]<<<(int)std::min(p->sp_naitems + p->sp_nbitems, cap), kSliceWarps * 32, 0, s>>>(g);
    SHT_CUDA(cudaGetLastError());
  }
}

// The kernel arguments of one plan's execute (sa: the FP64 view of the same execute).
static SplitArgs split_args(sht_plan* p, const SparseArgs& sa) {
  uint64_t one, bb;
  const double d1 = 1.0;
  std::memcpy(&one, &d1, 8);
  std::memcpy(&bb, &sa.sc.beta, 8);
  SplitArgs g{};
  g.beta = sa.sc.beta;
  g.beta_zero = sa.sc.beta_zero;
  g.alpha_zero = sa.sc.alpha_zero;
  g.S = p->split_slices;
  g.As = p->sp_a.as<signed char>();
  g.Ae = p->sp_ae.as<short>();
  g.Bs = p->sp_b.as<signed char>();
  g.Be = p->sp_be.as<short>();
  g.Bsc = p->sp_bsc.as<double>();
  g.C = sa.C;
  g.rowtab = p->sp_rowtab.as<int>();
  g.coltab = p->sp_coltab.as<int>();
  g.items = p->sp_items.as<SplitItem>();
  g.prs = p->sp_pairs.as<SplitPair>();
  g.nwork = (int)((bb == one) ? p->bwork_touched : p->bwork);
  g.flags = p->sp_err;
  g.err = ctx_error_word(p->ctx);
  g.wait_limit = p->ctx->wait_limit > 0 ? p->ctx->wait_limit : (1LL << 22);
  g.drain_limit = 1LL << 26;
  return g;
}

void split_launch(sht_plan* p, const SparseArgs& sa, cudaStream_t s) {
  const SplitArgs g = split_args(p, sa);
  if (g.nwork <= 0) return;
  const int grid = (int)std::min<long long>(split_grid(p->ctx), g.nwork);
  kSplitKernels[0][split_narrow(p, g.S) ? 1 : 0][g.S - 1]<<<grid, kSplitThreads, kSplitSmemBytes[g.S - 1], s>>>(g);
  SHT_CUDA(cudaGetLastError());
  // an operand held a non-finite value (the slicer's flag): the tensor-core kernel returned at
  // once and the FP64 tiles compute the execute, with IEEE propagation as in the FP64 forms
  fallback_tiles_if(sa, p->d_bwork.as<int4>(), g.nwork, p->sp_err + kFlagNonFinite, p->ctx->num_sms * 4, s);
}

int split_kind(const sht_plan* p) { return p->split_slices * 2 + (split_narrow(p, p->split_slices) ? 1 : 0); }

size_t split_desc_bytes() { return sizeof(SplitArgs) + sizeof(int); }

bool split_flags_clear(sht_plan* p, cudaStream_t s) {
  int f[2] = {0, 0};
  SHT_CUDA(cudaMemcpyAsync(f, p->sp_err, 8, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
  return f[kFlagNonFinite] == 0 && f[kFlagGeneralExp] == 0;
}

long long split_multi_launch(sht_ctx* ctx, const std::vector<sht_plan*>& plans, const std::vector<SparseArgs>& args,
                             void* host_descs, PoolBuf& descs, cudaStream_t s) {
  if (plans.empty()) return 0;
  const int kind = split_kind(plans[0]);
  const size_t n = plans.size();
  SplitArgs* h = static_cast<SplitArgs*>(host_descs);
  int* first = reinterpret_cast<int*>(h + n);
  long long total = 0;
  for (size_t i = 0; i < n; ++i) {
    if (split_kind(plans[i]) != kind) fail(SHT_ERR_STATE, "one split launch needs one slice count and reassembly");
    h[i] = split_args(plans[i], args[i]);
    first[i] = (int)total;
    total += h[i].nwork;
    if (total > (long long)INT32_MAX) fail(SHT_ERR_UNSUPPORTED, "split launch above 2^31 tiles");
  }
  if (total == 0) return 0;
  const size_t bytes = n * sizeof(SplitArgs) + n * sizeof(int);
  descs = PoolBuf(ctx->pool.get(), bytes, s);
  SHT_CUDA(cudaMemcpyAsync(descs.ptr, h, bytes, cudaMemcpyHostToDevice, s));
  SplitArgs g = h[0];
  g.nwork = (int)total;
  g.multi = descs.as<SplitArgs>();
  g.mfirst = reinterpret_cast<const int*>(descs.as<SplitArgs>() + n);
  g.nmulti = (int)n;
  const int S = plans[0]->split_slices;
  const int grid = (int)std::min<long long>(split_grid(ctx), total);
  kSplitKernels[1][kind & 1][S - 1]<<<grid, kSplitThreads, kSplitSmemBytes[S - 1], s>>>(g);
  SHT_CUDA(cudaGetLastError());
  return total;
}

// ------------------------------------------------------------------ INT8 tensor-core peak
// Roofline denominator of the split kernel: every SM issues `iters` dense 128 x 256 x 32
// kind::i8 MMAs from shared memory into one TMEM accumulator (operands are zero) and waits
// for them with a bounded mbarrier wait; *status is set if a wait expires.
__global__ void __launch_bounds__(128, 1) k_int8_peak(int iters, long long wait_limit, int* status) {
  __shared__ __align__(1024) signed char a[kSplitM * kSplitK];
  __shared__ __align__(1024) signed char b[256 * kSplitK];
  __shared__ __align__(8) unsigned long long done;
  __shared__ unsigned tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < (int)sizeof(a) / 16; i += blockDim.x) reinterpret_cast<int4*>(a)[i] = make_int4(0, 0, 0, 0);
  for (int i = tid; i < (int)sizeof(b) / 16; i += blockDim.x) reinterpret_cast<int4*>(b)[i] = make_int4(0, 0, 0, 0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tbase)), "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tbase;
  if (tid == 0) {
    const unsigned long long da = umma_desc(a), db = umma_desc(b);
    for (int i = 0; i < iters; ++i) umma_i8(tmem, da, db, idesc_i8(256), i > 0 ? 1 : 0);
    umma_commit(&done);
    bool ok = false;
    for (long long i = 0; i < wait_limit && !ok; ++i) ok = mbar_try(&done, 0);
    if (!ok) atomicExch(status, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

double measure_int8_tops(sht_ctx* ctx) {
  const int iters = 1 << 14;
  PoolBuf st(ctx->pool.get(), 256, nullptr);
  SHT_CUDA(cudaMemsetAsync(st.ptr, 0, 4, nullptr));
  cudaEvent_t e0, e1;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    SHT_CUDA(cudaEventRecord(e0, nullptr));
    k_int8_peak<<<ctx->num_sms, 128, 0, nullptr>>>(iters, 1LL << 24, st.as<int>());
    SHT_CUDA(cudaEventRecord(e1, nullptr));
    SHT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double ops = 2.0 * kSplitM * 256.0 * kSplitK * (double)iters * ctx->num_sms;
    if (rep > 0) best = std::max(best, ops / (ms * 1e-3) / 1e12);
  }
  int status = 0;
  SHT_CUDA(cudaMemcpy(&status, st.ptr, 4, cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status) fail(SHT_ERR_TIMEOUT, "INT8 peak probe: a bounded wait on the tensor cores expired");
  return best;
}

// ------------------------------------------------------------------ operand pipeline ceiling
// The split kernel's operand pipeline with nothing after it: per k-step the producer bulk-copies
// one stage (the A and B slabs of 7 slices, 28 KB + 7 KB, from a buffer resident in L2) into a
// six-deep ring and the MMA issuer runs the seven-MMA triangle on it (N = 224 .. 32) into one
// of two TMEM sets.  The stage copies and the tensor core's operand reads share the SM's
// shared-memory bandwidth, so this rate, not the dense INT8 peak, is what the split kernel can
// reach per k-step.  Waits are bounded; *status is set if one expires.
constexpr int kPipeS = 7, kPipeStages = 6, kPipeStage = kPipeS * (kAChunk + kBChunk);
__global__ void __launch_bounds__(64, 1) k_split_pipe_peak(const signed char* __restrict__ src, long long nstage_src,
                                                           int iters, long long wait_limit, int* status) {
  extern __shared__ __align__(1024) unsigned char pipe_smem[];
  __shared__ __align__(8) unsigned long long full[kPipeStages], empty[kPipeStages], done;
  __shared__ unsigned tbase;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tbase)), "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < kPipeStages; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tbase;
  const unsigned a_bytes = kPipeS * kAChunk, b_bytes = kPipeS * kBChunk;
  auto wait = [&](unsigned long long* bar, unsigned parity) {
    for (long long w = 0; w < wait_limit; ++w)
      if (mbar_try(bar, parity)) return true;
    atomicExch(status, 1);
    return false;
  };
  if (tid == 0) {
    int issued = 0;
    for (int i = 0; i < iters; ++i, ++issued) {
      const int st = i % kPipeStages;
      if (i >= kPipeStages && !wait(&empty[st], (unsigned)(((i / kPipeStages) - 1) & 1))) break;
      const signed char* s = src + ((blockIdx.x * 7919LL + i * 131LL) % nstage_src) * kPipeStage;
      unsigned char* d = pipe_smem + st * kPipeStage;
      mbar_expect_tx(&full[st], a_bytes + b_bytes);
      bulk_g2s(d, s, a_bytes, &full[st]);
      bulk_g2s(d + a_bytes, s + a_bytes, b_bytes, &full[st]);
    }
    // copies still in flight write into shared memory: wait for them before the CTA exits
    for (int j = issued > kPipeStages ? issued - kPipeStages : 0; j < issued; ++j)
      wait(&full[j % kPipeStages], (unsigned)((j / kPipeStages) & 1));
  } else if (tid == 32) {
    for (int i = 0; i < iters; ++i) {
      const int st = i % kPipeStages;
      if (!wait(&full[st], (unsigned)((i / kPipeStages) & 1))) break;
      tc_fence_after();
      const unsigned char* a = pipe_smem + st * kPipeStage;
      const unsigned d = tmem + (unsigned)((i & 1) * (kPipeS * kSplitN + kSplitN));
#pragma unroll
      for (int t = 1; t <= kPipeS; ++t)
        umma_i8(d + (unsigned)((t - 1) * kSplitN), umma_desc(a + (t - 1) * kAChunk), umma_desc(a + a_bytes),
                idesc_i8(kSplitN * (kPipeS + 1 - t)), t == 1 ? 0 : 1);
      umma_commit(&empty[st]);
    }
    umma_commit(&done);  // every MMA issued has finished before TMEM is released
    wait(&done, 0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
}

double measure_split_pipe_tops(sht_ctx* ctx) {
  const int iters = 4000;
  const long long nstage_src = (32LL << 20) / kPipeStage;  // 32 MB of slabs: resident in L2
  PoolBuf src(ctx->pool.get(), nstage_src * kPipeStage, nullptr), st(ctx->pool.get(), 256, nullptr);
  // non-zero slices (0x5b = 91 in every byte): the tensor core's rate does not depend on zero operands
  SHT_CUDA(cudaMemsetAsync(src.ptr, 0x5b, nstage_src * kPipeStage, nullptr));
  SHT_CUDA(cudaMemsetAsync(st.ptr, 0, 4, nullptr));
  const int smem = kPipeStages * kPipeStage;
  SHT_CUDA(cudaFuncSetAttribute(k_split_pipe_peak, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  cudaEvent_t e0, e1;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    SHT_CUDA(cudaEventRecord(e0, nullptr));
    k_split_pipe_peak<<<ctx->num_sms, 64, smem, nullptr>>>(src.as<signed char>(), nstage_src, iters, 1LL << 24,
                                                           st.as<int>());
    SHT_CUDA(cudaEventRecord(e1, nullptr));
    SHT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    // the triangle's slice products: 28 of 128 x 32 x 32 per k-step
    const double ops = 2.0 * kSplitM * (kSplitN * kPipeS * (kPipeS + 1) / 2) * kSplitK * (double)iters * ctx->num_sms;
    if (rep > 0) best = std::max(best, ops / (ms * 1e-3) / 1e12);
  }
  int status = 0;
  SHT_CUDA(cudaMemcpy(&status, st.ptr, 4, cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status) fail(SHT_ERR_TIMEOUT, "split pipeline probe: a bounded wait expired");
  return best;
}

}  // namespace sht
