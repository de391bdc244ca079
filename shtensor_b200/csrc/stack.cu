// stack.cu -- Kernel<T>::call on the device: nb_ops same-shape (A, B, C) block triples.
//
// Replaces the two CPU back ends of src/Kernel/KernelImpl.cpp (LAPACK reshape+gemm, :75-208,
// and the asmjit AVX2 gather/FMA/scatter microkernel, :210-770) with one CUDA kernel: every
// CTA takes one tile of one op's C block and runs the shared output-stationary tile
// (tile_core.cuh), so the permutes are fused into the operand gathers and the per-element
// arithmetic is the XMM kernel's.  FP64 and FP32 (Kernel<double>, Kernel<float>).
#include <algorithm>
#include <cstring>

#include "device_common.cuh"
#include "tile_core.cuh"

namespace sht {

template <typename T>
struct StackArgs {
  TileMaps mp;
  TileScalars<T> sc;
  const T* A; const T* B; T* C;
  long long size_a, size_b, size_c;
  int dimsA[kMaxOrder], dimsB[kMaxOrder], dimsC[kMaxOrder];
  int tiles_per_op;
};

template <typename T, class Cfg>
__global__ void __launch_bounds__(Cfg::kThreads) k_stack(StackArgs<T> g) {
  __shared__ TileSmem<T, Cfg> sm;
  const long long op = blockIdx.x / g.tiles_per_op;
  const int tile = (int)(blockIdx.x % g.tiles_per_op);
  auto getc = [&](T*& p, const int*& d) {
    p = g.C + op * g.size_c;
    d = g.dimsC;
  };
  auto getpair = [&](int, const T*& a, const int*& ad, const T*& b, const int*& bd) {
    a = g.A + op * g.size_a;
    ad = g.dimsA;
    b = g.B + op * g.size_b;
    bd = g.dimsB;
  };
  tile_run<T, Cfg>(g.mp, g.sc, tile, getc, getpair, 0, 1, sm);
}

using S64x64 = TileCfg<64, 64, 16, 4, 4>;
using S128x32 = TileCfg<128, 32, 16, 8, 2>;
using S32x128 = TileCfg<32, 128, 16, 2, 8>;
using S32x32 = TileCfg<32, 32, 16, 2, 2>;
using S16x16 = TileCfg<16, 16, 16, 2, 2>;

struct StackShape { int tm, tn; };
static const StackShape kStackShapes[] = {{64, 64}, {128, 32}, {32, 128}, {32, 32}, {16, 16}};

static int pick_stack_shape(long long m, long long n) {
  double best = 1e300;
  int bi = 0;
  for (int i = 0; i < 5; ++i) {
    const long long tm = kStackShapes[i].tm, tn = kStackShapes[i].tn;
    const long long tiles = ((m + tm - 1) / tm) * ((n + tn - 1) / tn);
    const double cost = (double)tiles * (double)(tm * tn + 1024);
    if (cost < best) { best = cost; bi = i; }
  }
  return bi;
}

static bool is_device_pointer(const void* p) {
  cudaPointerAttributes at{};
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

template <typename T>
static void launch_stack(sht_kernel* k, const T* a, const T* b, T* c, long long nb_ops, cudaStream_t s) {
  StackArgs<T> g{};
  g.mp.row.n = (int)k->maps.rowA.size();
  for (size_t i = 0; i < k->maps.rowA.size(); ++i) { g.mp.row.x[i] = k->maps.rowA[i]; g.mp.row.y[i] = k->maps.rowC[i]; }
  g.mp.kk.n = (int)k->maps.colA.size();
  for (size_t i = 0; i < k->maps.colA.size(); ++i) { g.mp.kk.x[i] = k->maps.colA[i]; g.mp.kk.y[i] = k->maps.rowB[i]; }
  g.mp.col.n = (int)k->maps.colB.size();
  for (size_t i = 0; i < k->maps.colB.size(); ++i) { g.mp.col.x[i] = k->maps.colB[i]; g.mp.col.y[i] = k->maps.colC[i]; }
  g.mp.oA = (int)k->sa.size();
  g.mp.oB = (int)k->sb.size();
  g.mp.oC = (int)k->sc.size();
  for (size_t i = 0; i < k->sa.size(); ++i) g.dimsA[i] = k->sa[i];
  for (size_t i = 0; i < k->sb.size(); ++i) g.dimsB[i] = k->sb[i];
  for (size_t i = 0; i < k->sc.size(); ++i) g.dimsC[i] = k->sc[i];
  g.sc.alpha = (T)k->alpha;
  g.sc.beta = (T)k->beta;
  const T al = (T)k->alpha, be = (T)k->beta;
  unsigned char zb[sizeof(T)] = {0};
  g.sc.alpha_zero = std::memcmp(&al, zb, sizeof(T)) == 0;
  g.sc.beta_zero = std::memcmp(&be, zb, sizeof(T)) == 0;
  g.A = a; g.B = b; g.C = c;
  g.size_a = k->size_a; g.size_b = k->size_b; g.size_c = k->size_c;
  const int sh = pick_stack_shape(k->m, k->n);
  const long long tm = kStackShapes[sh].tm, tn = kStackShapes[sh].tn;
  g.tiles_per_op = (int)(((k->m + tm - 1) / tm) * ((k->n + tn - 1) / tn));
  const long long blocks = nb_ops * g.tiles_per_op;
  if (blocks > 0x7fffffffLL) fail(SHT_ERR_UNSUPPORTED, "stack too large for one launch");
  const unsigned grid = (unsigned)blocks;
  switch (sh) {
    case 0: k_stack<T, S64x64><<<grid, S64x64::kThreads, 0, s>>>(g); break;
    case 1: k_stack<T, S128x32><<<grid, S128x32::kThreads, 0, s>>>(g); break;
    case 2: k_stack<T, S32x128><<<grid, S32x128::kThreads, 0, s>>>(g); break;
    case 3: k_stack<T, S32x32><<<grid, S32x32::kThreads, 0, s>>>(g); break;
    default: k_stack<T, S16x16><<<grid, S16x16::kThreads, 0, s>>>(g); break;
  }
  SHT_CUDA(cudaGetLastError());
}

void stack_call(sht_kernel* k, const void* a, const void* b, void* c, int64_t nb_ops, cudaStream_t s) {
  if (nb_ops < 0) fail(SHT_ERR_INVALID, "nb_ops < 0");
  if (nb_ops == 0) return;
  if (!a || !b || !c) fail(SHT_ERR_INVALID, "null operand");
  const size_t es = k->dtype == SHT_F64 ? 8 : 4;
  const bool dev = is_device_pointer(a) && is_device_pointer(b) && is_device_pointer(c);
  if (dev) {
    if (k->dtype == SHT_F64)
      launch_stack<double>(k, (const double*)a, (const double*)b, (double*)c, nb_ops, s);
    else
      launch_stack<float>(k, (const float*)a, (const float*)b, (float*)c, nb_ops, s);
    return;
  }
  // host operands: stage through the pool
  DevicePool* pool = k->ctx->pool.get();
  const size_t ba = (size_t)nb_ops * k->size_a * es, bb = (size_t)nb_ops * k->size_b * es,
               bc = (size_t)nb_ops * k->size_c * es;
  PoolBuf da(pool, ba, s), db(pool, bb, s), dc(pool, bc, s);
  SHT_CUDA(cudaMemcpyAsync(da.ptr, a, ba, cudaMemcpyHostToDevice, s));
  SHT_CUDA(cudaMemcpyAsync(db.ptr, b, bb, cudaMemcpyHostToDevice, s));
  SHT_CUDA(cudaMemcpyAsync(dc.ptr, c, bc, cudaMemcpyHostToDevice, s));
  if (k->dtype == SHT_F64)
    launch_stack<double>(k, da.as<double>(), db.as<double>(), dc.as<double>(), nb_ops, s);
  else
    launch_stack<float>(k, da.as<float>(), db.as<float>(), dc.as<float>(), nb_ops, s);
  SHT_CUDA(cudaMemcpyAsync(c, dc.ptr, bc, cudaMemcpyDeviceToHost, s));
  SHT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace sht
