// noalloc.cu -- Kernel<double>::call for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc at all: code running inside a CUDA
// graph that is being captured or replayed by someone else, allocator-free plugin hosts that
// hand over only pre-registered buffers, or processes whose device memory is fully reserved
// by another runtime.  For them sht_kernel_call_static runs the FP64 stack product of a
// Kernel<double> (the same result bits as sht_kernel_call) on the FP64 tensor cores, with its
// only scratch -- the operands rewritten into matrix form -- in a file-scope device array of
// kStaticScratchBytes.  Every GPU that loads this library holds that array until the process
// exits.
//
// Set-up: the first call on a device (with that device current) looks up the array's device
// address with cudaGetSymbolAddress and caches it.  Under CUDA's lazy module loading that
// first call is also the one that loads this library's module on the device, which commits
// the 32 MiB array; make that first call outside any stream capture.  All calls share the one
// array and it keeps the last call's contents: every call rewrites the part it uses (padding
// included) before reading it, and calls whose work overlaps on the GPU (other streams, or
// another thread) race on it.
#include <cstring>
#include <map>
#include <mutex>

#include "device_common.cuh"
#include "tile_pipe.cuh"

namespace sht {

constexpr size_t kStaticScratchBytes = 32u << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// device address of g_static_scratch per device, filled on the first call on that device
static std::mutex g_scratch_mu;
static std::map<int, void*> g_scratch_addr;

static void* static_scratch() {
  int dev = 0;
  SHT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  auto it = g_scratch_addr.find(dev);
  if (it != g_scratch_addr.end()) return it->second;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess || !p)
    fail(SHT_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch: ") + cudaGetErrorString(e));
  g_scratch_addr[dev] = p;
  return p;
}

struct StackForm {
  int order;
  int dims[kMaxOrder];
  ModeMap fm, km;        // free / contracted modes of this operand
  long long src_stride;  // elements between consecutive ops
  int ld, K4;            // matrix form: ld (free extent rounded up to even) x K4
  double scale;
  int scale_on;
  double kpad;
};

// one CTA per op: the op's block into matrix form (as k_matform does for block-sparse plans)
__global__ void __launch_bounds__(256) k_matform_stack(const double* __restrict__ src, StackForm f,
                                                       double* __restrict__ dst, long long nb_ops) {
  int st[kMaxOrder];
  block_strides(f.dims, f.order, st);
  int m = 1, K = 1;
  for (int t = 0; t < f.fm.n; ++t) m *= f.dims[f.fm.x[t]];
  for (int t = 0; t < f.km.n; ++t) K *= f.dims[f.km.x[t]];
  auto offset = [&](const ModeMap& mm, int idx) {
    int off = 0;
    for (int t = 0; t < mm.n; ++t) {
      const int e = f.dims[mm.x[t]];
      off += (idx % e) * st[mm.x[t]];
      idx /= e;
    }
    return off;
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (long long op = blockIdx.x; op < nb_ops; op += gridDim.x) {
    const double* s = src + op * f.src_stride;
    double* o = dst + op * (long long)f.ld * f.K4;
    for (int k = warp; k < f.K4; k += nwarps) {
      const int okk = k < K ? offset(f.km, k) : 0;
      for (int r = lane; r < f.ld; r += 32) {
        double v;
        if (k >= K) {
          v = f.kpad;
        } else if (r < m) {
          v = s[offset(f.fm, r) + okk];
          if (f.scale_on) v = mul_rn(f.scale, v);
        } else {
          v = 0.0;
        }
        o[(long long)k * f.ld + r] = v;
      }
    }
  }
}

using StaticCfg = PipeCfg<64, 64, 2>;
// launched with the default dynamic shared-memory limit on every device: no per-device
// cudaFuncSetAttribute is needed
static_assert(sizeof(PipeSmem<StaticCfg>) <= 48 * 1024, "static stack tile must fit the default 48 KB");

struct StackTiles {
  TileMaps mp;
  TileScalars<double> sc;
  const double* Am; const double* Bm; double* C;
  long long size_c, a_op, b_op;  // elements per op in C, A_mat, B_mat
  int lda, ldb, K4;
  int dimsC[kMaxOrder];
  int tiles_per_op;
};

__global__ void __launch_bounds__(128) k_stack_tc(StackTiles g) {
  extern __shared__ __align__(16) unsigned char smem[];
  PipeSmem<StaticCfg>& sm = *reinterpret_cast<PipeSmem<StaticCfg>*>(smem);
  const long long op = blockIdx.x / g.tiles_per_op;
  const int tile = (int)(blockIdx.x % g.tiles_per_op);
  auto getc = [&](double*& p, const int*& d) {
    p = g.C + op * g.size_c;
    d = g.dimsC;
  };
  auto getpair = [&](int, PairView& v) {
    v.a = g.Am + op * g.a_op;
    v.lda = g.lda;
    v.b = g.Bm + op * g.b_op;
    v.ldb = g.ldb;
    v.K4 = g.K4;
  };
  tile_run_pipe<StaticCfg>(g.mp, g.sc, tile, getc, getpair, 0, 1, sm);
}

static ModeMap modes_of(const std::vector<int>& v) {
  ModeMap m{};
  m.n = (int)v.size();
  for (size_t i = 0; i < v.size(); ++i) m.x[i] = m.y[i] = v[i];
  return m;
}

void stack_call_static(sht_kernel* k, const double* a, const double* b, double* c, int64_t nb_ops, cudaStream_t s) {
  if (k->dtype != SHT_F64) fail(SHT_ERR_UNSUPPORTED, "the allocation-free call runs Kernel<double>");
  if (nb_ops < 0) fail(SHT_ERR_INVALID, "nb_ops < 0");
  if (nb_ops == 0) return;
  if (!a || !b || !c) fail(SHT_ERR_INVALID, "null operand");
  const long long m = k->m, n = k->n, K = k->k;
  const long long lda = (m + 1) & ~1LL, ldb = (n + 1) & ~1LL, K4 = (K + 3) & ~3LL;
  const long long a_op = lda * K4, b_op = ldb * K4;
  const long double need = (long double)nb_ops * (long double)(a_op + b_op) * 8.0L;
  if (need > (long double)kStaticScratchBytes)
    fail(SHT_ERR_SIZE, "sht_kernel_call_static: " + std::to_string((long long)need) +
                           " bytes of scratch needed, the static scratch holds " +
                           std::to_string(kStaticScratchBytes) + " bytes (split the stack)");
  double* scratch = static_cast<double*>(static_scratch());
  double* Am = scratch;
  double* Bm = scratch + nb_ops * a_op;

  StackForm fa{};
  fa.order = (int)k->sa.size();
  for (int i = 0; i < fa.order; ++i) fa.dims[i] = k->sa[i];
  fa.fm = modes_of(k->maps.rowA);
  fa.km = modes_of(k->maps.colA);
  fa.src_stride = k->size_a;
  fa.ld = (int)lda;
  fa.K4 = (int)K4;
  fa.scale = k->alpha;
  fa.scale_on = k->alpha != 1.0;
  fa.kpad = -0.0;
  StackForm fb{};
  fb.order = (int)k->sb.size();
  for (int i = 0; i < fb.order; ++i) fb.dims[i] = k->sb[i];
  fb.fm = modes_of(k->maps.colB);
  fb.km = modes_of(k->maps.rowB);
  fb.src_stride = k->size_b;
  fb.ld = (int)ldb;
  fb.K4 = (int)K4;
  fb.scale = 1.0;
  fb.scale_on = 0;
  fb.kpad = 0.0;
  const int grid = (int)std::min<long long>(nb_ops, (long long)k->ctx->num_sms * 8);
  k_matform_stack<<<grid, 256, 0, s>>>(a, fa, Am, nb_ops);
  k_matform_stack<<<grid, 256, 0, s>>>(b, fb, Bm, nb_ops);

  StackTiles g{};
  g.mp.row.n = (int)k->maps.rowA.size();
  for (size_t i = 0; i < k->maps.rowA.size(); ++i) { g.mp.row.x[i] = k->maps.rowA[i]; g.mp.row.y[i] = k->maps.rowC[i]; }
  g.mp.kk.n = (int)k->maps.colA.size();
  for (size_t i = 0; i < k->maps.colA.size(); ++i) { g.mp.kk.x[i] = k->maps.colA[i]; g.mp.kk.y[i] = k->maps.rowB[i]; }
  g.mp.col.n = (int)k->maps.colB.size();
  for (size_t i = 0; i < k->maps.colB.size(); ++i) { g.mp.col.x[i] = k->maps.colB[i]; g.mp.col.y[i] = k->maps.colC[i]; }
  g.mp.oA = (int)k->sa.size();
  g.mp.oB = (int)k->sb.size();
  g.mp.oC = (int)k->sc.size();
  for (size_t i = 0; i < k->sc.size(); ++i) g.dimsC[i] = k->sc[i];
  uint64_t ab, bb;
  std::memcpy(&ab, &k->alpha, 8);
  std::memcpy(&bb, &k->beta, 8);
  g.sc = {k->alpha, k->beta, bb == 0, ab == 0};
  g.Am = Am;
  g.Bm = Bm;
  g.C = c;
  g.size_c = k->size_c;
  g.a_op = a_op;
  g.b_op = b_op;
  g.lda = (int)lda;
  g.ldb = (int)ldb;
  g.K4 = (int)K4;
  g.tiles_per_op = (int)(((m + StaticCfg::TM - 1) / StaticCfg::TM) * ((n + StaticCfg::TN - 1) / StaticCfg::TN));
  const long long blocks = nb_ops * g.tiles_per_op;
  if (blocks > 0x7fffffffLL) fail(SHT_ERR_UNSUPPORTED, "stack too large for one launch");
  k_stack_tc<<<(unsigned)blocks, 128, sizeof(PipeSmem<StaticCfg>), s>>>(g);
  SHT_CUDA(cudaGetLastError());
}

}  // namespace sht
