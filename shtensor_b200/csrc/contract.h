// contract.h -- plan object and entry points of the block-sparse contraction.
#pragma once

#include "sht_internal.h"
#include "tile_types.h"

struct sht_plan {
  std::shared_ptr<sht::DevicePool> keep;  // declared first: released after the buffers below
  sht_ctx* ctx = nullptr;
  sht_mode mode = SHT_MODE_PLAIN_FP64;
  sht_tensor *A = nullptr, *B = nullptr, *C = nullptr;
  ShtMaps maps;
  sht::TileMaps tmaps{};
  long long npairs = 0, ncblk = 0, nwork = 0, nwork_touched = 0;
  double flops = 0.0, plan_ms = 0.0, exec_ms = 0.0;
  double eps = 0.0;                 // screening threshold and norm of the pair list
  sht_norm norm = SHT_NORM_FROBENIUS;
  sht::PoolBuf d_flops;             // device total of the flop count until it is read
  sht::PoolBuf d_npairs;            // device pair count, when the host's sized the pair list
  sht::PoolBuf d_missing;           // product blocks absent from C, when the build assumed none
  bool flops_pending = false;       // d_flops not yet copied into flops
  cudaEvent_t flops_event = nullptr;  // recorded after d_flops is computed
  int shape = 0, work_tm = 64, work_tn = 64;
  sht::PoolBuf d_pair_a, d_pair_b;  // int32 storage indices into A / B, canonical order
  sht::PoolBuf d_pstart;            // int32[ncblk + 1]
  sht::PoolBuf d_work;              // int2 (C block, tile) for the plain path
  sht::PoolBuf d_cm, d_cn, d_cksum; // per C block: rows, columns, sum of the pairs' k
  // batched path
  sht::PoolBuf d_bwork;             // int4 (C block, tile, class, 0)
  sht::PoolBuf d_counter;           // work counter of the persistent kernel
  long long bwork = 0, bwork_touched = 0;
  int bclass_shape[8] = {0};
  int nclass = 0;
  // matrix form of the operands (batched and split paths)
  sht::PoolBuf mf_a, mf_b;          // A_mat / B_mat elements
  sht::PoolBuf mf_aoff, mf_boff;    // int64 per block offsets
  sht::PoolBuf mf_ald, mf_bld;      // int32 per block leading dimensions (even)
  sht::PoolBuf mf_ak4;              // int32 per A block contracted extent rounded up to 4
  sht::PoolBuf mf_aitems, mf_bitems;  // int4 (block, k0, k1, 0) slabs of the matform kernel
  long long mf_naitems = 0, mf_nbitems = 0;
  long long mf_elems = 0;
  // split path: INT8 slices (K-major rows), row / column exponents, error words
  sht::PoolBuf sp_a, sp_b, sp_ae, sp_be;
  sht::PoolBuf sp_bsc;                // B column scales 2^f as doubles (the reassembly's)
  // one upload: per block of A and of B its slice offset, exponent offset and first slicer
  // item (items of 32 rows), and the kernels' error words (zero)
  sht::PoolBuf sp_meta;
  long long *sp_aoff = nullptr, *sp_aeoff = nullptr, *sp_aistart = nullptr;
  long long *sp_boff = nullptr, *sp_beoff = nullptr, *sp_bistart = nullptr;
  int* sp_err = nullptr;            // the execute's flag words (non-finite input, wide exponents)
  long long sp_naitems = 0, sp_nbitems = 0;
  sht::PoolBuf sp_items, sp_pairs;    // per-tile and per-pair records of the split kernel
  sht::PoolBuf sp_rowtab, sp_coltab;  // element offsets of every C row / column in its block
  int split_slices = 0;
  // graph replay
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  double graph_alpha = 0.0, graph_beta = 0.0;
  ~sht_plan() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (flops_event) cudaEventDestroy(flops_event);
  }
};

namespace sht {

sht_plan* plan_create(sht_ctx* ctx, const std::string& expr, sht_tensor* A, sht_tensor* B, sht_tensor* C,
                      double eps, sht_norm norm, sht_mode mode, cudaStream_t s);
// plan_create in two steps: the host checks and the parse (no device work but reading stale
// host patterns back on s), then the pair list, result pattern and per-block statistics on s
sht_plan* plan_init(sht_ctx* ctx, const std::string& expr, sht_tensor* A, sht_tensor* B, sht_tensor* C,
                    double eps, sht_norm norm, sht_mode mode, cudaStream_t s);
// speculate: when C already has a pattern, assume the product adds no block to it and check
// that at the work list's read-back (device_work_list throws PatternGrew if it did), which
// saves a synchronization when C is contracted into repeatedly.
void plan_build(sht_plan* p, cudaStream_t s, bool speculate = false);
struct PatternGrew {};
void build_work(sht_plan* p, int TM, int TN, cudaStream_t s);
void cblock_stats(sht_plan* p, cudaStream_t s);
// The plan's flop count; the first call after planning copies it from the device (a sync),
// so callers that synchronize anyway read it right after.
double plan_flops(sht_plan* p, cudaStream_t s);
// Cost-ordered work list (C block, tile, shape) on the device: fixed_shape >= 0 uses one
// shape (tm x tn) for every block, otherwise per size class from class_shape (or the model).
// A device scalar, or the sum of two (b may be null), for a read-back.
struct DevSum {
  const long long* a;
  const long long* b;
};
// extra (up to three device scalars) are read back with the list's own counts into extra_out.
// order_key (per C block, ascending, order_bits wide; blocks without pairs must key last)
// replaces the cost order when given.
void device_work_list(sht_plan* p, int fixed_tm, int fixed_tn, bool per_class, cudaStream_t s,
                      const DevSum* extra = nullptr, long long* extra_out = nullptr, int nextra = 0,
                      const unsigned long long* order_key = nullptr, int order_bits = 0);
void plan_execute(sht_plan* p, double alpha, double beta, cudaStream_t s);
void batched_prepare(sht_plan* p, cudaStream_t s);
// the persistent kernel alone, with the operands already in matrix form (matform_execute)
void batched_launch(sht_plan* p, const SparseArgs& g, cudaStream_t s);
void batched_execute(sht_plan* p, const SparseArgs& g, long long nwork_plain, cudaStream_t s);
void autotune(sht_plan* p, const char* cache_file, cudaStream_t s);
void matform_prepare(sht_plan* p, cudaStream_t s);
size_t batched_desc_bytes();
int batched_ctas_per_sm(sht_ctx* ctx);
long long batched_multi_launch(sht_ctx* ctx, const std::vector<sht_plan*>& plans, const std::vector<SparseArgs>& args,
                               void* host_descs, PoolBuf& descs, PoolBuf& counter, int ctas_per_sm, cudaStream_t s);
SparseArgs sparse_args(sht_plan* p, double alpha, double beta);
void plan_touch(sht_plan* p, cudaStream_t s);  // plan buffers and tensors: next used on s
void split_prepare(sht_plan* p, int S, cudaStream_t s);  // split_layout + split_records
void split_execute(sht_plan* p, const SparseArgs& sa, cudaStream_t s);  // split_slice + split_launch
// slice buffers and the slicer's items: depends on the patterns of A and B only
void split_layout(sht_plan* p, int S, cudaStream_t s);
// work list, C offset tables, tile and pair records: needs plan_build
void split_records(sht_plan* p, cudaStream_t s);
// the slicer over A (scaled by alpha) and B: needs split_layout only
void split_slice(sht_plan* p, double alpha, cudaStream_t s);
// the tensor-core kernel: needs everything above
void split_launch(sht_plan* p, const SparseArgs& sa, cudaStream_t s);
// The FP64 tile kernel over the split work list (int4 (C block, 128 x 32 tile, ., .)), run only
// when the device word *flag is set (persistent grid; it returns at once otherwise).
void fallback_tiles_if(const SparseArgs& g, const int4* work, long long nwork, const int* flag, int grid,
                       cudaStream_t s);
int split_slices_default();
// Serving: requests of one launch share the kind (slice count and reassembly instance); the
// host buffer holds split_desc_bytes() per request; the flags are read after the slicer (a
// synchronization of s) and must be clear for a request to join a split launch.
int split_kind(const sht_plan* p);
size_t split_desc_bytes();
bool split_flags_clear(sht_plan* p, cudaStream_t s);
long long split_multi_launch(sht_ctx* ctx, const std::vector<sht_plan*>& plans, const std::vector<SparseArgs>& args,
                             void* host_descs, PoolBuf& descs, cudaStream_t s);
void matform_execute(sht_plan* p, double alpha, cudaStream_t s);
void block_dims_sizes(const sht_tensor* t, const long long* ids, long long n, int* dims, long long* sizes,
                      cudaStream_t s);
void tensor_compress_device(sht_tensor* t, cudaStream_t s);
void tensor_filter_device(sht_tensor* t, double eps, sht_norm norm, int compress, cudaStream_t s);

}  // namespace sht
