// capi.cpp -- the extern "C" boundary.  Every entry point catches the runtime's errors and
// returns a status; sht_last_error() gives the message of the calling thread's last failure.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "contract.h"

namespace sht {

double measure_fp64_tflops(sht_ctx* ctx);
double measure_int8_tops(sht_ctx* ctx);
double measure_split_pipe_tops(sht_ctx* ctx);
double measure_dmma_tflops(sht_ctx* ctx);
void stack_call_static(sht_kernel* k, const double* a, const double* b, double* c, int64_t nb_ops, cudaStream_t s);

// A lane (stream + two events) borrowed from the context for the length of one call.
struct LaneLease {
  sht_ctx* ctx;
  sht_ctx::Lane lane;
  explicit LaneLease(sht_ctx* c) : ctx(c) {
    {
      std::lock_guard<std::mutex> lk(ctx->lanes_mu);
      if (!ctx->lanes.empty()) {
        lane = ctx->lanes.back();
        ctx->lanes.pop_back();
        return;
      }
    }
    // the highest priority: the plan's short kernels are scheduled ahead of the slicer's
    // remaining blocks on the caller's stream
    int lo = 0, hi = 0;
    SHT_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    SHT_CUDA(cudaStreamCreateWithPriority(&lane.stream, cudaStreamNonBlocking, hi));
    SHT_CUDA(cudaEventCreateWithFlags(&lane.start, cudaEventDisableTiming));
    SHT_CUDA(cudaEventCreateWithFlags(&lane.done, cudaEventDisableTiming));
  }
  ~LaneLease() {
    // work still queued on the stream stays ordered by the events of whoever uses it next
    std::lock_guard<std::mutex> lk(ctx->lanes_mu);
    ctx->lanes.push_back(lane);
  }
  LaneLease(const LaneLease&) = delete;
  LaneLease& operator=(const LaneLease&) = delete;
};

// Split form of sht_contract with the slicer overlapped: the slices depend on the patterns and
// values of A and B only, so they run on the caller's stream s while the pair list, result
// pattern and records are built on a second stream, which first waits for the work already
// on s (earlier writes of C) and which s waits for before the tensor-core kernel.
static void contract_split(sht_plan* p, double alpha, double beta, cudaStream_t s) {
  sht_ctx* ctx = p->ctx;
  LaneLease lane(ctx);
  const cudaStream_t ps = lane.lane.stream;
  SHT_CUDA(cudaEventRecord(lane.lane.start, s));
  split_layout(p, ctx->split_slices ? ctx->split_slices : split_slices_default(), s);
  split_slice(p, alpha, s);
  trace("contract: slicer launched", s);
  // The build reads the tensors' indices (complete: every index change in this library returns
  // after it is done) and, with screening, A's and B's values, which earlier work on s may still
  // write: only then does it wait for s.  So a contraction into a C whose pattern holds the
  // product plans while the previous contraction on s still runs.
  if (p->eps > 0.0) SHT_CUDA(cudaStreamWaitEvent(ps, lane.lane.start, 0));
  try {
    plan_build(p, ps, true);
    split_records(p, ps);
  } catch (const PatternGrew&) {
    // the product adds blocks to C: build again, growing C's pattern, which moves C's values
    // (after earlier work on s has written them)
    SHT_CUDA(cudaStreamWaitEvent(ps, lane.lane.start, 0));
    plan_build(p, ps, false);
    split_records(p, ps);
  }
  SHT_CUDA(cudaEventRecord(lane.lane.done, ps));
  SHT_CUDA(cudaStreamWaitEvent(s, lane.lane.done, 0));
  plan_touch(p, s);
  split_launch(p, sparse_args(p, alpha, beta), s);
  trace("contract: split kernel launched", s);
}

// A bounded wait of an earlier split launch on this context ran out: report it at this call.
static void raise_pending(sht_ctx* ctx) {
  if (const int e = ctx_take_error(ctx))
    fail((sht_status)e, "an earlier split-precision launch on this context failed: a bounded wait on the tensor "
                        "cores expired (its result is undefined)");
}

// Batched form of sht_contract, overlapped the same way: the matrix form of A and B (patterns
// and values of A and B only) on the caller's stream, the plan and its size-class work list on
// the lane stream.
static void contract_batched(sht_plan* p, double alpha, double beta, cudaStream_t s) {
  sht_ctx* ctx = p->ctx;
  LaneLease lane(ctx);
  const cudaStream_t ps = lane.lane.stream;
  SHT_CUDA(cudaEventRecord(lane.lane.start, s));
  p->d_counter = PoolBuf(ctx->pool.get(), 256, s);
  matform_prepare(p, s);
  uint64_t ab;
  std::memcpy(&ab, &alpha, 8);
  if (ab != 0) matform_execute(p, alpha, s);
  trace("contract: matrix form launched", s);
  // as in the split form: the build waits for earlier work on s only when it reads values
  if (p->eps > 0.0) SHT_CUDA(cudaStreamWaitEvent(ps, lane.lane.start, 0));
  try {
    plan_build(p, ps, true);
    device_work_list(p, 0, 0, true, ps);
  } catch (const PatternGrew&) {
    SHT_CUDA(cudaStreamWaitEvent(ps, lane.lane.start, 0));
    plan_build(p, ps, false);
    device_work_list(p, 0, 0, true, ps);
  }
  SHT_CUDA(cudaEventRecord(lane.lane.done, ps));
  SHT_CUDA(cudaStreamWaitEvent(s, lane.lane.done, 0));
  plan_touch(p, s);
  batched_launch(p, sparse_args(p, alpha, beta), s);
  trace("contract: batched kernel launched", s);
}

static void prepare_mode(sht_plan* p, cudaStream_t s) {
  if (p->mode == SHT_MODE_BATCHED_FP64) batched_prepare(p, s);
  if (p->mode == SHT_MODE_SPLIT) split_prepare(p, p->ctx->split_slices ? p->ctx->split_slices : split_slices_default(), s);
}

volatile int* ctx_error_word(sht_ctx* ctx) {
  std::lock_guard<std::mutex> lk(ctx->err_mu);
  if (!ctx->err_host) {
    void* h = nullptr;
    SHT_CUDA(cudaHostAlloc(&h, 64, cudaHostAllocMapped));
    std::memset(h, 0, 64);
    void* d = nullptr;
    SHT_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    ctx->err_host = static_cast<int*>(h);
    ctx->err_dev = static_cast<int*>(d);
  }
  return ctx->err_dev;
}

int ctx_take_error(sht_ctx* ctx) {
  std::lock_guard<std::mutex> lk(ctx->err_mu);
  if (!ctx->err_host) return 0;
  volatile int* w = ctx->err_host;
  const int e = *w;
  if (e) *w = 0;
  return e;
}

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

[[noreturn]] void fail(sht_status code, const std::string& msg) { throw Error{code, msg}; }

static void need(bool cond, const char* msg) {
  if (!cond) fail(SHT_ERR_INVALID, msg);
}

static std::vector<int64_t> col_major_strides(const std::vector<int>& n) {
  std::vector<int64_t> s(n.size());
  int64_t acc = 1;
  for (size_t i = 0; i < n.size(); ++i) { s[i] = acc; acc *= n[i]; }
  return s;
}

}  // namespace sht

using namespace sht;

extern "C" {

const char* sht_last_error(void) { return g_last_error.c_str(); }

sht_status sht_init(sht_ctx** out, int device, size_t pool_bytes) {
  return guard([&] {
    need(out != nullptr, "null output handle");
    auto c = std::make_unique<sht_ctx>();
    c->device = device;
    SHT_CUDA(cudaSetDevice(device));
    int sms = 0;
    SHT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    c->num_sms = sms;
    c->pool = std::make_shared<DevicePool>(device, pool_bytes);
    SHT_CUDA(cudaStreamCreateWithFlags(&c->stage_stream, cudaStreamNonBlocking));
    ctx_error_word(c.get());  // the device error word exists before any capture
    *out = c.release();
  });
}

sht_status sht_finalize(sht_ctx* ctx) {
  return guard([&] {
    if (!ctx) return;
    cudaDeviceSynchronize();
    if (ctx->stage_stream) cudaStreamDestroy(ctx->stage_stream);
    if (ctx->err_host) cudaFreeHost(ctx->err_host);
    for (auto& l : ctx->lanes) {
      cudaEventDestroy(l.start);
      cudaEventDestroy(l.done);
      cudaStreamDestroy(l.stream);
    }
    delete ctx;
  });
}

sht_status sht_pool_info(sht_ctx* ctx, size_t* capacity, size_t* free_bytes, size_t* header, size_t* align) {
  return guard([&] {
    need(ctx, "null context");
    if (capacity) *capacity = ctx->pool->capacity();
    if (free_bytes) *free_bytes = ctx->pool->free_bytes();
    if (header) *header = ctx->pool->header();
    if (align) *align = ctx->pool->alignment();
  });
}

sht_status sht_pool_configure(sht_ctx* ctx, size_t header, size_t align) {
  return guard([&] {
    need(ctx, "null context");
    ctx->pool->configure(header, align);
  });
}

sht_status sht_pool_alloc(sht_ctx* ctx, size_t bytes, void** dptr) {
  return guard([&] {
    need(ctx && dptr, "null argument");
    *dptr = ctx->pool->allocate(bytes, nullptr);
  });
}

sht_status sht_pool_realloc(sht_ctx* ctx, void** dptr, size_t bytes, void* stream) {
  return guard([&] {
    need(ctx && dptr, "null argument");
    *dptr = ctx->pool->reallocate(*dptr, bytes, as_stream(stream));
  });
}

sht_status sht_pool_free(sht_ctx* ctx, void* dptr, void* stream) {
  return guard([&] {
    need(ctx, "null context");
    ctx->pool->free(dptr, as_stream(stream));
  });
}

// ---------------------------------------------------------------- Kernel<T>
sht_status sht_kernel_create(sht_ctx* ctx, const char* expr, const int* sa, int na, const int* sb, int nb,
                             const int* sc, int nc, double alpha, double beta, sht_dtype dtype,
                             sht_kernel_type type, sht_kernel** out) {
  return guard([&] {
    need(ctx && expr && out && sa && sb && sc, "null argument");
    need(dtype == SHT_F32 || dtype == SHT_F64, "unknown dtype");
    need(type == SHT_KERNEL_LAPACK || type == SHT_KERNEL_XMM, "Unknown kernel type");
    for (const int* s : {sa, sb, sc}) {
      const int n = s == sa ? na : (s == sb ? nb : nc);
      for (int i = 0; i < n; ++i) {
        need(s[i] > 0, "block extents must be positive");
        if (s[i] > 32767) fail(SHT_ERR_UNSUPPORTED, "block extent above 32767 in one mode");
      }
    }
    auto k = std::make_unique<sht_kernel>();
    k->ctx = ctx;
    k->expr = expr;
    k->sa.assign(sa, sa + na);
    k->sb.assign(sb, sb + nb);
    k->sc.assign(sc, sc + nc);
    parse_einsum(k->expr, na, sa, nb, sb, nc, sc, k->maps);
    k->alpha = alpha;
    k->beta = beta;
    k->dtype = dtype;
    k->type = type;
    k->m = 1; k->n = 1; k->k = 1;
    for (int ax : k->maps.rowA) k->m *= sa[ax];
    for (int ax : k->maps.colB) k->n *= sb[ax];
    for (int ax : k->maps.colA) k->k *= sa[ax];
    k->size_a = std::accumulate(k->sa.begin(), k->sa.end(), (int64_t)1, std::multiplies<int64_t>());
    k->size_b = std::accumulate(k->sb.begin(), k->sb.end(), (int64_t)1, std::multiplies<int64_t>());
    k->size_c = std::accumulate(k->sc.begin(), k->sc.end(), (int64_t)1, std::multiplies<int64_t>());
    need(k->size_a < (1LL << 31) && k->size_b < (1LL << 31) && k->size_c < (1LL << 31), "block above 2^31 elements");
    *out = k.release();
  });
}

sht_status sht_kernel_call(sht_kernel* k, const void* a, const void* b, void* c, int64_t nb_ops, void* stream) {
  return guard([&] {
    need(k, "null kernel");
    stack_call(k, a, b, c, nb_ops, as_stream(stream));
  });
}

sht_status sht_kernel_call_static(sht_kernel* k, const double* a, const double* b, double* c, int64_t nb_ops,
                                  void* stream) {
  return guard([&] {
    need(k, "null kernel");
    stack_call_static(k, a, b, c, nb_ops, as_stream(stream));
  });
}

sht_status sht_kernel_info(sht_kernel* k, char* buf, size_t len) {
  return guard([&] {
    need(k && buf, "null argument");
    auto join = [](const std::vector<int>& v) {
      std::string s;
      for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + std::to_string(v[i]);
      return s;
    };
    std::string o = "Kernel Info\n  Type: " + std::to_string((int)k->type) + "\n  Expression: " + k->expr + "\n";
    o += "Info Tensor In 1\n  Sizes: " + join(k->sa) + "\nmap_row: " + join(k->maps.rowA) + "\nmap_col: " + join(k->maps.colA) + "\n";
    o += "Info Tensor In 2\n  Sizes: " + join(k->sb) + "\nmap_row: " + join(k->maps.rowB) + "\nmap_col: " + join(k->maps.colB) + "\n";
    o += "Info Tensor Out\n  Sizes: " + join(k->sc) + "\nmap_row: " + join(k->maps.rowC) + "\nmap_col: " + join(k->maps.colC) + "\n";
    o += "Device: sm_100a output-stationary tile kernel, " + std::string(k->dtype == SHT_F64 ? "FP64" : "FP32") + "\n";
    std::snprintf(buf, len, "%s", o.c_str());
  });
}

sht_status sht_kernel_destroy(sht_kernel* k) {
  return guard([&] { delete k; });
}

// ---------------------------------------------------------------- Tensor<T,N>
sht_status sht_tensor_create(sht_ctx* ctx, int order, const int* nblk, const int* block_sizes, sht_dtype dtype,
                             sht_tensor** out) {
  return guard([&] {
    need(ctx && nblk && block_sizes && out, "null argument");
    if (order < 2) fail(SHT_ERR_INVALID, "Tensor has to have dimension >= 2");
    if (order > kMaxOrder) fail(SHT_ERR_UNSUPPORTED, "tensor order above 8");
    need(dtype == SHT_F32 || dtype == SHT_F64, "unknown dtype");
    auto t = std::make_unique<sht_tensor>();
    t->keep = ctx->pool;
    t->ctx = ctx;
    t->order = order;
    t->dtype = dtype;
    int pos = 0;
    long double grid = 1;
    std::vector<int> flat;
    for (int d = 0; d < order; ++d) {
      need(nblk[d] > 0, "every mode needs at least one block");
      t->nblk.push_back(nblk[d]);
      t->bs.emplace_back(block_sizes + pos, block_sizes + pos + nblk[d]);
      for (int i = 0; i < nblk[d]; ++i) {
        need(block_sizes[pos + i] > 0, "block sizes must be positive");
        if (block_sizes[pos + i] > 32767) fail(SHT_ERR_UNSUPPORTED, "block extent above 32767 in one mode");
      }
      flat.insert(flat.end(), block_sizes + pos, block_sizes + pos + nblk[d]);
      pos += nblk[d];
      grid *= nblk[d];
    }
    if (grid > 9.0e18L) fail(SHT_ERR_UNSUPPORTED, "block grid above 2^63 blocks");
    t->gstride = col_major_strides(t->nblk);
    t->rows.assign(t->nblk[0], 0);
    cudaStream_t s = ctx->stage_stream;
    t->d_bsizes = PoolBuf(ctx->pool.get(), flat.size() * 4, s);
    SHT_CUDA(cudaMemcpyAsync(t->d_bsizes.ptr, flat.data(), flat.size() * 4, cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaStreamSynchronize(s));
    *out = t.release();
  });
}

sht_status sht_tensor_reserve(sht_tensor* t, int64_t nblocks, const int* idx) {
  return guard([&] {
    need(t, "null tensor");
    need(nblocks >= 0 && (nblocks == 0 || idx), "bad index list");
    std::vector<int64_t> ids(nblocks, 0);
    for (int64_t b = 0; b < nblocks; ++b) {
      for (int d = 0; d < t->order; ++d) {
        const int v = idx[(int64_t)d * nblocks + b];
        if (v < 0 || v >= t->nblk[d]) fail(SHT_ERR_INVALID, "reserve: block index out of range");
        ids[b] += (int64_t)v * t->gstride[d];
      }
    }
    std::sort(ids.begin(), ids.end());
    if (std::adjacent_find(ids.begin(), ids.end()) != ids.end()) fail(SHT_ERR_INVALID, "reserve: duplicate block index");
    for (int64_t id : ids) {
      if (block_size_of(t, id) >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "block above 2^31 elements");
    }
    tensor_set_index(t, std::move(ids), t->ctx->stage_stream);
  });
}

sht_status sht_tensor_reserve_device(sht_tensor* t, int64_t nblocks, const int* idx, void* stream) {
  return guard([&] {
    need(t, "null tensor");
    tensor_reserve_device(t, nblocks, idx, as_stream(stream));
  });
}

sht_status sht_tensor_reserve_all(sht_tensor* t) {
  return guard([&] {
    need(t, "null tensor");
    int64_t n = 1;
    for (int d = 0; d < t->order; ++d) n *= t->nblk[d];
    std::vector<int64_t> ids(n);
    std::iota(ids.begin(), ids.end(), 0);
    for (int64_t id : ids) {
      if (block_size_of(t, id) >= (1LL << 31)) fail(SHT_ERR_UNSUPPORTED, "block above 2^31 elements");
    }
    tensor_set_index(t, std::move(ids), t->ctx->stage_stream);
  });
}

sht_status sht_tensor_info(const sht_tensor* t, int64_t* nblocks, int64_t* nnz) {
  return guard([&] {
    need(t, "null tensor");
    if (nblocks) *nblocks = t->nblocks;
    if (nnz) *nnz = t->nnz;
  });
}

sht_status sht_tensor_get_index(sht_tensor* t, int64_t* ids, int64_t* offsets, int64_t* rows) {
  return guard([&] {
    need(t, "null tensor");
    tensor_sync_host(t, t->ctx->stage_stream);
    if (ids) std::copy(t->ids.begin(), t->ids.end(), ids);
    if (offsets) std::copy(t->offsets.begin(), t->offsets.end(), offsets);
    if (rows) std::copy(t->rows.begin(), t->rows.end(), rows);
  });
}

sht_status sht_tensor_upload(sht_tensor* t, const void* host, int64_t nelem, void* stream) {
  return guard([&] {
    need(t && (host || nelem == 0), "null argument");
    if (nelem != t->nnz) fail(SHT_ERR_SIZE, "upload: element count differs from the tensor's");
    if (nelem == 0) return;
    cudaStream_t s = as_stream(stream);
    tensor_touch(t, s);
    SHT_CUDA(cudaMemcpyAsync(t->d_data.ptr, host, nelem * t->esize(), cudaMemcpyHostToDevice, s));
    SHT_CUDA(cudaStreamSynchronize(s));
  });
}

sht_status sht_tensor_download(sht_tensor* t, void* host, int64_t nelem, void* stream) {
  return guard([&] {
    need(t && (host || nelem == 0), "null argument");
    if (nelem != t->nnz) fail(SHT_ERR_SIZE, "download: element count differs from the tensor's");
    if (nelem == 0) return;
    cudaStream_t s = as_stream(stream);
    tensor_touch(t, s);
    SHT_CUDA(cudaMemcpyAsync(host, t->d_data.ptr, nelem * t->esize(), cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaStreamSynchronize(s));
  });
}

sht_status sht_tensor_device_data(sht_tensor* t, void** dptr) {
  return guard([&] {
    need(t && dptr, "null argument");
    *dptr = t->d_data.ptr;
  });
}

sht_status sht_tensor_norms(sht_tensor* t, sht_norm norm, double* host_out, void* stream) {
  return guard([&] {
    need(t && host_out, "null argument");
    need(norm >= SHT_NORM_FROBENIUS && norm <= SHT_NORM_FROBENIUS_REFCOMPAT, "unknown norm");
    if (t->nblocks == 0) return;
    cudaStream_t s = as_stream(stream);
    PoolBuf d(t->ctx->pool.get(), t->nblocks * 8, s);
    tensor_norms_device(t, norm, d.as<double>(), s);
    SHT_CUDA(cudaMemcpyAsync(host_out, d.ptr, t->nblocks * 8, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaStreamSynchronize(s));
  });
}

sht_status sht_tensor_filter(sht_tensor* t, double eps, sht_norm norm, int compress, void* stream) {
  return guard([&] {
    need(t, "null tensor");
    need(norm >= SHT_NORM_FROBENIUS && norm <= SHT_NORM_FROBENIUS_REFCOMPAT, "unknown norm");
    tensor_filter_device(t, eps, norm, compress, as_stream(stream));
  });
}

sht_status sht_tensor_compress(sht_tensor* t, void* stream) {
  return guard([&] {
    need(t, "null tensor");
    tensor_compress_device(t, as_stream(stream));
  });
}

sht_status sht_tensor_destroy(sht_tensor* t) {
  return guard([&] { delete t; });
}

// ---------------------------------------------------------------- contraction
sht_status sht_plan_create(sht_ctx* ctx, const char* expr, sht_tensor* A, sht_tensor* B, sht_tensor* C,
                           double eps, sht_norm norm, sht_mode mode, void* stream, sht_plan** out) {
  return guard([&] {
    need(ctx && expr && out, "null argument");
    need(mode >= SHT_MODE_PLAIN_FP64 && mode <= SHT_MODE_SPLIT, "unknown mode");
    need(norm >= SHT_NORM_FROBENIUS && norm <= SHT_NORM_FROBENIUS_REFCOMPAT, "unknown norm");
    std::unique_ptr<sht_plan> p(plan_create(ctx, expr, A, B, C, eps, norm, mode, as_stream(stream)));
    prepare_mode(p.get(), as_stream(stream));
    *out = p.release();
  });
}

sht_status sht_plan_execute(sht_plan* p, double alpha, double beta, void* stream) {
  return guard([&] {
    need(p, "null plan");
    if (p->mode == SHT_MODE_SPLIT) raise_pending(p->ctx);
    plan_execute(p, alpha, beta, as_stream(stream));
  });
}

sht_status sht_plan_execute_graph(sht_plan* p, double alpha, double beta, void* stream) {
  return guard([&] {
    need(p, "null plan");
    cudaStream_t s = as_stream(stream);
    if (!s) fail(SHT_ERR_INVALID, "graph replay needs a non-default stream");
    if (p->graph_exec && (p->graph_alpha != alpha || p->graph_beta != beta)) {
      cudaGraphExecDestroy(p->graph_exec);
      cudaGraphDestroy(p->graph);
      p->graph_exec = nullptr;
      p->graph = nullptr;
    }
    if (!p->graph_exec) {
      SHT_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        plan_execute(p, alpha, beta, s);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      SHT_CUDA(cudaStreamEndCapture(s, &p->graph));
      SHT_CUDA(cudaGraphInstantiate(&p->graph_exec, p->graph, 0));
      p->graph_alpha = alpha;
      p->graph_beta = beta;
    }
    SHT_CUDA(cudaGraphLaunch(p->graph_exec, s));
  });
}

sht_status sht_plan_report(sht_plan* p, sht_contract_report* rep) {
  return guard([&] {
    need(p && rep, "null argument");
    std::memset(rep, 0, sizeof(*rep));
    rep->npairs = p->npairs;
    rep->nblocks_c = p->C->nblocks;
    rep->nnz_c = p->C->nnz;
    rep->nwork = p->mode == SHT_MODE_BATCHED_FP64 ? p->bwork : p->nwork;
    rep->flops = plan_flops(p, p->ctx->stage_stream);  // waits for the count's own event
    rep->plan_ms = p->plan_ms;
    rep->exec_ms = p->exec_ms;
    rep->slices = p->split_slices;
  });
}

sht_status sht_plan_pairs(sht_plan* p, int64_t* triples, int64_t capacity) {
  return guard([&] {
    need(p && (triples || capacity == 0), "null argument");
    if (capacity < p->npairs) fail(SHT_ERR_SIZE, "pair buffer too small");
    const long long np = p->npairs;
    if (np == 0) return;
    cudaStream_t s = p->ctx->stage_stream;
    std::vector<int> ha(np), hb(np), ps(p->ncblk + 1);
    SHT_CUDA(cudaMemcpyAsync(ha.data(), p->d_pair_a.ptr, np * 4, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaMemcpyAsync(hb.data(), p->d_pair_b.ptr, np * 4, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaMemcpyAsync(ps.data(), p->d_pstart.ptr, (p->ncblk + 1) * 4, cudaMemcpyDeviceToHost, s));
    SHT_CUDA(cudaStreamSynchronize(s));
    tensor_sync_host(p->C, s);
    for (long long c = 0; c < p->ncblk; ++c)
      for (int i = ps[c]; i < ps[c + 1]; ++i) {
        triples[3 * i] = p->C->ids[c];
        triples[3 * i + 1] = p->A->ids[ha[i]];
        triples[3 * i + 2] = p->B->ids[hb[i]];
      }
  });
}

sht_status sht_plan_destroy(sht_plan* p) {
  return guard([&] { delete p; });
}

sht_status sht_contract(sht_ctx* ctx, const char* expr, double alpha, sht_tensor* A, sht_tensor* B, double beta,
                        sht_tensor* C, double eps, sht_norm norm, sht_mode mode, void* stream,
                        sht_contract_report* rep) {
  return guard([&] {
    need(ctx && expr, "null argument");
    need(mode >= SHT_MODE_PLAIN_FP64 && mode <= SHT_MODE_SPLIT, "unknown mode");
    need(norm >= SHT_NORM_FROBENIUS && norm <= SHT_NORM_FROBENIUS_REFCOMPAT, "unknown norm");
    cudaStream_t s = as_stream(stream);
    std::unique_ptr<sht_plan> p;
    if (mode == SHT_MODE_SPLIT) raise_pending(ctx);
    if (mode == SHT_MODE_SPLIT) {
      p.reset(plan_init(ctx, expr, A, B, C, eps, norm, mode, s));
      contract_split(p.get(), alpha, beta, s);
    } else if (mode == SHT_MODE_BATCHED_FP64) {
      p.reset(plan_init(ctx, expr, A, B, C, eps, norm, mode, s));
      contract_batched(p.get(), alpha, beta, s);
    } else {
      p.reset(plan_create(ctx, expr, A, B, C, eps, norm, mode, s));
      prepare_mode(p.get(), s);
      plan_execute(p.get(), alpha, beta, s);
    }
    if (rep) {
      std::memset(rep, 0, sizeof(*rep));
      rep->npairs = p->npairs;
      rep->nblocks_c = C->nblocks;
      rep->nnz_c = C->nnz;
      rep->nwork = p->mode == SHT_MODE_BATCHED_FP64 ? p->bwork : p->nwork;
      rep->flops = plan_flops(p.get(), s);
      rep->plan_ms = p->plan_ms;
      rep->slices = p->split_slices;
    }
    // the plan's buffers return to the pool stream-ordered after the launch
  });
}

sht_status sht_tensor_compare(sht_tensor* X, sht_tensor* Ref, double* max_abs, double* rel_fro, void* stream) {
  return guard([&] {
    need(X && Ref, "null tensor");
    tensor_compare_device(X, Ref, max_abs, rel_fro, nullptr, as_stream(stream));
  });
}

sht_status sht_tensor_bitdiff(sht_tensor* X, sht_tensor* Ref, int64_t* ndiff, void* stream) {
  return guard([&] {
    need(X && Ref && ndiff, "null argument");
    long long n = 0;
    tensor_compare_device(X, Ref, nullptr, nullptr, &n, as_stream(stream));
    *ndiff = n;
  });
}

sht_status sht_autotune(sht_plan* p, const char* cache_file, void* stream) {
  return guard([&] {
    need(p, "null plan");
    if (p->mode != SHT_MODE_BATCHED_FP64) fail(SHT_ERR_STATE, "autotune applies to batched plans");
    autotune(p, cache_file, as_stream(stream));
  });
}

sht_status sht_set_split_slices(sht_ctx* ctx, int slices) {
  return guard([&] {
    need(ctx, "null context");
    if (slices < 1 || slices > 8) fail(SHT_ERR_INVALID, "split slices must be 1..8");
    ctx->split_slices = slices;
  });
}

sht_status sht_set_wait_limit(sht_ctx* ctx, int64_t polls) {
  return guard([&] {
    need(ctx, "null context");
    need(polls >= 0, "wait limit must be >= 0");
    ctx->wait_limit = polls;
  });
}

sht_status sht_stream_sync(sht_ctx* ctx, void* stream) {
  return guard([&] {
    need(ctx, "null context");
    SHT_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (const int e = ctx_take_error(ctx))
      fail((sht_status)e, "a split-precision launch on this context failed: a bounded wait on the tensor cores "
                          "expired (its result is undefined)");
  });
}

sht_status sht_measure_peak(sht_ctx* ctx, int which, double* value) {
  return guard([&] {
    need(ctx && value, "null argument");
    if (which == 0)
      *value = measure_fp64_tflops(ctx);
    else if (which == 1)
      *value = measure_int8_tops(ctx);
    else if (which == 2)
      *value = measure_dmma_tflops(ctx);
    else if (which == 3)
      *value = measure_split_pipe_tops(ctx);
    else
      fail(SHT_ERR_UNSUPPORTED, "unknown peak");
  });
}

}  // extern "C"
