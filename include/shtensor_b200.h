/*
 * shtensor_b200.h -- C ABI of the B200 (sm_100a) block-sparse tensor contraction library.
 *
 * Drop-in boundary for shtensor's single-rank contraction path.  Every entry point returns
 * an sht_status (0 = success) and never throws; the message of the last failure on the
 * calling thread is returned by sht_last_error().  Handles are opaque.  Device memory for
 * tensors, plans and scratch comes from the context's device pool.  A context and the
 * handles made from it are not thread-safe: one host thread drives a context at a time.
 * After sht_finalize the only valid calls on tensors and plans made from the context are
 * their destroy calls; the device arena is released when the last of them is destroyed.
 * Stream arguments are cudaStream_t values passed as void* (NULL = the legacy default stream).
 *
 * Reference interfaces each entry point replaces (paths relative to the shtensor root):
 *   sht_init / sht_finalize      Context(MPI_Comm, int64_t pool_bytes)   src/Shmem/Context.h:30
 *   sht_pool_*                   MemoryPool::{allocate,reallocate,free,get_free_mem}
 *                                src/Shmem/MemoryPool.h:51-96,126-354
 *   sht_kernel_create            Kernel<T>::Kernel(expr, sizes_in1, sizes_in2, sizes_out,
 *                                alpha, beta, KernelType)               src/Kernel/Kernel.h:69-86
 *   sht_kernel_call              Kernel<T>::call(T* a, T* b, T* c, int64_t nb_ops)
 *                                                                       src/Kernel/Kernel.h:88-91
 *   sht_kernel_info              KernelBase::get_info()                 src/Kernel/Kernel.cpp:29-32
 *   sht_tensor_create            Tensor<T,N>(ctx, VArray<N> block_sizes) src/Tensor/Tensor.h:27-32
 *   sht_tensor_reserve(_all)     BaseTensor::reserve / reserve_all      src/Tensor/BaseTensor.cpp:97-251
 *   sht_tensor_reserve_device    BaseTensor::reserve, index lists on the device  BaseTensor.cpp:117-251
 *   sht_tensor_get_index         BaseTensor::get_sparse_info()          src/Tensor/BaseTensor.h:51
 *   sht_tensor_upload/download   block data access (get_local_block, iterators)
 *                                                                       src/Tensor/Tensor.h:38-52,75-258
 *   sht_tensor_norms             BlockSpan::get_norm                    src/Basics/BlockSpan.h:140-164
 *   sht_tensor_filter            Tensor<T,N>::filter(eps, norm, compress) src/Tensor/Tensor.h:337-363
 *   sht_tensor_compress          BaseTensor::compress                   src/Tensor/BaseTensor.cpp:253-354
 *   sht_contract, sht_plan_*     the block-sparse contract the reference lacks
 *                                (src/Tensor/Tensor.cpp is empty; test/test_contract.cpp:5-23)
 *   sht_server_*                 serving loop (no reference counterpart)
 */
#ifndef SHTENSOR_B200_H
#define SHTENSOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SHT_OK = 0,
  SHT_ERR_INVALID = 1,      /* bad argument or handle */
  SHT_ERR_PARSE = 2,        /* einsum expression rejected */
  SHT_ERR_SIZE = 3,         /* size / block-size mismatch */
  SHT_ERR_OOM = 4,          /* device pool exhausted */
  SHT_ERR_CUDA = 5,         /* CUDA runtime error */
  SHT_ERR_TIMEOUT = 6,      /* a bounded device or host wait expired */
  SHT_ERR_UNSUPPORTED = 7,  /* valid request outside the implemented envelope */
  SHT_ERR_STATE = 8         /* operation not valid in the handle's current state */
} sht_status;

typedef enum { SHT_F32 = 0, SHT_F64 = 1 } sht_dtype;                 /* FloatType, Definitions.h:44-48 */
typedef enum { SHT_KERNEL_LAPACK = 0, SHT_KERNEL_XMM = 1 } sht_kernel_type; /* KernelType, KernelDefinitions.h:11-15 */
typedef enum {
  SHT_NORM_FROBENIUS = 0,            /* sqrt(sum v^2) in a fixed chunked order (bit-reproducible) */
  SHT_NORM_MAXABS = 1,
  SHT_NORM_FROBENIUS_REFCOMPAT = 2   /* the reference's int-accumulator evaluation */
} sht_norm;
typedef enum {
  SHT_MODE_PLAIN_FP64 = 0,   /* output-stationary FP64 DFMA tiles, one launch, bit-exact order */
  SHT_MODE_BATCHED_FP64 = 1, /* persistent kernel over a size-class work list, tuned tiles */
  SHT_MODE_SPLIT = 2         /* split-precision (Ozaki) INT8 tensor-core slices, FP64 reassembly */
} sht_mode;

typedef struct sht_ctx sht_ctx;
typedef struct sht_kernel sht_kernel;
typedef struct sht_tensor sht_tensor;
typedef struct sht_plan sht_plan;

typedef struct {
  int64_t npairs;       /* surviving block pairs */
  int64_t nblocks_c;    /* C blocks after the contraction */
  int64_t nnz_c;        /* C elements after the contraction */
  int64_t nwork;        /* tiles launched */
  double flops;         /* sum over pairs of 2*m*n*k */
  double plan_ms;       /* host-timed plan phase (matching, pattern, work list) */
  double exec_ms;       /* device-timed execute phase (0 unless timing was requested) */
  int32_t slices;       /* split mode: INT8 slices per operand (0 otherwise) */
  int32_t reserved;
} sht_contract_report;

/* ---- context and device pool (Context / MemoryPool) ---- */
sht_status sht_init(sht_ctx** ctx, int device, size_t pool_bytes);
sht_status sht_finalize(sht_ctx* ctx);
const char* sht_last_error(void);
sht_status sht_pool_info(sht_ctx* ctx, size_t* capacity, size_t* free_bytes, size_t* chunk_header,
                         size_t* alignment);
sht_status sht_pool_alloc(sht_ctx* ctx, size_t bytes, void** dptr);
sht_status sht_pool_realloc(sht_ctx* ctx, void** dptr, size_t bytes, void* stream);
sht_status sht_pool_free(sht_ctx* ctx, void* dptr, void* stream);
/* accounting parameters (chunk header bytes, alignment); only on an empty pool */
sht_status sht_pool_configure(sht_ctx* ctx, size_t chunk_header, size_t alignment);

/* ---- per-block stack kernel (Kernel<T>) ---- */
sht_status sht_kernel_create(sht_ctx* ctx, const char* expr, const int* sizes_a, int na,
                             const int* sizes_b, int nb, const int* sizes_c, int nc, double alpha,
                             double beta, sht_dtype dtype, sht_kernel_type type, sht_kernel** out);
/* a, b, c: nb_ops contiguous same-shape blocks each, column-major.  Device pointers run in
 * place on `stream`; host pointers are staged through the pool and the call returns after
 * the result is back in host memory. */
sht_status sht_kernel_call(sht_kernel* k, const void* a, const void* b, void* c, int64_t nb_ops,
                           void* stream);
/* Allocation-free Kernel<double>::call (no counterpart in the reference).  For callers that
 * cannot call cudaMalloc -- code inside someone else's CUDA-graph capture, plugin hosts that
 * only hand over pre-registered buffers, processes whose device memory another runtime has
 * reserved.  a, b, c are device pointers (the caller passes inputs and outputs); the result
 * bits equal sht_kernel_call's.  Its only scratch is a static 32 MiB device array that every
 * GPU loading the library keeps until exit: a stack needing more (nb_ops * (m_pad + n_pad) *
 * K4 * 8 bytes, m_pad/n_pad rounded up to even, K4 to a multiple of 4) is rejected with
 * SHT_ERR_SIZE.  The first call on a device looks the array up (cudaGetSymbolAddress) and,
 * under lazy module loading, loads the module (committing the array): it should come before
 * any stream capture.  Calls share the array: calls that overlap on the
 * GPU race. */
sht_status sht_kernel_call_static(sht_kernel* k, const double* a, const double* b, double* c, int64_t nb_ops,
                                  void* stream);
sht_status sht_kernel_info(sht_kernel* k, char* buf, size_t len);
sht_status sht_kernel_destroy(sht_kernel* k);

/* ---- block-sparse tensors (Tensor<T,N>) ---- */
/* nblk[d] blocks in mode d; block_sizes holds the sizes of mode 0, then mode 1, ... */
sht_status sht_tensor_create(sht_ctx* ctx, int order, const int* nblk, const int* block_sizes,
                             sht_dtype dtype, sht_tensor** out);
/* idx is mode-major like VArray<N>: idx[d*nblocks + b]; zero-fills the data */
sht_status sht_tensor_reserve(sht_tensor* t, int64_t nblocks, const int* idx);
/* The same as sht_tensor_reserve (BaseTensor::reserve, src/Tensor/BaseTensor.cpp:117-251) with
 * the index lists already in device memory (idx[d * nblocks + b], int32): the ids, their sort,
 * the range / duplicate / size checks and the offsets are built on the GPU, with one read-back
 * of the checks and the element count; blocks start zero-filled.  Returns after the build and
 * the zero fill are done. */
sht_status sht_tensor_reserve_device(sht_tensor* t, int64_t nblocks, const int* idx, void* stream);
sht_status sht_tensor_reserve_all(sht_tensor* t);
sht_status sht_tensor_info(const sht_tensor* t, int64_t* nblocks, int64_t* nnz);
/* host copies of the sparse index: sorted rolled ids, element offsets, rows (nblk[0]) */
sht_status sht_tensor_get_index(sht_tensor* t, int64_t* ids, int64_t* offsets, int64_t* rows);
sht_status sht_tensor_upload(sht_tensor* t, const void* host, int64_t nelem, void* stream);
sht_status sht_tensor_download(sht_tensor* t, void* host, int64_t nelem, void* stream);
sht_status sht_tensor_device_data(sht_tensor* t, void** dptr);
sht_status sht_tensor_norms(sht_tensor* t, sht_norm norm, double* host_out, void* stream);
sht_status sht_tensor_filter(sht_tensor* t, double eps, sht_norm norm, int compress, void* stream);
sht_status sht_tensor_compress(sht_tensor* t, void* stream);
sht_status sht_tensor_destroy(sht_tensor* t);

/* ---- block-sparse contraction: C = beta*C + alpha * contract(expr, A, B) ---- */
/* pairs with norm(a)*norm(b) < screen_eps are dropped (screen_eps <= 0 keeps all) */
sht_status sht_contract(sht_ctx* ctx, const char* expr, double alpha, sht_tensor* A,
                        sht_tensor* B, double beta, sht_tensor* C, double screen_eps,
                        sht_norm norm, sht_mode mode, void* stream, sht_contract_report* rep);
/* plan = matching + C pattern (C is re-reserved to the result pattern) + work list */
sht_status sht_plan_create(sht_ctx* ctx, const char* expr, sht_tensor* A, sht_tensor* B,
                           sht_tensor* C, double screen_eps, sht_norm norm, sht_mode mode,
                           void* stream, sht_plan** out);
sht_status sht_plan_execute(sht_plan* p, double alpha, double beta, void* stream);
/* captures sht_plan_execute into a CUDA graph on first use and replays it after */
sht_status sht_plan_execute_graph(sht_plan* p, double alpha, double beta, void* stream);
sht_status sht_plan_report(sht_plan* p, sht_contract_report* rep);
/* pair list as (idC, idA, idB) triples by block id, in execution order */
sht_status sht_plan_pairs(sht_plan* p, int64_t* triples, int64_t capacity);
sht_status sht_plan_destroy(sht_plan* p);

/* ---- split-precision error report (max abs and relative Frobenius vs an FP64 result) ---- */
sht_status sht_tensor_compare(sht_tensor* X, sht_tensor* Ref, double* max_abs, double* rel_fro,
                              void* stream);
/* number of elements whose bit patterns differ between X and Ref (same block pattern): 0 means
 * bit-identical results, signed zeros included (no reference counterpart; a parity check) */
sht_status sht_tensor_bitdiff(sht_tensor* X, sht_tensor* Ref, int64_t* ndiff, void* stream);

/* ---- autotuner ---- */
/* sweeps tile shapes per (m,n,k) size class of the plan and stores the choice; file may be NULL */
sht_status sht_autotune(sht_plan* p, const char* cache_file, void* stream);

/* INT8 slices per operand used by SHT_MODE_SPLIT plans made after the call (1..8, default 7) */
sht_status sht_set_split_slices(sht_ctx* ctx, int slices);

/* Split mode is asynchronous like the FP64 forms: sht_contract and sht_plan_execute return once
 * the work is queued on `stream`.  The split kernel's pipeline waits are bounded; a wait that
 * runs out (a hardware or scheduling fault) leaves C undefined and records SHT_ERR_TIMEOUT on
 * the context.  The next split call on the context reports it (without queueing its own work),
 * and sht_stream_sync reports it after the stream's work is done.  Non-finite inputs are not an
 * error: such an execute is computed by the FP64 tiles, with IEEE propagation as in the FP64
 * forms. */
/* waits for the work queued on `stream`, then returns (and clears) the first failure recorded
 * by this context's device work, if any */
sht_status sht_stream_sync(sht_ctx* ctx, void* stream);
/* diagnostic: polls of one device pipeline wait of the split kernel before the launch gives up
 * (0 = the default, about a second); waits for work already issued keep their own bound */
sht_status sht_set_wait_limit(sht_ctx* ctx, int64_t polls);

/* ---- diagnostics ---- */
/* which = 0: FP64 FMA peak of this GPU in TFLOP/s (the FP64 kernels' roofline denominator);
 * which = 1: dense INT8 tensor-core (tcgen05 kind::i8) peak in TOPS (the split kernel's);
 * which = 2: FP64 tensor-core (mma.sync m8n8k4) peak in TFLOP/s (the batched kernel's);
 * which = 3: the split kernel's operand pipeline alone (stage bulk copies from L2 plus the
 *            seven-MMA triangle per k-step, 7 slices) in INT8 TOPS: the rate the split kernel
 *            can reach once its epilogue is hidden */
sht_status sht_measure_peak(sht_ctx* ctx, int which, double* value);

/* ---- serving loop (no reference counterpart: shtensor has no request loop) ----
 * A server owns one host thread and its own CUDA streams.  Requests are block-sparse
 * contractions over device-resident tensors, computed in the server's form: the batched FP64
 * form (the result bits equal sht_contract with SHT_MODE_BATCHED_FP64 or SHT_MODE_PLAIN_FP64
 * run alone), or the split-precision form (the result bits equal sht_contract with
 * SHT_MODE_SPLIT run alone; a request whose operands hold a non-finite value or an exponent
 * outside the split kernel's scale-folded range is served in the batched FP64 form).
 * Continuous batching: a request that arrives while others run is planned at once (by one of
 * several planner threads) if a slot is free and the pool has room, and joins the next
 * persistent launch together with every other planned request; up to two launches are
 * queued, so the next one starts as soon as the running one drains.  Admission: at most max_active requests planned or running, and a
 * request is planned only if the pool keeps reserve_bytes free after its estimated scratch;
 * a plan that runs out of pool memory while other requests hold memory is retried after the
 * next completion (a deferral).  Requests that write a tensor another active or earlier
 * queued request reads or writes wait for it, so each tensor sees its requests in order.
 * Threads: while a server runs, the context's owner thread may create, reserve, upload,
 * download and destroy tensors and submit/poll/wait; it must not destroy a tensor that an
 * unfinished request names, nor call sht_contract, sht_plan_* or sht_autotune on the
 * context.  Latencies are host steady-clock times, submit to observed completion. */
typedef struct sht_server sht_server;

typedef struct {
  int max_active;        /* requests planned or running at once (0 = 64) */
  int max_batch;         /* requests fused into one launch (0 = 32) */
  size_t reserve_bytes;  /* pool bytes that admission leaves free (0 = none) */
  int planners;          /* planner threads, each with its own stream (0 = 8) */
  int ctas_per_sm;       /* persistent CTAs per SM of a batched serving launch (0 = the most
                            that fit minus one, leaving room for planning kernels) */
  int mode;              /* 0 or SHT_MODE_BATCHED_FP64: batched FP64; SHT_MODE_SPLIT: split
                            precision.  One launch holds requests of one form (and, in split
                            form, one slice count and reassembly instance). */
} sht_server_config;

typedef struct {
  sht_status status;     /* the request's own result */
  int64_t npairs;        /* block products after screening */
  double flops;          /* 2*m*n*k summed over the pairs */
  double queue_ms;       /* submit -> planning starts */
  double plan_ms;        /* planning (matching, C pattern, work list, matrix-form layout) */
  double run_ms;         /* launch -> completion observed */
  double gpu_ms;         /* device time of its launch: the exec stream reaching it -> done */
  double latency_ms;     /* submit -> completion observed */
  int64_t batch;         /* id of the launch that computed it (-1 if it never ran) */
  int form;              /* the form that computed it (an sht_mode value) */
  int batch_size;        /* requests in that launch */
  int deferrals;         /* admissions put off for pool memory */
} sht_request_report;

typedef struct {
  int64_t submitted, completed, failed, batches, deferrals;
  int max_active_seen;   /* most requests planned or running at once */
  double mean_batch;     /* requests per launch */
  double p50_ms, p99_ms, max_ms;  /* latency of the completed requests since the last reset */
  double flops;          /* algorithmic flops of the completed requests */
  double span_s;         /* first submit -> last completion */
  double gflops;         /* flops / span_s / 1e9 */
} sht_server_stats;

sht_status sht_server_create(sht_ctx* ctx, const sht_server_config* cfg, sht_server** out);
/* queue C = beta*C + alpha*contract(expr, A, B) with screening eps (0 = none) */
sht_status sht_server_submit(sht_server* srv, const char* expr, double alpha, sht_tensor* A, sht_tensor* B,
                             double beta, sht_tensor* C, double eps, sht_norm norm, int64_t* request_id);
/* *state: 0 queued or running, 1 finished (the report is ready) */
sht_status sht_server_poll(sht_server* srv, int64_t request_id, int* state);
/* wait up to timeout_s (< 0: no limit); returns the request's status (SHT_ERR_TIMEOUT if it
 * is still pending) and forgets the request once it has finished */
sht_status sht_server_wait(sht_server* srv, int64_t request_id, double timeout_s, sht_request_report* rep);
sht_status sht_server_get_stats(sht_server* srv, sht_server_stats* out);
sht_status sht_server_reset_stats(sht_server* srv);
/* finishes every submitted request, then stops the thread and frees the server */
sht_status sht_server_destroy(sht_server* srv);

#ifdef __cplusplus
}
#endif

#endif
