// sht_internal.h -- internal types shared by the host runtime and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/shtensor_b200.h"

namespace sht {

constexpr int kMaxOrder = 8;

// ---------------------------------------------------------------------------------------
// errors: every C entry point converts a thrown Error into its status + thread-local text
// ---------------------------------------------------------------------------------------
struct Error {
  sht_status code;
  std::string msg;
};
[[noreturn]] void fail(sht_status code, const std::string& msg);
void set_last_error(const std::string& msg);

// runs f, turning whatever it throws into a status and the calling thread's message
template <class F>
sht_status guard(F&& f) {
  try {
    f();
    return SHT_OK;
  } catch (const Error& e) {
    set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host out of memory");
    return SHT_ERR_OOM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SHT_ERR_INVALID;
  }
}

#define SHT_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      ::sht::fail(SHT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------------------
// Device pool.  One cudaMalloc arena, first-fit chunk list kept on the host, with the
// accounting of the reference's MemoryPool (src/Shmem/MemoryPool.h:126-354): each chunk
// costs `header` bytes, data sizes are rounded up to `align`, frees coalesce both sides.
// Frees are stream-ordered: a freed chunk carries the event recorded on the freeing stream
// and the next allocation from it makes its own stream wait on that event.  Every piece of
// a split or merged free chunk keeps the events of the memory it covers (events are shared
// and recycled when the last chunk holding them is handed out), so memory freed on one
// stream is never reused on another before the freeing stream's work is done.
// ---------------------------------------------------------------------------------------
class DevicePool {
 public:
  DevicePool(int device, size_t bytes);
  ~DevicePool();
  void* allocate(size_t bytes, cudaStream_t stream);
  void free(void* p, cudaStream_t stream);
  void* reallocate(void* p, size_t bytes, cudaStream_t stream);
  size_t size_of(void* p) const;
  size_t capacity() const { return cap_; }
  size_t free_bytes() const {
    std::lock_guard<std::recursive_mutex> lk(mu_);
    return free_;
  }
  size_t header() const { return header_; }
  size_t alignment() const { return align_; }
  void configure(size_t header, size_t align);
  bool owns(const void* p) const;

 private:
  // an event recorded at a free, with the stream it was recorded on (an allocation on that
  // same stream is ordered after the free already and needs no wait)
  struct PoolEvent {
    cudaEvent_t event;
    cudaStream_t stream;
  };
  using EventRef = std::shared_ptr<PoolEvent>;
  struct Chunk {
    size_t size = 0;  // data bytes (header excluded)
    bool free = true;
    std::vector<EventRef> pending;
  };
  // chunk start offset (its header starts here; data at off + header) -> chunk
  std::map<size_t, Chunk> chunks_;
  char* base_ = nullptr;
  size_t cap_ = 0, free_ = 0, header_ = 256, align_ = 256;
  std::vector<cudaEvent_t> spare_events_;
  // the serving loop allocates from its own thread while callers create tensors
  mutable std::recursive_mutex mu_;
  EventRef record_event(cudaStream_t stream);
  static void prune(std::vector<EventRef>& v);
  void wait_pending(const Chunk& c, cudaStream_t stream);
  std::map<size_t, Chunk>::iterator find_data(const void* p);
};

// RAII pool buffer
struct PoolBuf {
  DevicePool* pool = nullptr;
  void* ptr = nullptr;
  size_t bytes = 0;
  PoolBuf() = default;
  PoolBuf(DevicePool* p, size_t b, cudaStream_t s) : pool(p), bytes(b), stream_(s) {
    ptr = b ? p->allocate(b, s) : nullptr;
  }
  PoolBuf(const PoolBuf&) = delete;
  PoolBuf& operator=(const PoolBuf&) = delete;
  PoolBuf(PoolBuf&& o) noexcept { *this = std::move(o); }
  PoolBuf& operator=(PoolBuf&& o) noexcept {
    if (this != &o) {
      release();
      pool = o.pool; ptr = o.ptr; bytes = o.bytes;
      stream_.store(o.stream_.load(std::memory_order_relaxed), std::memory_order_relaxed);
      o.ptr = nullptr; o.bytes = 0;
    }
    return *this;
  }
  ~PoolBuf() { release(); }
  void release() noexcept {
    // runs in destructors: a failing free (lost CUDA context) leaks instead of terminating
    try {
      if (ptr && pool) pool->free(ptr, stream_.load(std::memory_order_relaxed));
    } catch (...) {
    }
    ptr = nullptr;
    bytes = 0;
  }
  template <typename T> T* as() const { return static_cast<T*>(ptr); }
  // the stream whose work must finish before the memory is reused (atomic: the serving
  // loop's planner threads record their streams on shared input tensors concurrently)
  void use_on(cudaStream_t s) { stream_.store(s, std::memory_order_relaxed); }

 private:
  std::atomic<cudaStream_t> stream_{nullptr};
};

}  // namespace sht

// ---------------------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------------------
struct sht_ctx {
  int device = 0;
  int num_sms = 148;
  // shared with every tensor and plan: the arena outlives sht_finalize until the last
  // handle made from the context is destroyed
  std::shared_ptr<sht::DevicePool> pool;
  cudaStream_t stage_stream = nullptr;  // host-staging copies
  // non-blocking streams, each with two events, lent to contractions that plan on a second
  // stream while the caller's stream slices the operands (created on demand, kept)
  struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, done = nullptr;
  };
  std::mutex lanes_mu;
  std::vector<Lane> lanes;
  std::map<std::string, int> tuned;     // autotuner choices: size-class key -> tile id
  int split_slices = 0;                 // INT8 slices per operand in split mode (0 = default)
  long long wait_limit = 0;             // polls of a device pipeline wait (0 = default)
  // Error word of device work (a bounded wait of the split kernel that ran out): host memory
  // mapped into the device, written by a kernel only on failure and read by the host without
  // a synchronization; sticky until reported (created on first use)
  int* err_host = nullptr;
  int* err_dev = nullptr;
  std::mutex err_mu;
};

// Parsed einsum: matrix dimension <-> tensor modes (local positions)
struct ShtMaps {
  std::vector<int> rowA, colA, rowB, colB, rowC, colC;
};

struct sht_kernel {
  sht_ctx* ctx = nullptr;
  std::string expr;
  std::vector<int> sa, sb, sc;
  ShtMaps maps;
  double alpha = 1.0, beta = 0.0;
  sht_dtype dtype = SHT_F64;
  sht_kernel_type type = SHT_KERNEL_XMM;
  int64_t m = 0, n = 0, k = 0, size_a = 0, size_b = 0, size_c = 0;
};

struct sht_tensor {
  std::shared_ptr<sht::DevicePool> keep;  // declared first: released after the buffers below
  sht_ctx* ctx = nullptr;
  int order = 0;
  sht_dtype dtype = SHT_F64;
  std::vector<std::vector<int>> bs;
  std::vector<int> nblk;
  std::vector<int64_t> gstride;
  // host index (authoritative unless host_stale)
  std::vector<int64_t> ids, offsets, rows;
  bool host_stale = false;
  bool has_marked = false;  // the host index holds filtered (negative) ids
  // per-block extents and block-grid coordinates (nblocks x order each) of the host index,
  // computed on first use after the host index changes (tensor_host_dims, tensor_host_coords)
  std::vector<int> hdims, hcoords;
  bool hdims_valid = false;
  std::mutex hmu;  // the serving loop's planner threads share input tensors
  int64_t nblocks = 0, nnz = 0;
  // device arrays
  sht::PoolBuf d_bsizes;   // int32, concatenated per mode
  sht::PoolBuf d_bstart;   // int32[order], start of each mode in d_bsizes
  sht::PoolBuf d_ids;      // int64[nblocks]
  sht::PoolBuf d_offsets;  // int64[nblocks]
  sht::PoolBuf d_dims;     // int32[nblocks*order]
  sht::PoolBuf d_data;     // elements
  size_t esize() const { return dtype == SHT_F64 ? 8 : 4; }
};

namespace sht {

// einsum parsing (einsum.cpp)
void parse_einsum(const std::string& expr, int nA, const int* sA, int nB, const int* sB, int nC,
                  const int* sC, ShtMaps& m);

// tensors (tensor.cu)
void tensor_set_index(sht_tensor* t, std::vector<int64_t>&& ids, cudaStream_t s);
// reserve from mode-major index lists in device memory (ids, sort, checks and offsets on the GPU)
void tensor_reserve_device(sht_tensor* t, long long n, const int* d_idx, cudaStream_t s);
void tensor_sync_host(sht_tensor* t, cudaStream_t s);
// per-block extents of the host index, nblocks x order (the host index must be current)
const int* tensor_host_dims(sht_tensor* t);
const int* tensor_host_coords(sht_tensor* t);
void tensor_upload_index(sht_tensor* t, cudaStream_t s);
void tensor_norms_device(sht_tensor* t, sht_norm norm, double* d_out, cudaStream_t s);
// Record that `s` uses the tensor's device buffers: when they are freed, reuse of the memory
// is ordered after the work queued on `s` so far.
void tensor_touch(sht_tensor* t, cudaStream_t s);
int64_t block_size_of(const sht_tensor* t, int64_t id);
void tensor_compare_device(sht_tensor* X, sht_tensor* R, double* max_abs, double* rel_fro, long long* ndiff,
                           cudaStream_t s);

// stack kernel (stack.cu)
void stack_call(sht_kernel* k, const void* a, const void* b, void* c, int64_t nb_ops,
                cudaStream_t s);

// the context's device error word (host-mapped; created on first use)
volatile int* ctx_error_word(sht_ctx* ctx);
// the first device-side failure recorded since the last call (0 if none); clears it
int ctx_take_error(sht_ctx* ctx);

// timing helpers
double now_ms();
// Phase trace of the host runtime, printed to stderr when SHT_TRACE=1 (the stream is
// synchronized at each point so the times are device-inclusive).
void trace(const char* what, cudaStream_t s);

}  // namespace sht
