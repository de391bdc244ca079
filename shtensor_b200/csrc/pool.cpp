// pool.cpp -- one-GPU device memory pool replacing shtensor's MPI-RMA MemoryPool.
//
// The reference allocates one MPI window (src/Shmem/MemoryPool.cpp:68) and manages it with a
// first-fit list of inline chunk headers (src/Shmem/MemoryPool.h:126-354).  Here the arena is
// one cudaMalloc and the chunk list lives on the host (device memory holds no headers), while
// the free-byte accounting keeps the reference's rules so its test (test/test_mempool.cpp)
// carries over: a chunk costs `header_` bytes, data is rounded up to `align_`, a split that
// would leave no room for a header keeps the whole chunk, frees coalesce right then left.
#include <algorithm>

#include "sht_internal.h"

namespace sht {

static size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

DevicePool::DevicePool(int device, size_t bytes) {
  SHT_CUDA(cudaSetDevice(device));
  cap_ = bytes;
  if (bytes < header_ + align_) fail(SHT_ERR_INVALID, "pool smaller than one chunk");
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(SHT_ERR_OOM, std::string("cudaMalloc of the device pool failed: ") + cudaGetErrorString(e));
  }
  base_ = static_cast<char*>(p);
  Chunk c;
  c.size = cap_ - header_;
  chunks_[0] = c;
  free_ = cap_ - header_;
}

DevicePool::~DevicePool() {
  chunks_.clear();  // returns every pending event to spare_events_
  for (cudaEvent_t ev : spare_events_) cudaEventDestroy(ev);
  if (base_) cudaFree(base_);
}

void DevicePool::configure(size_t header, size_t align) {
  std::lock_guard<std::recursive_mutex> lk(mu_);
  if (chunks_.size() != 1 || !chunks_.begin()->second.free)
    fail(SHT_ERR_STATE, "pool_configure needs an empty pool");
  if (align == 0 || (align & (align - 1))) fail(SHT_ERR_INVALID, "alignment must be a power of two");
  if (header % align) fail(SHT_ERR_INVALID, "chunk header must be a multiple of the alignment");
  header_ = header;
  align_ = align;
  chunks_.begin()->second.size = cap_ - header_;
  free_ = cap_ - header_;
}

// An event recorded on `stream` now, shared by the chunks that cover the freed memory; the
// handle goes back to spare_events_ when the last of them drops it (always under mu_).
DevicePool::EventRef DevicePool::record_event(cudaStream_t stream) {
  cudaEvent_t e;
  if (!spare_events_.empty()) {
    e = spare_events_.back();
    spare_events_.pop_back();
  } else {
    SHT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const cudaError_t rc = cudaEventRecord(e, stream);
  if (rc != cudaSuccess) {
    spare_events_.push_back(e);
    fail(SHT_ERR_CUDA, std::string("cudaEventRecord in pool free: ") + cudaGetErrorString(rc));
  }
  return EventRef(new PoolEvent{e, stream}, [this](PoolEvent* p) {
    spare_events_.push_back(p->event);
    delete p;
  });
}

// Drop duplicate events and events whose work is done: they order nothing any more.  Keeps
// the lists of long-lived free chunks (the arena's tail) short.
void DevicePool::prune(std::vector<EventRef>& v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  v.erase(std::remove_if(v.begin(), v.end(), [](const EventRef& e) { return cudaEventQuery(e->event) == cudaSuccess; }),
          v.end());
}

void DevicePool::wait_pending(const Chunk& c, cudaStream_t stream) {
  for (const EventRef& ev : c.pending)
    if (ev->stream != stream) SHT_CUDA(cudaStreamWaitEvent(stream, ev->event, 0));
}

bool DevicePool::owns(const void* p) const {
  const char* q = static_cast<const char*>(p);
  return q >= base_ && q < base_ + cap_;
}

std::map<size_t, DevicePool::Chunk>::iterator DevicePool::find_data(const void* p) {
  if (!owns(p)) fail(SHT_ERR_INVALID, "pointer not from this pool");
  const size_t off = static_cast<size_t>(static_cast<const char*>(p) - base_) - header_;
  auto it = chunks_.find(off);
  if (it == chunks_.end() || it->second.free) fail(SHT_ERR_INVALID, "pointer is not a live pool allocation");
  return it;
}

void* DevicePool::allocate(size_t bytes, cudaStream_t stream) {
  std::lock_guard<std::recursive_mutex> lk(mu_);
  const size_t real = round_up(std::max<size_t>(bytes, 1), align_);
  for (auto it = chunks_.begin(); it != chunks_.end(); ++it) {
    Chunk& c = it->second;
    if (!c.free || c.size < real) continue;
    prune(c.pending);
    wait_pending(c, stream);
    const size_t diff = c.size - real;
    if (diff <= header_) {
      c.free = false;
      free_ -= c.size;
    } else {
      Chunk rest;
      rest.size = diff - header_;
      rest.pending = c.pending;  // the remainder is still covered by the same frees
      chunks_[it->first + header_ + real] = std::move(rest);
      c.size = real;
      c.free = false;
      free_ -= real + header_;
    }
    c.pending.clear();
    return base_ + it->first + header_;
  }
  fail(SHT_ERR_OOM, "device pool is out of memory: requested " + std::to_string(bytes) + " bytes, " +
                        std::to_string(free_) + " free");
}

void DevicePool::free(void* p, cudaStream_t stream) {
  std::lock_guard<std::recursive_mutex> lk(mu_);
  if (!p) return;
  auto it = find_data(p);
  Chunk& c = it->second;
  EventRef ev = record_event(stream);
  c.free = true;
  c.pending.push_back(std::move(ev));
  free_ += c.size;
  auto nx = std::next(it);
  if (nx != chunks_.end() && nx->second.free) {
    c.size += header_ + nx->second.size;
    c.pending.insert(c.pending.end(), nx->second.pending.begin(), nx->second.pending.end());
    chunks_.erase(nx);
    free_ += header_;
  }
  if (it != chunks_.begin()) {
    auto pv = std::prev(it);
    if (pv->second.free) {
      pv->second.size += header_ + c.size;
      pv->second.pending.insert(pv->second.pending.end(), c.pending.begin(), c.pending.end());
      prune(pv->second.pending);
      chunks_.erase(it);
      free_ += header_;
      return;
    }
  }
  prune(c.pending);
}

size_t DevicePool::size_of(void* p) const {
  std::lock_guard<std::recursive_mutex> lk(mu_);
  auto self = const_cast<DevicePool*>(this);
  return self->find_data(p)->second.size;
}

// Intended semantics of MemoryPool::reallocate (MemoryPool.h:187-318): shrink in place and
// hand the tail to a free neighbour or a new free chunk; grow in place into a free right
// neighbour when it is large enough; otherwise allocate, copy on `stream`, free the old one.
void* DevicePool::reallocate(void* p, size_t bytes, cudaStream_t stream) {
  std::lock_guard<std::recursive_mutex> lk(mu_);
  if (!p) return allocate(bytes, stream);
  auto it = find_data(p);
  Chunk& c = it->second;
  const size_t real = round_up(std::max<size_t>(bytes, 1), align_);
  if (real == c.size) return p;
  auto nx = std::next(it);
  if (real < c.size) {
    const size_t diff = c.size - real;
    if (nx != chunks_.end() && nx->second.free) {
      Chunk moved = std::move(nx->second);
      chunks_.erase(nx);
      moved.size += diff;
      moved.pending.push_back(record_event(stream));  // the tail was in use on `stream`
      c.size = real;
      chunks_[it->first + header_ + real] = std::move(moved);
      free_ += diff;
    } else if (diff > header_) {
      Chunk rest;
      rest.size = diff - header_;
      rest.pending.push_back(record_event(stream));
      c.size = real;
      chunks_[it->first + header_ + real] = std::move(rest);
      free_ += diff - header_;
    }
    return p;
  }
  const size_t need = real - c.size;
  if (nx != chunks_.end() && nx->second.free && header_ + nx->second.size >= need) {
    wait_pending(nx->second, stream);
    const size_t left = header_ + nx->second.size - need;  // bytes of the neighbour left over
    std::vector<EventRef> nx_pending = std::move(nx->second.pending);
    chunks_.erase(nx);
    if (left >= header_ + align_) {
      Chunk rest;
      rest.size = left - header_;
      rest.pending = std::move(nx_pending);
      c.size = real;
      chunks_[it->first + header_ + real] = std::move(rest);
      free_ -= need;
    } else {
      c.size = real + left;
      free_ -= need + left - header_;
    }
    return p;
  }
  const size_t old = c.size;
  void* q = allocate(bytes, stream);
  SHT_CUDA(cudaMemcpyAsync(q, p, std::min(old, real), cudaMemcpyDeviceToDevice, stream));
  free(p, stream);
  return q;
}

}  // namespace sht
