// shtensor_b200.hpp -- C++ drop-in layer over the C ABI, shaped like shtensor's own API.
//
// Code written against shtensor's Kernel<T> (src/Kernel/Kernel.h:62-93) and Tensor<T,N>
// (src/Tensor/Tensor.h:19-366) switches by including this header instead and linking
// libshtensor_b200.so.  Differences a caller sees:
//   * Context takes a pool size and a device, not an MPI communicator (single rank, no MPI);
//   * Kernel<T>::call accepts host or device pointers (host buffers are staged through the
//     device pool and the call returns once the result is back on the host);
//   * Tensor<T,N> keeps its blocks in device memory.  get_local_block(b) and the block
//     iterators (begin/end/cbegin/cend) work on a host mirror of the data, read from the
//     device on first use; a non-const access marks the mirror modified, and every
//     device-side step (filter, compress, norms, contract, data(), sync_device()) writes a
//     modified mirror back first.  Device steps that change the tensor drop the mirror, so the
//     next access reads it again.  get_device_block(b) gives the same view on device memory;
//     data()/upload() move the whole tensor;
//   * iterators and get_local_block address a block by its storage position b and take its
//     sizes from indices[b] (the reference unrolls the position itself, Tensor.h:42,241, which
//     gives the right sizes only after reserve_all on a full grid);
//   * contract() is the block-sparse contraction the reference does not have.
// Errors surface as std::runtime_error carrying the library's message, as the reference's
// constructors do.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <iterator>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "shtensor_b200.h"

namespace Shtensor {

enum class KernelType { LAPACK = 0, XMM = 1 };                    // KernelDefinitions.h:11-15
enum class BlockNorm { FROBENIUS = 0, MAXABS = 1, FROBENIUS_REFCOMPAT = 2 };  // BlockSpan.h:87-91
enum class ContractMode { PLAIN_FP64 = SHT_MODE_PLAIN_FP64, BATCHED_FP64 = SHT_MODE_BATCHED_FP64,
                          SPLIT = SHT_MODE_SPLIT };

template <int N>
using VArray = std::array<std::vector<int>, N>;                   // Definitions.h:50-51

// Contiguous view of n elements (Span<T>, src/Basics/BlockSpan.h:16-92).
template <typename T>
class Span {
 public:
  using iterator = T*;
  using const_iterator = const T*;
  Span() = default;
  Span(T* p, int64_t n) : p_(p), n_(n) {}
  T* data() { return p_; }
  const T* data() const { return p_; }
  iterator begin() { return p_; }
  iterator end() { return p_ + n_; }
  const_iterator begin() const { return p_; }
  const_iterator end() const { return p_ + n_; }
  std::size_t size() const { return (std::size_t)n_; }
  int64_t ssize() const { return n_; }
  T& operator[](int64_t i) { return p_[i]; }
  const T& operator[](int64_t i) const { return p_[i]; }
  void swap(T* p) { p_ = p; }

 protected:
  T* p_ = nullptr;
  int64_t n_ = 0;
};

namespace detail {
// Block norm in this library's fixed chunked order, the order of the device's
// sht_tensor_norms (so both give the same bits): chunks of 4096 consecutive elements; in a
// chunk, lane j (0..127) folds elements j, j+128, ... in ascending order (FROBENIUS: fma(v, v,
// p) in FP64; MAXABS: max |v|); the 128 lane values are halved in place (p[j] op= p[j + h] for
// h = 64 .. 1); chunk results fold in ascending order; FROBENIUS ends with sqrt.
// FROBENIUS_REFCOMPAT is the reference's evaluation, which truncates its running sum to int
// after every element (BlockSpan.h:147-148).
template <typename T>
double chunked_norm(const T* d, int64_t n, int norm) {
  if (norm == 2) {
    int acc = 0;
    for (int64_t i = 0; i < n; ++i) acc = (int)((double)acc + (double)d[i] * (double)d[i]);
    return std::sqrt((double)acc);
  }
  const bool maxabs = norm == 1;
  double total = 0.0;
  for (int64_t base = 0; base < n; base += 4096) {
    double p[128] = {0.0};
    const int64_t end = std::min<int64_t>(n, base + 4096);
    for (int64_t e = base; e < end; ++e) {
      const double v = (double)d[e];
      double& q = p[(e - base) & 127];
      q = maxabs ? std::max(q, std::fabs(v)) : std::fma(v, v, q);
    }
    for (int h = 64; h >= 1; h >>= 1)
      for (int j = 0; j < h; ++j) p[j] = maxabs ? std::max(p[j], p[j + h]) : p[j] + p[j + h];
    total = base == 0 ? p[0] : (maxabs ? std::max(total, p[0]) : total + p[0]);
  }
  return maxabs ? total : std::sqrt(total);
}
}  // namespace detail

// One dense block: extents, column-major strides, element access by multi-index
// (BlockSpan<T,N>, src/Basics/BlockSpan.h:100-170).  The pointer may be a host pointer (from
// Tensor::get_local_block and the iterators) or a device pointer (Tensor::get_device_block):
// the view itself never dereferences it.
template <typename T, int N>
class BlockSpan : public Span<T> {
 public:
  BlockSpan() { dims_.fill(0); strides_.fill(0); }
  BlockSpan(T* p, const std::array<int, N>& dims) : Span<T>(p, volume(dims)), dims_(dims) {
    int64_t acc = 1;
    for (int i = 0; i < N; ++i) { strides_[i] = acc; acc *= dims[i]; }
  }
  int dim(int i) const { return dims_[i]; }
  const std::array<int, N>& dims() const { return dims_; }
  template <class... Idx>
  T& operator()(Idx... idx) { return this->p_[roll(idx...)]; }
  template <class... Idx>
  const T& operator()(Idx... idx) const { return this->p_[roll(idx...)]; }
  // host pointers only
  T get_norm(BlockNorm norm) const { return (T)detail::chunked_norm(this->p_, this->n_, (int)norm); }

 private:
  static int64_t volume(const std::array<int, N>& d) {
    int64_t v = 1;
    for (int x : d) v *= x;
    return v;
  }
  template <class... Idx>
  int64_t roll(Idx... idx) const {
    static_assert(sizeof...(Idx) == N, "Incorrect number of indices passed to function");
    const int64_t v[N] = {(int64_t)idx...};
    int64_t off = 0;
    for (int i = 0; i < N; ++i) off += v[i] * strides_[i];
    return off;
  }
  std::array<int, N> dims_;
  std::array<int64_t, N> strides_;
};

// A block that owns its storage (Block<T,N>, src/Basics/BlockSpan.h:172-216).
template <typename T, int N>
class Block : public BlockSpan<T, N> {
 public:
  explicit Block(const std::array<int, N>& dims) : BlockSpan<T, N>(nullptr, dims), store_(this->size()) {
    this->swap(store_.data());
  }
  Block(const BlockSpan<T, N>& v) : BlockSpan<T, N>(v), store_(v.begin(), v.end()) { this->swap(store_.data()); }
  Block(const Block& o) : BlockSpan<T, N>(o), store_(o.store_) { this->swap(store_.data()); }
  Block& operator=(const Block& o) {
    BlockSpan<T, N>::operator=(o);
    store_ = o.store_;
    this->swap(store_.data());
    return *this;
  }

 private:
  std::vector<T> store_;
};

namespace detail {
inline void check(sht_status s) {
  if (s != SHT_OK) throw std::runtime_error(sht_last_error());
}
template <typename T>
constexpr sht_dtype dtype() {
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "Invalid float type");
  return std::is_same<T, double>::value ? SHT_F64 : SHT_F32;
}
}  // namespace detail

class Context {
 public:
  explicit Context(int64_t pool_bytes, int device = 0) { detail::check(sht_init(&ctx_, device, (size_t)pool_bytes)); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  ~Context() { sht_finalize(ctx_); }
  int64_t get_free_mem() const {
    size_t cap = 0, fr = 0;
    detail::check(sht_pool_info(ctx_, &cap, &fr, nullptr, nullptr));
    return (int64_t)fr;
  }
  sht_ctx* handle() const { return ctx_; }

 private:
  sht_ctx* ctx_ = nullptr;
};

template <class T>
class Kernel {
 public:
  template <class ArrayIn1, class ArrayIn2, class ArrayOut>
  Kernel(const Context& ctx, const std::string expr, const ArrayIn1& sizes_in1, const ArrayIn2& sizes_in2,
         const ArrayOut& sizes_out, T alpha, T beta, KernelType type = KernelType::XMM) {
    const std::vector<int> a(sizes_in1.begin(), sizes_in1.end()), b(sizes_in2.begin(), sizes_in2.end()),
        c(sizes_out.begin(), sizes_out.end());
    detail::check(sht_kernel_create(ctx.handle(), expr.c_str(), a.data(), (int)a.size(), b.data(), (int)b.size(),
                                    c.data(), (int)c.size(), (double)alpha, (double)beta, detail::dtype<T>(),
                                    (sht_kernel_type)type, &k_));
  }
  Kernel(const Kernel&) = delete;
  Kernel& operator=(const Kernel&) = delete;
  ~Kernel() { sht_kernel_destroy(k_); }

  // Kernel<T>::call(T* a, T* b, T* c, int64_t nb_ops), Kernel.h:88-91
  void call(T* a, T* b, T* c, int64_t nb_ops, void* stream = nullptr) {
    detail::check(sht_kernel_call(k_, a, b, c, nb_ops, stream));
  }

  std::string get_info() {
    std::string s(16384, '\0');
    detail::check(sht_kernel_info(k_, &s[0], s.size()));
    s.resize(s.find('\0'));
    return s;
  }

 private:
  sht_kernel* k_ = nullptr;
};

template <typename T, int N>
class Tensor {
  static_assert(N >= 2, "Tensor has to have dimension >= 2");

 public:
  Tensor(const Context& ctx, const VArray<N>& block_sizes) : ctx_(&ctx), block_sizes_(block_sizes) {
    std::vector<int> nb, flat;
    int64_t acc = 1;
    for (int d = 0; d < N; ++d) {
      const auto& v = block_sizes[d];
      nb.push_back((int)v.size());
      flat.insert(flat.end(), v.begin(), v.end());
      grid_strides_[d] = acc;
      acc *= (int64_t)v.size();
    }
    detail::check(sht_tensor_create(ctx.handle(), N, nb.data(), flat.data(), detail::dtype<T>(), &t_));
  }
  Tensor(const Tensor&) = delete;
  Tensor& operator=(const Tensor&) = delete;
  ~Tensor() { sht_tensor_destroy(t_); }

  void reserve_all() {
    drop_mirror();
    detail::check(sht_tensor_reserve_all(t_));
  }
  void reserve(const std::vector<int>* idx) {
    std::vector<int> flat;
    const size_t n = idx[0].size();
    for (int d = 0; d < N; ++d) {
      if (idx[d].size() != n) throw std::runtime_error("reserve: Indices do not have the same size in each dimension");
      flat.insert(flat.end(), idx[d].begin(), idx[d].end());
    }
    drop_mirror();
    detail::check(sht_tensor_reserve(t_, (int64_t)n, flat.data()));
  }
  void reserve(const VArray<N>& idx) { reserve(idx.data()); }
  // index lists already in device memory, mode-major (d_idx[d * nblocks + b]); see
  // sht_tensor_reserve_device
  void reserve_device(const int* d_idx, int64_t nblocks, void* stream = nullptr) {
    drop_mirror();
    detail::check(sht_tensor_reserve_device(t_, nblocks, d_idx, stream));
  }

  int64_t get_nb_nzblocks_local() const {
    int64_t nb = 0, nnz = 0;
    detail::check(sht_tensor_info(t_, &nb, &nnz));
    return nb;
  }
  // one rank: every block is local
  int64_t get_nb_nzblocks_global() const { return get_nb_nzblocks_local(); }
  int64_t get_nb_nonzeros() const {
    int64_t nb = 0, nnz = 0;
    detail::check(sht_tensor_info(t_, &nb, &nnz));
    return nnz;
  }

  struct SparseInfo {
    std::vector<int64_t> rows, indices, offsets;
  };
  // BaseTensor::get_sparse_info (BaseTensor.h:51), copied to the host
  SparseInfo get_sparse_info() const {
    SparseInfo s;
    s.indices.resize(get_nb_nzblocks_local());
    s.offsets.resize(s.indices.size());
    s.rows.resize(block_sizes_[0].size());
    detail::check(sht_tensor_get_index(t_, s.indices.data(), s.offsets.data(), s.rows.data()));
    return s;
  }

  // ---- block access (Tensor::get_local_block and the block iterators, Tensor.h:38-52,76-291)

  // Block at storage position b, a view into the host mirror.  The mirror counts as modified
  // from here on (the caller may write through the view).
  BlockSpan<T, N> get_local_block(int64_t b) {
    load_mirror();
    dirty_ = true;
    return view(b, host_.data());
  }
  // Block at storage position b in device memory (a device pointer; nothing is copied).
  BlockSpan<T, N> get_device_block(int64_t b) {
    sync_device();
    load_index();
    void* d = nullptr;
    detail::check(sht_tensor_device_data(t_, &d));
    return view(b, static_cast<T*>(d));
  }
  // Block-grid multi-index of the block at storage position b (from indices[b]; a block that
  // filter() marked, id -(id)-1, gives the indices of its original id).
  std::array<int, N> get_block_indices(int64_t b) const {
    load_index();
    int64_t id = index_.indices.at((size_t)b);
    if (id < 0) id = -(id + 1);
    std::array<int, N> out;
    for (int d = N - 1; d >= 0; --d) {
      out[d] = (int)(id / grid_strides_[d]);
      id %= grid_strides_[d];
    }
    return out;
  }
  // process-grid coordinates and rank of a block: one rank, so all zero (Tensor.h:54-72)
  std::array<int, N> get_coords_block(const std::array<int, N>&) const { return std::array<int, N>{}; }
  int get_rank_block(const std::array<int, N>&) const { return 0; }

  // Random-access iterator over the stored blocks in storage order
  // (BlockIteratorDetail, Tensor.h:76-258).
  template <bool Const>
  class BlockIteratorDetail {
   public:
    using iterator_category = std::random_access_iterator_tag;
    using difference_type = int64_t;
    using value_type = Block<T, N>;
    using pointer = typename std::conditional<Const, const BlockSpan<T, N>*, BlockSpan<T, N>*>::type;
    using reference = typename std::conditional<Const, const BlockSpan<T, N>&, BlockSpan<T, N>&>::type;

    BlockIteratorDetail(const Tensor* t, int64_t b) : t_(t), b_(b) { update(); }
    std::array<int, N> get_indices() const { return t_->get_block_indices(b_); }
    int64_t get_block_index() const { return t_->index_.indices.at((size_t)b_); }
    reference operator*() { return span_; }
    pointer operator->() { return &span_; }
    reference operator[](difference_type d) { return *(*this + d); }
    BlockIteratorDetail& operator++() { ++b_; update(); return *this; }
    BlockIteratorDetail operator++(int) { BlockIteratorDetail o(*this); ++*this; return o; }
    BlockIteratorDetail& operator--() { --b_; update(); return *this; }
    BlockIteratorDetail operator--(int) { BlockIteratorDetail o(*this); --*this; return o; }
    BlockIteratorDetail& operator+=(difference_type d) { b_ += d; update(); return *this; }
    BlockIteratorDetail& operator-=(difference_type d) { b_ -= d; update(); return *this; }
    BlockIteratorDetail operator+(difference_type d) const { BlockIteratorDetail o(*this); return o += d; }
    BlockIteratorDetail operator-(difference_type d) const { BlockIteratorDetail o(*this); return o -= d; }
    difference_type operator-(const BlockIteratorDetail& o) const { return b_ - o.b_; }
    bool operator==(const BlockIteratorDetail& o) const { return b_ == o.b_; }
    bool operator!=(const BlockIteratorDetail& o) const { return b_ != o.b_; }
    bool operator<(const BlockIteratorDetail& o) const { return b_ < o.b_; }
    bool operator>(const BlockIteratorDetail& o) const { return b_ > o.b_; }
    bool operator<=(const BlockIteratorDetail& o) const { return b_ <= o.b_; }
    bool operator>=(const BlockIteratorDetail& o) const { return b_ >= o.b_; }

   private:
    void update() {
      // before the first or past the last block: an empty view
      if (b_ < 0 || b_ >= (int64_t)t_->index_.indices.size()) {
        span_ = BlockSpan<T, N>();
        return;
      }
      span_ = t_->view(b_, const_cast<T*>(t_->host_.data()));
    }
    const Tensor* t_;
    int64_t b_;
    BlockSpan<T, N> span_;
  };
  using BlockIterator = BlockIteratorDetail<false>;
  using ConstBlockIterator = BlockIteratorDetail<true>;

  BlockIterator begin() {
    load_mirror();
    dirty_ = true;
    return BlockIterator(this, 0);
  }
  BlockIterator end() {
    load_mirror();
    return BlockIterator(this, (int64_t)index_.indices.size());
  }
  ConstBlockIterator cbegin() const {
    load_mirror();
    return ConstBlockIterator(this, 0);
  }
  ConstBlockIterator cend() const {
    load_mirror();
    return ConstBlockIterator(this, (int64_t)index_.indices.size());
  }

  // "(i,j,..)[v0,v1,..]" per block in storage order (Tensor::print_blocks, Tensor.h:264-272)
  void print_blocks(std::ostream& os) const {
    for (auto it = cbegin(); it < cend(); ++it) {
      const auto idx = it.get_indices();
      os << "(";
      for (int d = 0; d < N; ++d) os << (d ? "," : "") << idx[d];
      os << ")[";
      for (size_t e = 0; e < it->size(); ++e) os << (e ? "," : "") << (*it)[(int64_t)e];
      os << "]\n";
    }
  }

  // Writes a modified host mirror back to the device (the steps below call it themselves).
  void sync_device() {
    if (dirty_ && mirror_valid_) {
      detail::check(sht_tensor_upload(t_, host_.data(), (int64_t)host_.size(), nullptr));
    }
    dirty_ = false;
  }
  // Frees the host mirror (after writing it back if it was modified).
  void release_host() {
    sync_device();
    drop_mirror();
  }
  // The device copy changed (by a step outside this object, e.g. a kernel of the caller's):
  // the next host access reads it again.  A modified mirror is discarded.
  void invalidate_host() { drop_mirror(); }

  std::vector<T> data() {
    sync_device();
    std::vector<T> h(get_nb_nonzeros());
    detail::check(sht_tensor_download(t_, h.data(), (int64_t)h.size(), nullptr));
    return h;
  }
  void upload(const std::vector<T>& h) {
    drop_mirror();
    detail::check(sht_tensor_upload(t_, h.data(), (int64_t)h.size(), nullptr));
  }

  // Tensor::filter(eps, norm, compress), Tensor.h:337-363
  void filter(T eps, BlockNorm norm, bool compress = true) {
    sync_device();
    drop_mirror();
    detail::check(sht_tensor_filter(t_, (double)eps, (sht_norm)norm, compress ? 1 : 0, nullptr));
  }
  void compress() {
    sync_device();
    drop_mirror();
    detail::check(sht_tensor_compress(t_, nullptr));
  }
  std::vector<double> norms(BlockNorm norm) {
    sync_device();
    std::vector<double> out(get_nb_nzblocks_local());
    detail::check(sht_tensor_norms(t_, (sht_norm)norm, out.data(), nullptr));
    return out;
  }

  sht_tensor* handle() const { return t_; }
  const VArray<N>& block_sizes() const { return block_sizes_; }

 private:
  BlockSpan<T, N> view(int64_t b, T* base) const {
    std::array<int, N> dims;
    const auto idx = get_block_indices(b);
    for (int d = 0; d < N; ++d) dims[d] = block_sizes_[d][idx[d]];
    return BlockSpan<T, N>(base ? base + index_.offsets.at((size_t)b) : nullptr, dims);
  }
  void load_index() const {
    if (!index_valid_) {
      index_ = get_sparse_info();
      index_valid_ = true;
    }
  }
  void load_mirror() const {
    load_index();
    if (!mirror_valid_) {
      host_.resize((size_t)get_nb_nonzeros());
      if (!host_.empty())
        detail::check(sht_tensor_download(t_, host_.data(), (int64_t)host_.size(), nullptr));
      mirror_valid_ = true;
    }
  }
  void drop_mirror() {
    mirror_valid_ = index_valid_ = dirty_ = false;
    host_.clear();
    host_.shrink_to_fit();
  }

  const Context* ctx_;
  VArray<N> block_sizes_;
  std::array<int64_t, N> grid_strides_{};
  sht_tensor* t_ = nullptr;
  // host mirror of the index and the data (read on first use)
  mutable SparseInfo index_;
  mutable std::vector<T> host_;
  mutable bool index_valid_ = false, mirror_valid_ = false;
  bool dirty_ = false;
};

// C = beta*C + alpha * contract(expr, A, B) over the block-sparse tensors (single rank).
// Modified host mirrors of A, B and C are written back first; C's mirror is dropped after.
template <typename T, int NA, int NB, int NC>
sht_contract_report contract(const Context& ctx, const std::string& expr, T alpha, Tensor<T, NA>& A,
                             Tensor<T, NB>& B, T beta, Tensor<T, NC>& C, double screen_eps = 0.0,
                             BlockNorm norm = BlockNorm::FROBENIUS,
                             ContractMode mode = ContractMode::BATCHED_FP64, void* stream = nullptr) {
  A.sync_device();
  B.sync_device();
  C.sync_device();
  C.invalidate_host();
  sht_contract_report rep{};
  detail::check(sht_contract(ctx.handle(), expr.c_str(), (double)alpha, A.handle(), B.handle(), (double)beta,
                             C.handle(), screen_eps, (sht_norm)norm, (sht_mode)mode, stream, &rep));
  return rep;
}

}  // namespace Shtensor
