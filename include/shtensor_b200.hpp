// shtensor_b200.hpp -- C++ drop-in layer over the C ABI, shaped like shtensor's own API.
//
// Code written against shtensor's Kernel<T> (src/Kernel/Kernel.h:62-93) and Tensor<T,N>
// (src/Tensor/Tensor.h:19-366) switches by including this header instead and linking
// libshtensor_b200.so.  Differences a caller sees:
//   * Context takes a pool size and a device, not an MPI communicator (single rank, no MPI);
//   * Kernel<T>::call accepts host or device pointers (host buffers are staged through the
//     device pool and the call returns once the result is back on the host);
//   * Tensor<T,N> keeps its blocks in device memory; get_block()/set_block() copy one block
//     and data()/upload() move the whole tensor;
//   * contract() is the block-sparse contraction the reference does not have.
// Errors surface as std::runtime_error carrying the library's message, as the reference's
// constructors do.
#pragma once

#include <array>
#include <cstdint>
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
    for (const auto& v : block_sizes) {
      nb.push_back((int)v.size());
      flat.insert(flat.end(), v.begin(), v.end());
    }
    detail::check(sht_tensor_create(ctx.handle(), N, nb.data(), flat.data(), detail::dtype<T>(), &t_));
  }
  Tensor(const Tensor&) = delete;
  Tensor& operator=(const Tensor&) = delete;
  ~Tensor() { sht_tensor_destroy(t_); }

  void reserve_all() { detail::check(sht_tensor_reserve_all(t_)); }
  void reserve(const std::vector<int>* idx) {
    std::vector<int> flat;
    const size_t n = idx[0].size();
    for (int d = 0; d < N; ++d) {
      if (idx[d].size() != n) throw std::runtime_error("reserve: Indices do not have the same size in each dimension");
      flat.insert(flat.end(), idx[d].begin(), idx[d].end());
    }
    detail::check(sht_tensor_reserve(t_, (int64_t)n, flat.data()));
  }
  void reserve(const VArray<N>& idx) { reserve(idx.data()); }
  // index lists already in device memory, mode-major (d_idx[d * nblocks + b]); see
  // sht_tensor_reserve_device
  void reserve_device(const int* d_idx, int64_t nblocks, void* stream = nullptr) {
    detail::check(sht_tensor_reserve_device(t_, nblocks, d_idx, stream));
  }

  int64_t get_nb_nzblocks_local() const {
    int64_t nb = 0, nnz = 0;
    detail::check(sht_tensor_info(t_, &nb, &nnz));
    return nb;
  }
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

  std::vector<T> data() const {
    std::vector<T> h(get_nb_nonzeros());
    detail::check(sht_tensor_download(t_, h.data(), (int64_t)h.size(), nullptr));
    return h;
  }
  void upload(const std::vector<T>& h) { detail::check(sht_tensor_upload(t_, h.data(), (int64_t)h.size(), nullptr)); }

  // Tensor::filter(eps, norm, compress), Tensor.h:337-363
  void filter(T eps, BlockNorm norm, bool compress = true) {
    detail::check(sht_tensor_filter(t_, (double)eps, (sht_norm)norm, compress ? 1 : 0, nullptr));
  }
  void compress() { detail::check(sht_tensor_compress(t_, nullptr)); }
  std::vector<double> norms(BlockNorm norm) const {
    std::vector<double> out(get_nb_nzblocks_local());
    detail::check(sht_tensor_norms(t_, (sht_norm)norm, out.data(), nullptr));
    return out;
  }

  sht_tensor* handle() const { return t_; }
  const VArray<N>& block_sizes() const { return block_sizes_; }

 private:
  const Context* ctx_;
  VArray<N> block_sizes_;
  sht_tensor* t_ = nullptr;
};

// C = beta*C + alpha * contract(expr, A, B) over the block-sparse tensors (single rank)
template <typename T, int NA, int NB, int NC>
sht_contract_report contract(const Context& ctx, const std::string& expr, T alpha, Tensor<T, NA>& A,
                             Tensor<T, NB>& B, T beta, Tensor<T, NC>& C, double screen_eps = 0.0,
                             BlockNorm norm = BlockNorm::FROBENIUS,
                             ContractMode mode = ContractMode::BATCHED_FP64, void* stream = nullptr) {
  sht_contract_report rep{};
  detail::check(sht_contract(ctx.handle(), expr.c_str(), (double)alpha, A.handle(), B.handle(), (double)beta,
                             C.handle(), screen_eps, (sht_norm)norm, (sht_mode)mode, stream, &rep));
  return rep;
}

}  // namespace Shtensor
