// C++ drop-in check: code written against shtensor's Kernel<T> / Tensor<T,N> API, compiled
// against include/shtensor_b200.hpp and linked with libshtensor_b200.so.  Mirrors the
// reference's own tests: test/test_kernel.cpp (test_contract, test_kernel's beta identity)
// and test/test_tensor.cpp (360-block tensor walked with the block iterators, alternating-block
// filter + compress through get_local_block).
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <random>
#include <vector>

#include "shtensor_b200.hpp"

static int failures = 0;
#define CHECK(cond)                                               \
  do {                                                            \
    if (!(cond)) {                                                \
      std::printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                 \
    }                                                             \
  } while (0)

template <typename T>
static void test_contract(Shtensor::Context& ctx) {
  // "ik, kj -> ij" {8,5}{5,6}{8,6}, 20 ops, alpha 1 beta 0 (test_kernel.cpp:306-308)
  const int nops = 20, M = 8, K = 5, N = 6;
  std::mt19937 gen(5);
  std::uniform_real_distribution<double> dis(-1.0, 1.0);
  std::vector<T> a(nops * M * K), b(nops * K * N), c(nops * M * N, 0);
  for (auto& x : a) x = (T)dis(gen);
  for (auto& x : b) x = (T)dis(gen);
  Shtensor::Kernel<T> kernel(ctx, "ik, kj -> ij", std::array<int, 2>{M, K}, std::array<int, 2>{K, N},
                             std::array<int, 2>{M, N}, T(1), T(0), Shtensor::KernelType::XMM);
  kernel.call(a.data(), b.data(), c.data(), nops);
  double maxerr = 0;
  for (int op = 0; op < nops; ++op)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < M; ++i) {
        T ref = 0;
        for (int k = 0; k < K; ++k) ref = std::fma(a[op * M * K + k * M + i], b[op * K * N + j * K + k], ref);
        maxerr = std::fmax(maxerr, std::fabs((double)(ref - c[op * M * N + j * M + i])));
      }
  CHECK(maxerr == 0.0);  // same fma chain: bit-exact
  CHECK(kernel.get_info().find("map_row") != std::string::npos);
}

static void test_beta(Shtensor::Context& ctx) {
  // alpha 0, beta 2: sum(C') = 2 sum(C) (test_kernel.cpp:241-285)
  std::vector<double> a(16, 1.0), b(16, 1.0), c(16);
  for (int i = 0; i < 16; ++i) c[i] = i * 0.25;
  double s0 = 0, s1 = 0;
  for (double v : c) s0 += v;
  Shtensor::Kernel<double> k(ctx, "ij, jk -> ki", std::vector<int>{4, 4}, std::vector<int>{4, 4},
                             std::vector<int>{4, 4}, 0.0, 2.0);
  k.call(a.data(), b.data(), c.data(), 1);
  for (double v : c) s1 += v;
  CHECK(s1 == 2.0 * s0);
}

static void test_tensor(Shtensor::Context& ctx) {
  Shtensor::VArray<4> bs = {std::vector<int>{4, 5, 3, 4}, std::vector<int>{5, 5, 8, 9, 2},
                            std::vector<int>{5, 6, 3, 7, 7, 9}, std::vector<int>{4, 3, 2}};
  Shtensor::Tensor<float, 4> t(ctx, bs);
  t.reserve_all();
  CHECK(t.get_nb_nzblocks_local() == 360);
  auto info = t.get_sparse_info();
  std::vector<float> data(t.get_nb_nonzeros());
  for (size_t b = 0; b < info.indices.size(); ++b) {
    const int64_t end = b + 1 < info.indices.size() ? info.offsets[b + 1] : (int64_t)data.size();
    for (int64_t e = info.offsets[b]; e < end; ++e) data[e] = (info.indices[b] % 2 == 0) ? 0.f : 1.f;
  }
  t.upload(data);
  t.filter(1e-6f, Shtensor::BlockNorm::FROBENIUS, true);
  CHECK(t.get_nb_nzblocks_local() == 180);
  for (float v : t.data()) CHECK(v == 1.f);
}

static void test_block_iteration(Shtensor::Context& ctx) {
  // test/test_tensor.cpp:53-125: a 360-block tensor walked with the block iterators; every
  // block filled through get_local_block with 0 or 1 by the parity of its id; filter without
  // compress marks the zero blocks (negative ids), compress drops them
  std::vector<int> dim0 = {4, 5, 3, 4}, dim1 = {5, 5, 8, 9, 2}, dim2 = {5, 6, 3, 7, 7, 9}, dim3 = {4, 3, 2};
  Shtensor::VArray<4> bs4 = {dim0, dim1, dim2, dim3};
  Shtensor::Tensor<float, 4> t(ctx, bs4);
  t.reserve_all();
  CHECK(t.get_nb_nzblocks_global() == 360);
  int64_t nblocks = 0;
  for (auto iter = t.begin(); iter != t.end(); ++iter) {
    auto idx = iter.get_indices();
    for (int d = 0; d < 4; ++d) CHECK(bs4[d][idx[d]] == iter->dim(d));
    ++nblocks;
  }
  CHECK(nblocks == 360);
  for (auto iter = t.begin(); iter != t.end(); ++iter) {
    const int64_t iblk = iter - t.begin();
    const int64_t blkid = iter.get_block_index();
    auto block = t.get_local_block(iblk);
    std::fill(block.begin(), block.end(), (blkid % 2 == 0) ? 0.f : 1.f);
  }
  t.filter(1e-6f, Shtensor::BlockNorm::FROBENIUS, false);
  int64_t kept = 0;
  for (auto iter = t.begin(); iter != t.end(); ++iter) {
    const int64_t blkid = iter.get_block_index();
    const int64_t ablkid = blkid >= 0 ? blkid : -(blkid + 1);
    CHECK((ablkid % 2 == 0) == (blkid < 0));
    kept += blkid < 0 ? 0 : 1;
    // a marked block keeps its extents (indices of its original id)
    auto idx = iter.get_indices();
    for (int d = 0; d < 4; ++d) CHECK(bs4[d][idx[d]] == iter->dim(d));
  }
  t.compress();
  for (auto iter = t.cbegin(); iter != t.cend(); ++iter) {
    CHECK(iter.get_block_index() >= 0);
    for (float v : *iter) CHECK(v == 1.f);
  }
  CHECK(kept == t.get_nb_nzblocks_local());
  CHECK(kept == 180);
}

static void test_sparse_blocks_and_views(Shtensor::Context& ctx) {
  // a sparse pattern: block sizes come from indices[b], not from the storage position
  Shtensor::VArray<3> bs = {std::vector<int>{2, 3, 4}, std::vector<int>{5, 1}, std::vector<int>{3, 2, 6}};
  Shtensor::Tensor<double, 3> t(ctx, bs);
  const std::vector<int> i0 = {2, 0, 1, 2}, i1 = {1, 0, 1, 0}, i2 = {2, 1, 0, 0};
  t.reserve(Shtensor::VArray<3>{i0, i1, i2});
  auto info = t.get_sparse_info();
  CHECK(info.indices.size() == 4);
  // fill element (a, b, c) of every block with id * 1000 + a + 10 b + 100 c through operator()
  for (int64_t b = 0; b < t.get_nb_nzblocks_local(); ++b) {
    auto blk = t.get_local_block(b);
    const auto idx = t.get_block_indices(b);
    int64_t rolled = idx[0] + 3 * (idx[1] + 2 * idx[2]);
    CHECK(rolled == info.indices[b]);
    for (int d = 0; d < 3; ++d) CHECK(blk.dim(d) == bs[d][idx[d]]);
    for (int c = 0; c < blk.dim(2); ++c)
      for (int y = 0; y < blk.dim(1); ++y)
        for (int a = 0; a < blk.dim(0); ++a) blk(a, y, c) = (double)(info.indices[b] * 1000 + a + 10 * y + 100 * c);
  }
  // data() writes the modified mirror back first; column-major layout within a block
  const std::vector<double> all = t.data();
  for (int64_t b = 0; b < (int64_t)info.indices.size(); ++b) {
    auto blk = t.get_local_block(b);
    for (int c = 0; c < blk.dim(2); ++c)
      for (int y = 0; y < blk.dim(1); ++y)
        for (int a = 0; a < blk.dim(0); ++a) {
          const int64_t e = info.offsets[b] + a + blk.dim(0) * (y + blk.dim(1) * c);
          CHECK(all[e] == (double)(info.indices[b] * 1000 + a + 10 * y + 100 * c));
        }
  }
  // host norms of the views equal the device's, bit for bit (FROBENIUS and MAXABS)
  for (auto norm : {Shtensor::BlockNorm::FROBENIUS, Shtensor::BlockNorm::MAXABS}) {
    const auto dn = t.norms(norm);
    int64_t b = 0;
    for (auto it = t.cbegin(); it != t.cend(); ++it, ++b) CHECK(it->get_norm(norm) == dn[b]);
  }
  // random access
  auto it = t.cbegin();
  CHECK((it + 3)->dim(0) == bs[0][t.get_block_indices(3)[0]]);
  CHECK(t.cend() - t.cbegin() == 4);
  CHECK((it + 4) == t.cend() && (it + 4)->size() == 0);
  // the device view points into the tensor's device data at the block's offset
  auto dv = t.get_device_block(2);
  auto hv = t.get_local_block(2);
  CHECK(dv.size() == hv.size() && dv.dim(1) == hv.dim(1));
  // an owning copy
  Shtensor::Block<double, 3> copy(hv);
  CHECK(copy.size() == hv.size() && copy(0, 0, 0) == hv(0, 0, 0) && copy.data() != hv.data());
}

static void test_blocksparse(Shtensor::Context& ctx) {
  // C[i,k] = sum_j A[i,j] B[j,k] over 3x3 block grids, all blocks present
  Shtensor::VArray<2> ba = {std::vector<int>{2, 3, 4}, std::vector<int>{3, 1, 2}};
  Shtensor::VArray<2> bb = {std::vector<int>{3, 1, 2}, std::vector<int>{5, 2, 3}};
  Shtensor::VArray<2> bc = {std::vector<int>{2, 3, 4}, std::vector<int>{5, 2, 3}};
  Shtensor::Tensor<double, 2> A(ctx, ba), B(ctx, bb), C(ctx, bc);
  A.reserve_all();
  B.reserve_all();
  C.reserve(std::array<std::vector<int>, 2>{std::vector<int>{}, std::vector<int>{}});
  std::vector<double> da(A.get_nb_nonzeros(), 1.0), db(B.get_nb_nonzeros(), 0.5);
  A.upload(da);
  B.upload(db);
  auto rep = Shtensor::contract(ctx, "ij, jk -> ik", 1.0, A, B, 0.0, C);
  CHECK(rep.npairs == 27);
  CHECK(C.get_nb_nzblocks_local() == 9);
  for (double v : C.data()) CHECK(v == 3.0);  // 6 terms of 0.5
}

int main() {
  try {
    Shtensor::Context ctx(1ll << 28);
    test_contract<double>(ctx);
    test_contract<float>(ctx);
    test_beta(ctx);
    test_tensor(ctx);
    test_block_iteration(ctx);
    test_sparse_blocks_and_views(ctx);
    test_blocksparse(ctx);
  } catch (const std::exception& e) {
    std::printf("exception: %s\n", e.what());
    return 2;
  }
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
  return failures ? 1 : 0;
}
