// oracle_internal.h -- C++ internals of the CPU restatement, shared with the harness that
// compiles the reference's own headers (oracle/ref_harness.cpp).  Test infrastructure only.
#ifndef SHT_ORACLE_INTERNAL_H
#define SHT_ORACLE_INTERNAL_H

#include <cstdint>
#include <string>
#include <vector>

namespace ora {

struct Maps {
  std::vector<int> rowA, colA, rowB, colB, rowC, colC;
};

struct BTensor {
  int order = 0;
  std::vector<int> nblk;
  std::vector<std::vector<int>> bs;
  std::vector<int64_t> gstride;
  std::vector<int64_t> ids, offsets, rows;
  int64_t nnz = 0;
  int64_t block_size(int64_t id) const;
  void block_dims(int64_t id, int* dims) const;
  void block_coords(int64_t id, int* coords) const;
};

struct Pair {
  int64_t c, a, b;
};

struct ContractResult {
  BTensor C;
  std::vector<double> data;
  std::vector<Pair> pairs;  // (idC, idA, idB) by id
  double flops = 0.0;
  double seconds = 0.0;
};

// column-major GEMM C = alpha*A*B + beta*C, A m×k (lda), B k×n (ldb), C m×n (ldc)
typedef void (*GemmFn)(int m, int n, int k, double alpha, const double* A, int lda,
                       const double* B, int ldb, double beta, double* C, int ldc);

typedef void (*ReshapeFn)(const double* in, const int* sizes, const int* order, int n,
                          double* out);

bool parse_contraction(const std::string& expr, int nA, const int* sA, int nB, const int* sB,
                       int nC, const int* sC, Maps& m, std::string& err);
std::vector<int64_t> strides_of(const int* sizes, int n);
std::vector<int64_t> scatter_of(const std::vector<int>& map, const int* sizes, int n);
template <typename T>
void reshape(const T* in, const int* sizes, const int* order, int n, T* out);
void lapack_triple(const double* a, const double* b, double* c, const int* sA, int nA,
                   const int* sB, int nB, const int* sC, int nC, const Maps& m, double alpha,
                   double beta, GemmFn gemm, ReshapeFn rfn, std::vector<double>& buf);
double block_norm(const double* d, int64_t n, int norm);
void load_tensor(int order, const int* nblk, const int* bsizes, int64_t n, const int64_t* ids,
                 const int64_t* offs, BTensor& t);
bool contract(const std::string& expr, double alpha, const BTensor& A, const double* dA,
              const BTensor& B, const double* dB, double beta, const BTensor& Cin,
              const double* dCin, double eps, int norm, int lapack_blocks, int nthreads,
              GemmFn gemm, ReshapeFn rfn, ContractResult& R, std::string& err);

}  // namespace ora

#endif
