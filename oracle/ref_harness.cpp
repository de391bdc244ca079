// ref_harness.cpp -- thin C entry points over the reference's own headers, compiled in place
// from the shtensor sources (src/Basics/ContractInfo.h, src/Basics/Utils.h) by
// oracle/Makefile into oracle/_ref/libshtref.so.  TEST INFRASTRUCTURE ONLY.
//
// It pins the CPU restatement (oracle.cpp) to the reference:
//   ref_contract_info  -> Shtensor::compute_contract_info   (ContractInfo.h:69-346)
//   ref_reshape_f64    -> Shtensor::Utils::reshape          (Utils.h:315-359)
// and provides the reference-faithful CPU baseline of the block-sparse path:
//   ref_kernel_lapack_f64 / ref_contract_run run the LAPACK path of KernelImpl.cpp:142-208
//   (reshape with Utils::reshape, ?gemm from OpenBLAS, reshape back) per block pair.
// KernelImpl.cpp itself cannot be compiled here: it includes asmjit (fetched from the network
// by the reference's CMake), so the 40-line lambda body is restated in oracle.cpp
// (lapack_triple) and driven with the reference's reshape and a real BLAS dgemm.
#include <dlfcn.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ContractInfo.h"
#include "Utils.h"
#include "oracle_internal.h"

namespace {

typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*,
                        const double*, const double*, const int*, const double*, const int*,
                        const double*, double*, const int*);
typedef void (*setthreads_t)(int);
dgemm_t g_dgemm = nullptr;

void blas_gemm(int m, int n, int k, double alpha, const double* A, int lda, const double* B,
               int ldb, double beta, double* C, int ldc) {
  const char N = 'N';
  g_dgemm(&N, &N, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}

void ref_reshape(const double* in, const int* sizes, const int* order, int n, double* out) {
  const std::vector<int> s(sizes, sizes + n), o(order, order + n);
  Shtensor::Utils::reshape(in, s, o, out);
}

void set_err(char* err, int errlen, const std::string& msg) {
  if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
}

}  // namespace

extern "C" {

// Loads ?gemm from an OpenBLAS shared object (the one bundled with scipy); returns 0 on success.
int ref_init_blas(const char* path, const char* dgemm_symbol, const char* threads_symbol,
                  int nthreads) {
  void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return 1;
  g_dgemm = (dgemm_t)dlsym(h, dgemm_symbol);
  if (!g_dgemm) return 2;
  if (threads_symbol && threads_symbol[0]) {
    auto st = (setthreads_t)dlsym(h, threads_symbol);
    if (st) st(nthreads);
  }
  return 0;
}

int ref_contract_info(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                      const int* sC, int* maps, int* counts, int* scatter, int scatter_cap,
                      char* err, int errlen) {
  Shtensor::ContractInfo a, b, c;
  std::string e;
  const std::vector<int> va(sA, sA + nA), vb(sB, sB + nB), vc(sC, sC + nC);
  if (!Shtensor::compute_contract_info(std::string(expr), va, vb, vc, a, b, c, e)) {
    set_err(err, errlen, e);
    return 1;
  }
  const std::vector<int>* lists[6] = {&a.map_row, &a.map_col, &b.map_row, &b.map_col, &c.map_row, &c.map_col};
  const std::vector<int>* scat[6] = {&a.scatter_row, &a.scatter_col, &b.scatter_row, &b.scatter_col, &c.scatter_row, &c.scatter_col};
  int pos = 0;
  for (int i = 0; i < 6; ++i) {
    counts[i] = (int)lists[i]->size();
    for (size_t j = 0; j < lists[i]->size() && j < 16; ++j) maps[i * 16 + (int)j] = (*lists[i])[j];
    counts[6 + i] = (int)scat[i]->size();
    for (int v : *scat[i]) {
      if (pos < scatter_cap) scatter[pos] = v;
      ++pos;
    }
  }
  return 0;
}

void ref_reshape_f64(const double* in, const int* sizes, const int* order, int n, double* out) {
  ref_reshape(in, sizes, order, n, out);
}

int ref_kernel_lapack_f64(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                          const int* sC, double alpha, double beta, const double* a,
                          const double* b, double* c, int64_t nb_ops, char* err, int errlen) {
  if (!g_dgemm) { set_err(err, errlen, "BLAS not initialised"); return 3; }
  ora::Maps m;
  std::string e;
  if (!ora::parse_contraction(expr, nA, sA, nB, sB, nC, sC, m, e)) { set_err(err, errlen, e); return 1; }
  int64_t za = 1, zb = 1, zc = 1;
  for (int i = 0; i < nA; ++i) za *= sA[i];
  for (int i = 0; i < nB; ++i) zb *= sB[i];
  for (int i = 0; i < nC; ++i) zc *= sC[i];
  std::vector<double> buf;
  for (int64_t op = 0; op < nb_ops; ++op)
    ora::lapack_triple(a + op * za, b + op * zb, c + op * zc, sA, nA, sB, nB, sC, nC, m, alpha,
                       beta, blas_gemm, ref_reshape, buf);
  return 0;
}

// Block-sparse contraction driven with the reference's reshape and BLAS per pair; same
// result handle as ora_contract_run (free it with ora_result_free from liboracle.so, which
// this library also exports).
void* ref_contract_run(const char* expr, double alpha, int oA, const int* nbA, const int* bsA,
                       int64_t nA, const int64_t* idsA, const int64_t* offA, const double* dA,
                       int oB, const int* nbB, const int* bsB, int64_t nB, const int64_t* idsB,
                       const int64_t* offB, const double* dB, double beta, int oC,
                       const int* nbC, const int* bsC, int64_t nC, const int64_t* idsC,
                       const int64_t* offC, const double* dC, double eps, int norm, int nthreads,
                       char* err, int errlen) {
  if (!g_dgemm) { set_err(err, errlen, "BLAS not initialised"); return nullptr; }
  ora::BTensor A, B, C;
  ora::load_tensor(oA, nbA, bsA, nA, idsA, offA, A);
  ora::load_tensor(oB, nbB, bsB, nB, idsB, offB, B);
  ora::load_tensor(oC, nbC, bsC, nC, idsC, offC, C);
  auto* R = new ora::ContractResult();
  std::string e;
  if (!ora::contract(expr, alpha, A, dA, B, dB, beta, C, dC, eps, norm, 1, nthreads, blas_gemm,
                     ref_reshape, *R, e)) {
    set_err(err, errlen, e);
    delete R;
    return nullptr;
  }
  return R;
}

}  // extern "C"
