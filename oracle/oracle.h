/*
 * oracle.h -- CPU restatement of shtensor's single-rank block-sparse contraction path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs, never by
 * the product library (shtensor_b200/), which fails loudly without its CUDA build.
 *
 * What it restates (reference paths are relative to the shtensor project root):
 *   ora_contract_info   src/Basics/ContractInfo.h:69-346  (einsum -> row/col axis maps)
 *   ora_scatter         src/Basics/ContractInfo.h:38-66   (create_scatter_vector)
 *   ora_reshape_*       src/Basics/Utils.h:315-359        (Utils::reshape)
 *   ora_kernel_xmm_*    src/Kernel/KernelImpl.cpp:210-770 + src/Kernel/AvxHelper.cpp
 *                       (arithmetic order of the asmjit AVX2 kernel: c = beta*c, then for
 *                       k ascending c = fma(alpha*a, b, c); scalar std::fma is bit-equal
 *                       to vmulpd + vfmadd231pd lane by lane)
 *   ora_kernel_lapack_* src/Kernel/KernelImpl.cpp:142-208 (reshape -> ?gemm -> reshape back;
 *                       the GEMM is the netlib reference loop order, j -> l -> i)
 *   ora_reserve         src/Tensor/BaseTensor.cpp:117-251 (sorted rolled ids, offsets, rows)
 *   ora_block_norm      src/Basics/BlockSpan.h:140-164    (FROBENIUS / MAXABS; see below)
 *   ora_filter          src/Tensor/Tensor.h:337-363, src/Tensor/BaseTensor.cpp:253-354
 *   ora_contract_*      block-pair matching + scatter-add: absent from the reference; the
 *                       canonical rules are written out in ora_contract_run below.
 *
 * Parity pins: the axis maps, scatter vectors and reshape are checked in tests against
 * the reference's own headers compiled in place (oracle/_ref, built by oracle/Makefile
 * from ContractInfo.h / Utils.h), and every kernel result against numpy.einsum with
 * order='F' (the cross-check test/test_kernel.cpp:44-116 carries).  The block-sparse
 * layer has no reference implementation; its fixtures are frozen under tests/golden/.
 */
#ifndef SHT_ORACLE_H
#define SHT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* maps: 6 lists (rowA,colA,rowB,colB,rowC,colC), each up to 16 ints; counts[6]. */
int ora_contract_info(const char* expr, int nA, const int* sA, int nB, const int* sB,
                      int nC, const int* sC, int* maps, int* counts, char* err, int errlen);
int ora_scatter(const int* map, int nmap, const int* sizes, int nsizes, int* out);
void ora_reshape_f64(const double* in, const int* sizes, const int* order, int n, double* out);

int ora_kernel_xmm_f64(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                       const int* sC, double alpha, double beta, const double* a,
                       const double* b, double* c, int64_t nb_ops, char* err, int errlen);
int ora_kernel_xmm_f32(const char* expr, int nA, const int* sA, int nB, const int* sB, int nC,
                       const int* sC, float alpha, float beta, const float* a, const float* b,
                       float* c, int64_t nb_ops, char* err, int errlen);
int ora_kernel_lapack_f64(const char* expr, int nA, const int* sA, int nB, const int* sB,
                          int nC, const int* sC, double alpha, double beta, const double* a,
                          const double* b, double* c, int64_t nb_ops, char* err, int errlen);

/* Block-sparse storage.  idx is mode-major: idx[d*n + b] = block index of block b in mode d. */
int ora_reserve(int order, const int* nblk, const int* bsizes, int64_t n, const int* idx,
                int64_t* ids_out, int64_t* offsets_out, int64_t* rows_out, int64_t* nnz_out,
                char* err, int errlen);

/* norm: 0 = FROBENIUS (canonical warp-strided order), 1 = MAXABS,
 *       2 = FROBENIUS as the reference evaluates it (int accumulator, BlockSpan.h:147-148) */
double ora_block_norm(const double* data, int64_t n, int norm);

/* filter(eps, norm, compress) on a host tensor: returns the new block count; ids/offsets/data
 * are compacted in place (the reference's compress moves data with a zero block size,
 * BaseTensor.cpp:283-288; this restatement moves the real block sizes). */
int64_t ora_filter(int order, const int* nblk, const int* bsizes, int64_t nblocks,
                   int64_t* ids, int64_t* offsets, double* data, double eps, int norm,
                   int compress, int64_t* rows_out, int64_t* nnz_out);

/* Block-sparse contraction.  Tensors are passed as (order, nblk per mode, concatenated block
 * sizes, nblocks, sorted ids, offsets, data).  Returns an opaque result handle or NULL. */
void* ora_contract_run(const char* expr, double alpha,
                       int oA, const int* nbA, const int* bsA, int64_t nA, const int64_t* idsA,
                       const int64_t* offA, const double* dA,
                       int oB, const int* nbB, const int* bsB, int64_t nB, const int64_t* idsB,
                       const int64_t* offB, const double* dB,
                       double beta,
                       int oC, const int* nbC, const int* bsC, int64_t nC, const int64_t* idsC,
                       const int64_t* offC, const double* dC,
                       double eps, int norm, int lapack_blocks, int nthreads,
                       char* err, int errlen);
int64_t ora_result_npairs(void* h);
void ora_result_pairs(void* h, int64_t* triples);   /* (idC, idA, idB) x npairs */
int64_t ora_result_nblocks(void* h);
int64_t ora_result_nnz(void* h);
double ora_result_flops(void* h);
void ora_result_index(void* h, int64_t* ids, int64_t* offsets);
void ora_result_data(void* h, double* data);
double ora_result_seconds(void* h);
void ora_result_free(void* h);

#ifdef __cplusplus
}
#endif

#endif
