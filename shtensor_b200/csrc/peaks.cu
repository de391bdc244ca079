// peaks.cu -- in-run roofline denominators that the measured-peaks file (HBM copy, bf16 GEMM) lacks.
//   which = 0: FP64 FMA throughput (TFLOP/s) from independent DFMA chains on every SM (the
//              roofline of the plain form's DFMA tile kernel);
//   which = 2: FP64 tensor-core throughput (TFLOP/s) from independent mma.sync m8n8k4 f64
//              chains on every SM (the roofline of the batched form's DMMA kernel).
#include <algorithm>

#include "sht_internal.h"

namespace sht {

__global__ void __launch_bounds__(256) k_dfma_chains(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = 1e-3 * (threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = fma(x[j], a, b);
  }
  double s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == 123456.789) out[blockIdx.x] = s;  // keeps the chains alive
}

double measure_fp64_tflops(sht_ctx* ctx) {
  const int threads = 256, blocks = ctx->num_sms * 8, iters = 1 << 14;
  PoolBuf out(ctx->pool.get(), blocks * 8, nullptr);
  cudaEvent_t e0, e1;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    SHT_CUDA(cudaEventRecord(e0, nullptr));
    k_dfma_chains<<<blocks, threads, 0, nullptr>>>(out.as<double>(), iters, 0.999999, 1e-9);
    SHT_CUDA(cudaEventRecord(e1, nullptr));
    SHT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double fl = 2.0 * 8.0 * iters * (double)threads * blocks;
    if (rep > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

// Every warp runs 8 independent accumulator chains of m8n8k4 FP64 MMAs (512 flops each).
__global__ void __launch_bounds__(256) k_dmma_chains(double* out, int iters) {
  const int lane = threadIdx.x & 31;
  const double a = 1e-3 * (lane + 1), b = 0.999 - 1e-4 * lane;
  double c[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = 1e-6 * j;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[j][0]), "+d"(c[j][1])
                   : "d"(a), "d"(b));
  }
  double s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1];
  if (s == 123456.789) out[blockIdx.x] = s;  // keeps the chains alive
}

double measure_dmma_tflops(sht_ctx* ctx) {
  const int threads = 256, blocks = ctx->num_sms * 8, iters = 1 << 12;
  PoolBuf out(ctx->pool.get(), blocks * 8, nullptr);
  cudaEvent_t e0, e1;
  SHT_CUDA(cudaEventCreate(&e0));
  SHT_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    SHT_CUDA(cudaEventRecord(e0, nullptr));
    k_dmma_chains<<<blocks, threads, 0, nullptr>>>(out.as<double>(), iters);
    SHT_CUDA(cudaEventRecord(e1, nullptr));
    SHT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SHT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double fl = 512.0 * 8.0 * iters * (double)(threads / 32) * blocks;
    if (rep > 0) best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace sht
