// device_common.cuh -- small device-side helpers shared by the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "sht_internal.h"

namespace sht {

// Block-grid description of a tensor, passed by value to kernels.
struct TensorMeta {
  int order;
  int nblk[kMaxOrder];
  int bstart[kMaxOrder];     // start of mode d's sizes in bsizes
  long long gstride[kMaxOrder];
  const int* bsizes;
};

TensorMeta make_meta(const sht_tensor* t);

__device__ __forceinline__ void unroll_block(const TensorMeta& m, long long id, int* coords) {
#pragma unroll
  for (int d = 0; d < kMaxOrder; ++d) {
    if (d < m.order) coords[d] = static_cast<int>((id / m.gstride[d]) % m.nblk[d]);
  }
}

inline int grid_for(int64_t n, int threads, int cap = 148 * 32) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return static_cast<int>(g);
}

}  // namespace sht
