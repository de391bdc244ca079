// tile_types.h -- plain descriptors shared by host code and the tile kernels.
#pragma once

#include <cuda_runtime.h>

#include "sht_internal.h"

namespace sht {

// One matrix dimension of the contraction as a list of tensor modes.
struct ModeMap {
  int n;                 // number of tensor modes forming this matrix dimension
  int x[kMaxOrder];      // mode index in the first operand (A for rows and k, B for cols)
  int y[kMaxOrder];      // mode index in the second (C for rows and cols, B for k)
};

struct TileMaps {
  ModeMap row, kk, col;
  int oA, oB, oC;
};

template <typename T>
struct TileScalars {
  T alpha, beta;
  int beta_zero;   // beta is +0.0: C is not read
  int alpha_zero;  // alpha is +0.0: products skipped
};

// Device pointers and scalars of one block-sparse execute (plain and batched forms).
struct SparseArgs {
  TileMaps mp;
  TileScalars<double> sc;
  const double* A; const long long* offA; const int* dimsA;
  const double* B; const long long* offB; const int* dimsB;
  double* C; const long long* offC; const int* dimsC;
  const int* pair_a; const int* pair_b; const int* pstart;
  const int2* work;
};

}  // namespace sht
