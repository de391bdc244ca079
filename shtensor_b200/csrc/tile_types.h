// tile_types.h -- plain descriptors shared by host code and the tile kernels.
#pragma once

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

}  // namespace sht
