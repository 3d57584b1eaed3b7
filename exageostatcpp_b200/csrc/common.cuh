// Shared definitions of the B200 ExaGeoStat path: status codes, the device tile
// layout of a symmetric matrix, and small device helpers.
//
// Device layout of one covariance matrix (the replacement of the Chameleon
// descriptor created by CHAMELEON_Desc_Create, src/data-units/descriptor/
// concrete/ChameleonDescriptor.cpp:19-35): the N x N matrix is padded to
// Np = nt * ts rows (ts a multiple of 64), and only the nt (nt + 1) / 2 lower
// tiles are stored, tile after tile, each ts x ts column-major with leading
// dimension ts.  Tile (i, j), i >= j, sits at linear slot
//     idx(i, j) = j * nt - j (j - 1) / 2 + (i - j)
// so every tile column j (tiles j..nt-1) is one contiguous range.  Padded rows
// and columns hold the identity, which leaves the Cholesky factor, the
// log-determinant and the quadratic form of the real N x N block unchanged.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "exageostat_b200.h"

namespace egs {

__host__ __device__ __forceinline__ long long tile_slot(int i, int j, int nt) {
  return (long long)j * nt - (long long)j * (j - 1) / 2 + (i - j);
}

__host__ __device__ __forceinline__ long long lower_tiles(int nt) {
  return (long long)nt * (nt + 1) / 2;
}

// Spin limit for every device-side wait: after this many polls a waiting thread
// records EGS_ERR_TIMEOUT in the launch's error word and gives up.
constexpr long long kSpinLimit = 1ll << 26;

}  // namespace egs

#define EGS_CUDA_TRY(expr)                                  \
  do {                                                      \
    cudaError_t egs_e_ = (expr);                            \
    if (egs_e_ != cudaSuccess) {                            \
      egs::set_last_error(cudaGetErrorString(egs_e_), #expr); \
      return EGS_ERR_CUDA;                                  \
    }                                                       \
  } while (0)

namespace egs {
void set_last_error(const char* what, const char* where);
}
