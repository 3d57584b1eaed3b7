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
#include <mutex>
#include <utility>
#include <cuda_runtime.h>
#include "exageostat_b200.h"

namespace egs {

__host__ __device__ __forceinline__ long long tile_slot(int i, int j, int nt) {
  return (long long)j * nt - (long long)j * (j - 1) / 2 + (i - j);
}

__host__ __device__ __forceinline__ long long lower_tiles(int nt) {
  return (long long)nt * (nt + 1) / 2;
}

// Runs f once for each device it is called on (kernel attributes such as the
// dynamic shared-memory limit belong to the current device's context, so a
// process that uses several devices sets them on each); devices with an
// ordinal of 64 or more run f on every call.
template <typename F>
inline void once_per_device(std::once_flag (&flags)[64], F&& f) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    f();
    return;
  }
  std::call_once(flags[dev], std::forward<F>(f));
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

// Status of the launches just issued: reads (and thereby clears) the runtime's
// last error once and records its text, so that a caller returning this code
// does not lose the error to a second cudaGetLastError().
inline int launch_status(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return EGS_OK;
  set_last_error(cudaGetErrorString(e), where);
  return EGS_ERR_CUDA;
}
}
