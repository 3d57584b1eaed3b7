// Device body of the Matern tile generator, shared by the single-problem
// kernel (matern.cu) and the batched kernel (batch.cu).
#pragma once
#include "bessel_k.cuh"

namespace egs {

constexpr int kGenThreads = 256;
constexpr int kGenPairsPerThread = 8;
constexpr int kGenPairsPerBlock = kGenThreads * kGenPairsPerThread;  // 4096 elements per block

// Copies one problem's Chebyshev table into shared memory when its nu uses it.
// Every thread of the block calls it (it ends with a barrier).
__device__ __forceinline__ void stage_ktab(double* __restrict__ stab, const double* __restrict__ tab,
                                           const MaternParams& p) {
  if (p.table) {
    for (int i = threadIdx.x; i < kKtabDoubles; i += blockDim.x) stab[i] = tab[i];
  }
  __syncthreads();
}

// Pairs [pair0, pair0 + kGenPairsPerBlock) of tile (ti, tj), column-major with
// ld ts: thread t writes rows (r, r+1) of column c for pair = pair0 + i*256 + t,
// e = 2*pair = c*ts + r, with one vector store (FP64 tiles: a warp stores 512
// contiguous bytes; FP32 tiles, rounded from the FP64 value: 256 bytes).
// Rows/columns past n are padding: identity on the diagonal, 0 elsewhere.  x and
// y hold the problem's padded locations (nt*ts entries).
template <typename Out>
__device__ __forceinline__ void matern_tile_pairs(Out* __restrict__ tile, const double* __restrict__ x,
                                                  const double* __restrict__ y, int n, int ts, int ti, int tj,
                                                  long long pair0, const MaternParams& p,
                                                  const double* __restrict__ tab) {
  const long long pairs_per_tile = (long long)ts * ts / 2;
#pragma unroll 1
  for (int i = 0; i < kGenPairsPerThread; ++i) {
    const long long pair = pair0 + i * kGenThreads + threadIdx.x;
    if (pair >= pairs_per_tile) return;
    const long long e = pair * 2;
    const int c = (int)(e / ts);
    const int r = (int)(e - (long long)c * ts);
    const int gr = ti * ts + r;
    const int gc = tj * ts + c;
    double v0, v1;
    if (gc >= n) {
      v0 = (gr == gc) ? 1.0 : 0.0;
      v1 = (gr + 1 == gc) ? 1.0 : 0.0;
    } else {
      const double xc = x[gc], yc = y[gc];
      const double2 xr = *reinterpret_cast<const double2*>(x + gr);
      const double2 yr = *reinterpret_cast<const double2*>(y + gr);
      v0 = (gr < n) ? matern_from_dist_tab(euclid_dist(xr.x, yr.x, xc, yc), p, tab) : 0.0;
      v1 = (gr + 1 < n) ? matern_from_dist_tab(euclid_dist(xr.y, yr.y, xc, yc), p, tab) : 0.0;
    }
    if constexpr (sizeof(Out) == 8) {
      *reinterpret_cast<double2*>(tile + e) = make_double2(v0, v1);
    } else {
      *reinterpret_cast<float2*>(tile + e) = make_float2((float)v0, (float)v1);
    }
  }
}

}  // namespace egs
