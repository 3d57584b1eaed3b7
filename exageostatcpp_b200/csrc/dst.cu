// Diagonal super-tile (band) approximation on the caller's tiles when they are
// not device tiles (dts not a multiple of 64): the factorisation of
// ChameleonDST<T>::ExaGeoStatParallelPotrfDiagonal (src/linear-algebra-solvers/
// concrete/chameleon/dst/ChameleonDST.cpp:90-150, lower case) on logical tiles
// of dts elements, element by element inside the lower-tile pool of device
// tiles (ts, a multiple of 64).  Which elements are factored, solved and
// updated depends only on the logical tiles, so the result is the reference's
// for any dts.  The device-tile path (dts == ts) stays in capi.cu; this one
// serves small or odd caller tiles such as the reference's dts = 8 tests.
#include <algorithm>
#include <cmath>
#include "common.cuh"
#include "kernels.cuh"

namespace egs {

// Element (i, j), i >= j, of the pool: tile (i / ts, j / ts), column-major inside.
__device__ __forceinline__ long long dst_elem(int ts, int nt, int i, int j) {
  return (tile_slot(i / ts, j / ts, nt) * ts + (j % ts)) * (long long)ts + (i % ts);
}

// Cholesky of the w x w logical diagonal tile at (c0, c0), right-looking, one
// column per iteration (dpotrf of tile (k, k)).  info records the 1-based global
// column of the first pivot that is not positive (or NaN).
__global__ void __launch_bounds__(256)
dst_potrf_kernel(double* __restrict__ a, int ts, int nt, int c0, int w, int* __restrict__ info) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  __shared__ double inv;
#pragma unroll 1
  for (int j = 0; j < w; ++j) {
    const int gj = c0 + j;
    if (threadIdx.x == 0) {
      const double d = a[dst_elem(ts, nt, gj, gj)];
      if (!(d > 0.0)) atomicCAS(info, 0, gj + 1);
      const double l = sqrt(d);
      a[dst_elem(ts, nt, gj, gj)] = l;
      inv = 1.0 / l;
    }
    __syncthreads();
    for (int r = j + 1 + threadIdx.x; r < w; r += blockDim.x) a[dst_elem(ts, nt, c0 + r, gj)] *= inv;
    __syncthreads();
    // trailing block: A(r, c) -= A(r, j) A(c, j), j < c <= r < w; one warp per column
    for (int c = j + 1 + warp; c < w; c += nwarps) {
      const double lcj = a[dst_elem(ts, nt, c0 + c, gj)];
      for (int r = c + lane; r < w; r += 32) {
        const long long e = dst_elem(ts, nt, c0 + r, c0 + c);
        a[e] = fma(-a[dst_elem(ts, nt, c0 + r, gj)], lcj, a[e]);
      }
    }
    __syncthreads();
  }
}

// X := A L^-T for rows [r0, r1) of the logical tile column at c0 (width w), L the
// factored diagonal tile (dtrsm Right/Lower/Trans/NonUnit): one thread per row,
// forward substitution in place.
__global__ void __launch_bounds__(128)
dst_trsm_kernel(double* __restrict__ a, int ts, int nt, int c0, int w, int r0, int r1) {
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= r1) return;
#pragma unroll 1
  for (int j = 0; j < w; ++j) {
    double v = a[dst_elem(ts, nt, r, c0 + j)];
#pragma unroll 4
    for (int q = 0; q < j; ++q) v = fma(-a[dst_elem(ts, nt, r, c0 + q)], a[dst_elem(ts, nt, c0 + j, c0 + q)], v);
    a[dst_elem(ts, nt, r, c0 + j)] = v / a[dst_elem(ts, nt, c0 + j, c0 + j)];
  }
}

// Update of step k (logical tile column at kc0, width kw): every target (i, j)
// with j in logical tile c, k < c < min(ntl, k + band), and j <= i <
// min(n, min(ntl, c + band) * dts) takes A(i, j) -= sum_l A(i, l) A(j, l) over
// the kw columns of tile k (dsyrk of (c, c), dgemm of (m, c)).  Tile (m, k) is
// read whether or not step k solved it.  One block per target column.
__global__ void __launch_bounds__(128)
dst_update_kernel(double* __restrict__ a, int ts, int nt, int n, int dts, int ntl, int band, int j0, int kc0,
                  int kw) {
  const int j = j0 + blockIdx.x;
  const int c = j / dts;
  const int iend = min(n, min(ntl, c + band) * dts);
  for (int i = j + threadIdx.x; i < iend; i += blockDim.x) {
    double acc = 0.0;
#pragma unroll 4
    for (int l = 0; l < kw; ++l)
      acc = fma(a[dst_elem(ts, nt, i, kc0 + l)], a[dst_elem(ts, nt, j, kc0 + l)], acc);
    const long long e = dst_elem(ts, nt, i, j);
    a[e] -= acc;
  }
}

int launch_dst_band(double* tiles, int ts, int nt, int n, int dts, int band, int* info, cudaStream_t st) {
  if (dts <= 0 || band <= 0 || n <= 0) return EGS_ERR_INVALID;
  const int ntl = (n + dts - 1) / dts;
  for (int k = 0; k < ntl; ++k) {
    const int c0 = k * dts;
    const int w = std::min(dts, n - c0);
    dst_potrf_kernel<<<1, 256, 0, st>>>(tiles, ts, nt, c0, w, info);
    const int mend = std::min(ntl, k + band);  // solved tiles: k < m < mend
    const int r0 = (k + 1) * dts, r1 = std::min(n, mend * dts);
    if (r1 > r0) {
      dst_trsm_kernel<<<(r1 - r0 + 127) / 128, 128, 0, st>>>(tiles, ts, nt, c0, w, r0, r1);
      // targets: the columns of tiles k+1 .. mend-1
      dst_update_kernel<<<r1 - r0, 128, 0, st>>>(tiles, ts, nt, n, dts, ntl, band, r0, c0, w);
    }
  }
  return launch_status("launch_dst_band");
}

}  // namespace egs
