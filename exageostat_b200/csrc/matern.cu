// Matern covariance generation on sm_100a.
//
// Replaces the dcmg codelet loop (RuntimeFunctions<T>::CovarianceMatrix,
// src/runtime/starpu/StarPuFunctions.cpp:24-45 -> DCMGCodelet<T>::InsertTask,
// src/runtime/starpu/concrete/dcmg-codelet.cpp:41-75, one CPU task per lower
// tile) by one launch over every stored lower tile.  Each thread produces two
// consecutive rows of one column and writes them with a single 16-byte store, so
// a warp writes 512 contiguous bytes of a column-major tile.
#include <cmath>
#include "common.cuh"
#include "bessel_k.cuh"
#include "kernels.cuh"

namespace egs {

int make_matern_params(const double* theta, MaternParams* out) {
  const double sigma2 = theta[0], beta = theta[1], nu = theta[2];
  if (!(sigma2 > 0.0) || !(beta > 0.0) || !(nu > 0.0) || !std::isfinite(sigma2) ||
      !std::isfinite(beta) || !std::isfinite(nu) || nu > 1000.0) {
    return EGS_ERR_INVALID;
  }
  MaternParams p;
  p.sigma2 = sigma2;
  p.beta = beta;
  p.nu = nu;
  // Same host expression as UnivariateMaternStationary.cpp:47-49.
  p.con = sigma2 * (1.0 / (std::pow(2.0, (nu - 1.0)) * std::tgamma(nu)));
  p.n = (int)std::floor(nu + 0.5);
  p.mu = nu - p.n;
  if (nu == 0.5) {
    p.kind = 0;
  } else if (p.mu == -0.5) {
    p.kind = 1;
  } else {
    p.kind = 2;
  }
  *out = p;
  return EGS_OK;
}

// Column of the lower-tile slot s in an nt x nt tile grid.
__device__ __forceinline__ void slot_to_tile(long long s, int nt, int& ti, int& tj) {
  // start(j) = j*nt - j(j-1)/2; invert the quadratic, then correct by +-1.
  double b = 2.0 * nt + 1.0;
  int j = (int)floor((b - sqrt(b * b - 8.0 * (double)s)) * 0.5);
  if (j < 0) j = 0;
  if (j > nt - 1) j = nt - 1;
  while (j > 0 && tile_slot(j, j, nt) > s) --j;
  while (j < nt - 1 && tile_slot(j + 1, j + 1, nt) <= s) ++j;
  tj = j;
  ti = j + (int)(s - tile_slot(j, j, nt));
}

// One thread = rows (r, r+1) of column c of one lower tile.
template <typename Real>
__global__ void __launch_bounds__(256)
matern_tiles_kernel(Real* __restrict__ tiles, const double* __restrict__ x, const double* __restrict__ y,
                    int n, int ts, int nt, long long slot_begin, const MaternParams* __restrict__ pp) {
  const MaternParams p = *pp;
  const long long slot = slot_begin + blockIdx.y;
  int ti, tj;
  slot_to_tile(slot, nt, ti, tj);
  const long long pair = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long pairs_per_tile = (long long)ts * ts / 2;
  if (pair >= pairs_per_tile) return;
  const long long e = pair * 2;
  const int c = (int)(e / ts);
  const int r = (int)(e - (long long)c * ts);
  const int gr = ti * ts + r;
  const int gc = tj * ts + c;
  const double xc = x[gc], yc = y[gc];
  const double2 xr = *reinterpret_cast<const double2*>(x + gr);
  const double2 yr = *reinterpret_cast<const double2*>(y + gr);
  double v0, v1;
  if (gc >= n) {
    v0 = (gr == gc) ? 1.0 : 0.0;
    v1 = (gr + 1 == gc) ? 1.0 : 0.0;
  } else {
    v0 = (gr < n) ? matern_from_dist(euclid_dist(xr.x, yr.x, xc, yc), p) : 0.0;
    v1 = (gr + 1 < n) ? matern_from_dist(euclid_dist(xr.y, yr.y, xc, yc), p) : 0.0;
  }
  Real* dst = tiles + slot * (long long)ts * ts + e;
  if constexpr (sizeof(Real) == 8) {
    *reinterpret_cast<double2*>(dst) = make_double2(v0, v1);
  } else {
    *reinterpret_cast<float2*>(dst) = make_float2((float)v0, (float)v1);
  }
}

// Generic rows x cols column-major block (leading dimension lda) at global
// offsets (row_offset, col_offset) into two location sets; the Kernel plugin
// interface (Kernel<T>::GenerateCovarianceMatrix, inst/include/kernels/Kernel.hpp:93-97).
__global__ void __launch_bounds__(256)
matern_block_kernel(double* __restrict__ a, int lda, int rows, int cols, const double* __restrict__ x1,
                    const double* __restrict__ y1, const double* __restrict__ x2,
                    const double* __restrict__ y2, MaternParams p) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= rows) return;
  a[(long long)c * lda + r] = matern_from_dist(euclid_dist(x1[r], y1[r], x2[c], y2[c]), p);
}

int launch_matern_tiles(double* tiles, const double* x, const double* y, int n, int ts, int nt,
                        const MaternParams* p, cudaStream_t st) {
  const long long pairs = (long long)ts * ts / 2;
  const int threads = 256;
  const unsigned gx = (unsigned)((pairs + threads - 1) / threads);
  const long long total = lower_tiles(nt);
  for (long long s0 = 0; s0 < total; s0 += 65535) {
    const unsigned gy = (unsigned)((total - s0) < 65535 ? (total - s0) : 65535);
    matern_tiles_kernel<double><<<dim3(gx, gy), threads, 0, st>>>(tiles, x, y, n, ts, nt, s0, p);
  }
  return cudaGetLastError() == cudaSuccess ? EGS_OK : EGS_ERR_CUDA;
}

int launch_matern_block(double* a, int lda, int rows, int cols, const double* x1, const double* y1,
                        const double* x2, const double* y2, const MaternParams& p, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return EGS_OK;
  const int threads = 256;
  for (int c0 = 0; c0 < cols; c0 += 65535) {
    const int nc = (cols - c0) < 65535 ? (cols - c0) : 65535;
    matern_block_kernel<<<dim3((rows + threads - 1) / threads, nc), threads, 0, st>>>(
        a + (long long)c0 * lda, lda, rows, nc, x1, y1, x2 + c0, y2 + c0, p);
  }
  return cudaGetLastError() == cudaSuccess ? EGS_OK : EGS_ERR_CUDA;
}

}  // namespace egs
