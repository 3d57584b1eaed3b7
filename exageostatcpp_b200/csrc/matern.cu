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
#include "matern_tile.cuh"

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
  p.table = (p.kind == 2 && nu <= kKtabMaxNu) ? 1 : 0;
  p.pad_ = 0;
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

// Chebyshev table of g(x) = e^x x^nu K_nu(x) for each problem whose nu needs one:
// block (interval, problem), thread j evaluates g at node j, then computes
// coefficient j of the interval's series (discrete cosine sum over the nodes).
__global__ void __launch_bounds__(kKtabDeg)
matern_ktab_kernel(const MaternParams* __restrict__ params, double* __restrict__ tab) {
  const MaternParams p = params[blockIdx.y];
  if (!p.table) return;
  __shared__ double f[kKtabDeg];
  const int idx = blockIdx.x, j = threadIdx.x;
  f[j] = matern_g_direct(ktab_node(idx, j), p);
  __syncthreads();
  double c = 0.0;
  for (int q = 0; q < kKtabDeg; ++q) c = fma(f[q], cospi((double)(j * (2 * q + 1)) / (2 * kKtabDeg)), c);
  c *= (j == 0 ? 1.0 : 2.0) / kKtabDeg;
  tab[blockIdx.y * (long long)kKtabDoubles + idx * kKtabStride + j] = c;
}

void launch_matern_ktab(const MaternParams* params, double* tab, int nproblems, cudaStream_t st) {
  matern_ktab_kernel<<<dim3(kKtabIntervals, nproblems), kKtabDeg, 0, st>>>(params, tab);
}

__global__ void __launch_bounds__(kGenThreads)
matern_tiles_kernel(double* __restrict__ tiles, const double* __restrict__ x, const double* __restrict__ y,
                    int n, int ts, int nt, long long slot_begin, const MaternParams* __restrict__ pp,
                    const double* __restrict__ tab) {
  __shared__ double stab[kKtabDoubles];
  const MaternParams p = *pp;
  stage_ktab(stab, tab, p);
  const long long slot = slot_begin + blockIdx.y;
  int ti, tj;
  slot_to_tile(slot, nt, ti, tj);
  matern_tile_pairs(tiles + slot * (long long)ts * ts, x, y, n, ts, ti, tj,
                    (long long)blockIdx.x * kGenPairsPerBlock, p, stab);
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
                        const MaternParams* p, double* ktab, cudaStream_t st) {
  launch_matern_ktab(p, ktab, 1, st);
  const long long pairs = (long long)ts * ts / 2;
  const unsigned gx = (unsigned)((pairs + kGenPairsPerBlock - 1) / kGenPairsPerBlock);
  const long long total = lower_tiles(nt);
  for (long long s0 = 0; s0 < total; s0 += 65535) {
    const unsigned gy = (unsigned)((total - s0) < 65535 ? (total - s0) : 65535);
    matern_tiles_kernel<<<dim3(gx, gy), kGenThreads, 0, st>>>(tiles, x, y, n, ts, nt, s0, p, ktab);
  }
  return launch_status("matern_tiles_kernel");
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
  return launch_status("matern_block_kernel");
}

}  // namespace egs
