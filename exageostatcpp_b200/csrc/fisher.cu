// Fisher information of the Matern parameters on the GPU.
//
// The reference (LinearAlgebraMethods<T>::ExaGeoStatFisherTile,
// src/linear-algebra-solvers/LinearAlgebraMethods.cpp:1133-1306) forms
//     A_jk = 1/2 tr(C^-1 C_j C^-1 C_k),   C_j = dC/dtheta_j,
// with two triangular solves per derivative and one dense product plus a
// trace per pair, and returns A^-1.  Here the same quantity is computed as
//     A_jk = 1/2 sum(M_j o M_k),   M_j = L^-1 C_j L^-T  (symmetric),
// which needs no N^3 product per pair.  M_j comes from two partial tiled
// Cholesky factorisations of the augmented matrix [[C, .], [B, I]]: the first
// nt tile steps leave B L^-T in the lower-left block, so B = C_j gives
// Y = C_j L^-T and then B = Y^T = L^-1 C_j gives L^-1 C_j L^-T = M_j.  Everything runs on
// the library's own tile kernels (64x64 potrf, row solves, DMMA updates).
//
// Derivative kernels (src/kernels/concrete/UnivariateMaternDdsigmaSquare.cpp,
// UnivariateMaternDbeta.cpp, UnivariateMaternDnu.cpp): at scaled distance
// x = d / beta > 0, with c = 1 / (2^(nu-1) Gamma(nu)),
//     dC/dsigma2 = c x^nu K_nu(x)                                 (1 at x = 0)
//     dC/dbeta   = sigma2 c [-nu/beta x^nu K_nu - x^nu (nu/x K_nu - K_nu+1) x/beta]
//     dC/dnu     = sigma2 [-2 ln2 2^-nu / Gamma(nu) x^nu K_nu + 2^(1-nu) (-psi(nu)/Gamma(nu) x^nu K_nu
//                          + (x^nu ln x K_nu + x^nu dK_nu/dnu) / Gamma(nu))]  (0 at x = 0).
// The reference differentiates K_nu in nu by a forward difference with step
// 1e-9 (src/helpers/BasselFunction.cpp:23-33); here central differences at
// steps 1e-3 and 5e-4 over the library's K_nu (Temme series / Steed CF2,
// ~1e-13 relative), combined by Richardson extrapolation, give dK/dnu to
// ~1e-9, well inside the reference's own noise.
#include <cmath>
#include <memory>
#include <vector>
#include "common.cuh"
#include "kernels.cuh"

namespace egs {

// K_nu(x) and K_{nu+1}(x) for any nu >= 0, x > 0 (unscaled).
__device__ __forceinline__ void bessel_k_pair(double nu, double x, double& knu, double& knu1) {
  const int n = (int)floor(nu + 0.5);
  const double mu = nu - n;
  double k0, k1;
  bool scaled;
  if (x <= 2.0) {
    k_temme_series(mu, x, k0, k1);
    scaled = false;
  } else {
    k_steed_cf2_scaled(mu, x, k0, k1);
    scaled = true;
  }
  double v = mu + 1.0;
  for (int j = 0; j < n; ++j) {  // (K_mu+j, K_mu+j+1) -> (K_mu+j+1, K_mu+j+2)
    const double k2 = k0 + (2.0 * v / x) * k1;
    k0 = k1;
    k1 = k2;
    v += 1.0;
  }
  if (scaled) {
    const double e = exp(-x);
    k0 *= e;
    k1 *= e;
  }
  knu = k0;
  knu1 = k1;
}

struct FisherParams {
  double sigma2, beta, nu;
  double con;    // 1 / (2^(nu-1) Gamma(nu))
  double ginv;   // 1 / Gamma(nu)
  double psi;    // digamma(nu)
};

// The three derivative matrices, dense column-major np x np (rows / columns
// past n are zero): d[j * np * np + c * np + r].
__global__ void __launch_bounds__(256)
matern_derivatives_kernel(const double* __restrict__ x, const double* __restrict__ y, int n, int np,
                          FisherParams q, double* __restrict__ d) {
  const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;
  const long long nn = (long long)np * np;
  if (idx >= nn) return;
  const int c = (int)(idx / np), r = (int)(idx - (long long)c * np);
  double ds = 0.0, db = 0.0, dn = 0.0;
  if (r < n && c < n) {
    const double e = euclid_dist(x[r], y[r], x[c], y[c]) / q.beta;
    if (e == 0.0) {
      ds = 1.0;
    } else {
      double k0, k1, kp, km, kq, kr, unused;
      bessel_k_pair(q.nu, e, k0, k1);
      // central differences at h and h/2 combined by Richardson extrapolation:
      // O(h^4) truncation, ~1e-13 / h rounding
      const double h = 1e-3;
      bessel_k_pair(q.nu + h, e, kp, unused);
      bessel_k_pair(q.nu - h, e, km, unused);
      bessel_k_pair(q.nu + 0.5 * h, e, kq, unused);
      bessel_k_pair(q.nu - 0.5 * h, e, kr, unused);
      const double d1 = (kp - km) / (2.0 * h), d2 = (kq - kr) / h;
      const double dk = (4.0 * d2 - d1) / 3.0;
      const double xn = pow(e, q.nu);
      ds = q.con * xn * k0;
      db = q.sigma2 * q.con * (-q.nu / q.beta * xn * k0 - xn * (q.nu / e * k0 - k1) * e / q.beta);
      dn = q.sigma2 * (-2.0 * log(2.0) * pow(2.0, -q.nu) * q.ginv * xn * k0 +
                       pow(2.0, 1.0 - q.nu) * (-q.psi * q.ginv * xn * k0 + (xn * log(e) * k0 + xn * dk) * q.ginv));
    }
  }
  d[idx] = ds;
  d[nn + idx] = db;
  d[2 * nn + idx] = dn;
}

// Lower tiles of the augmented 2nt x 2nt matrix [[C, .], [B, I]] from dense
// np x np column-major C (lower part used) and B.
// transB: take B transposed (B^T(r, c) = B[r * np + c]).
__global__ void __launch_bounds__(256)
augment_tiles_kernel(double* __restrict__ tiles, int ts, int nt, const double* __restrict__ C,
                     const double* __restrict__ B, int transB) {
  const int nt2 = 2 * nt;
  const long long slot = blockIdx.y;
  // slot -> (i, j) of the lower layout of nt2 tiles
  int j = 0;
  long long s = slot;
  while (s >= nt2 - j) {
    s -= nt2 - j;
    ++j;
  }
  const int i = j + (int)s;
  const long long np = (long long)nt * ts;
  double* t = tiles + slot * (long long)ts * ts;
  for (long long e = (long long)blockIdx.x * 256 + threadIdx.x; e < (long long)ts * ts; e += (long long)gridDim.x * 256) {
    const int c = (int)(e / ts), r = (int)(e - (long long)c * ts);
    double v;
    if (i < nt) {
      v = C[(long long)(j * ts + c) * np + i * ts + r];
    } else if (j < nt) {
      const long long br = (long long)(i - nt) * ts + r, bc = (long long)j * ts + c;
      v = transB ? B[br * np + bc] : B[bc * np + br];
    } else {
      v = (i == j && r == c) ? 1.0 : 0.0;
    }
    t[e] = v;
  }
}

// Dense np x np Y from the lower-left block tiles (nt + i, j).
__global__ void __launch_bounds__(256)
extract_block_kernel(const double* __restrict__ tiles, int ts, int nt, double* __restrict__ Y) {
  const long long np = (long long)nt * ts;
  const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;
  if (idx >= np * np) return;
  const int c = (int)(idx / np), r = (int)(idx - (long long)c * np);
  const int i = r / ts, j = c / ts;
  const long long slot = tile_slot(nt + i, j, 2 * nt);
  Y[idx] = tiles[slot * (long long)ts * ts + (long long)(c - j * ts) * ts + (r - i * ts)];
}

// Deterministic dot product of long vectors: per-block partial sums in a fixed
// order, then one block adds the partials in order.
__global__ void __launch_bounds__(256)
dot_partial_kernel(const double* __restrict__ a, const double* __restrict__ b, long long n,
                   double* __restrict__ partial) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
    acc = fma(a[i], b[i], acc);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int m, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += partial[i];
    *out = s;
  }
}

}  // namespace egs

using namespace egs;

namespace {

// digamma(x), x > 0: recurrence psi(x) = psi(x+1) - 1/x up to x >= 6, then the
// asymptotic series ln x - 1/(2x) - sum B_2k / (2k x^2k) (Abramowitz & Stegun 6.3.18).
double digamma(double x) {
  double r = 0.0;
  while (x < 6.0) {
    r -= 1.0 / x;
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  const double series = f * (1.0 / 12 - f * (1.0 / 120 - f * (1.0 / 252 - f * (1.0 / 240 - f * (1.0 / 132)))));
  return r + std::log(x) - 0.5 / x - series;
}

}  // namespace

namespace egs {
int enqueue_potrf_steps(egs_problem* p, int steps);
int problem_tiles(egs_problem* p, double** tiles, int* ts, int* nt, cudaStream_t* st);
}  // namespace egs

extern "C" int egs_fisher_host(int n, int dts, const double* x, const double* y, const double* theta,
                               double* fisher_inverse) {
  if (n <= 0 || dts <= 0 || !x || !y || !theta || !fisher_inverse) return EGS_ERR_INVALID;
  MaternParams mp;
  if (make_matern_params(theta, &mp) != EGS_OK) {
    set_last_error("theta outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "egs_fisher_host");
    return EGS_ERR_INVALID;
  }
  // the augmented problem: 2 np rows, tile ts
  egs_problem* probe = nullptr;
  int rc = egs_problem_create(&probe, n, dts);
  if (rc != EGS_OK) return rc;
  int nn = 0, ts = 0, nt = 0;
  long long bytes = 0;
  egs_problem_info(probe, &nn, &ts, &nt, &bytes);
  egs_problem_destroy(probe);
  const long long np = (long long)nt * ts;
  egs_problem* aug = nullptr;
  if ((rc = egs_problem_create(&aug, (int)(2 * np), ts)) != EGS_OK) return rc;
  std::unique_ptr<egs_problem, int (*)(egs_problem*)> guard(aug, egs_problem_destroy);
  double* tiles = nullptr;
  int ts2 = 0, nt2 = 0;
  cudaStream_t st = nullptr;
  problem_tiles(aug, &tiles, &ts2, &nt2, &st);
  if (ts2 != ts || nt2 != 2 * nt) {
    set_last_error("unexpected augmented layout", "egs_fisher_host");
    return EGS_ERR_INVALID;
  }
  const long long nn2 = np * np;
  double *dx = nullptr, *dy = nullptr, *C = nullptr, *D = nullptr, *M = nullptr, *part = nullptr, *dots = nullptr;
  const int nblk = 1184;
  auto cleanup = [&]() {
    cudaStreamSynchronize(st);
    for (void* b : {(void*)dx, (void*)dy, (void*)C, (void*)D, (void*)M, (void*)part, (void*)dots}) cudaFreeAsync(b, st);
    cudaStreamSynchronize(st);
  };
  if (cudaMallocAsync(&dx, np * sizeof(double), st) || cudaMallocAsync(&dy, np * sizeof(double), st) ||
      cudaMallocAsync(&C, nn2 * sizeof(double), st) || cudaMallocAsync(&D, 3 * nn2 * sizeof(double), st) ||
      cudaMallocAsync(&M, 3 * nn2 * sizeof(double), st) || cudaMallocAsync(&part, nblk * sizeof(double), st) ||
      cudaMallocAsync(&dots, 9 * sizeof(double), st)) {
    cudaGetLastError();
    cleanup();
    set_last_error("device allocation failed", "egs_fisher_host");
    return EGS_ERR_OOM;
  }
  cudaMemsetAsync(dx, 0, np * sizeof(double), st);
  cudaMemsetAsync(dy, 0, np * sizeof(double), st);
  cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dy, y, n * sizeof(double), cudaMemcpyHostToDevice, st);
  // C with identity padding, dense
  cudaMemsetAsync(C, 0, nn2 * sizeof(double), st);
  if ((rc = launch_matern_block(C, (int)np, n, n, dx, dy, dx, dy, mp, st)) != EGS_OK) {
    cleanup();
    return rc;
  }
  {
    std::vector<double> one(1, 1.0);
    for (long long r = n; r < np; ++r)
      cudaMemcpyAsync(C + r * np + r, one.data(), sizeof(double), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
  }
  FisherParams q;
  q.sigma2 = theta[0];
  q.beta = theta[1];
  q.nu = theta[2];
  q.ginv = 1.0 / std::tgamma(q.nu);
  q.con = 1.0 / (std::pow(2.0, q.nu - 1.0) * std::tgamma(q.nu));
  q.psi = digamma(q.nu);
  matern_derivatives_kernel<<<(unsigned)((nn2 + 255) / 256), 256, 0, st>>>(dx, dy, n, (int)np, q, D);
  const long long ntiles2 = lower_tiles(2 * nt);
  if (ntiles2 > 65535) {
    cleanup();
    set_last_error("the augmented matrix has more than 65535 tiles; use a larger dts", "egs_fisher_host");
    return EGS_ERR_INVALID;
  }
  const unsigned gx = (unsigned)std::min<long long>(64, ((long long)ts * ts + 255) / 256);
  for (int j = 0; j < 3; ++j) {
    // pass 1: B = C_j -> Y = C_j L^-T;  pass 2: B = Y^T = L^-1 C_j -> L^-1 C_j L^-T = M_j
    for (int pass = 0; pass < 2; ++pass) {
      const double* B = pass == 0 ? D + j * nn2 : M + j * nn2;
      augment_tiles_kernel<<<dim3(gx, (unsigned)ntiles2), 256, 0, st>>>(tiles, ts, nt, C, B, pass);
      if ((rc = enqueue_potrf_steps(aug, nt)) != EGS_OK) {
        cleanup();
        return rc;
      }
      extract_block_kernel<<<(unsigned)((nn2 + 255) / 256), 256, 0, st>>>(tiles, ts, nt, M + j * nn2);
    }
  }
  for (int j = 0; j < 3; ++j)
    for (int k = j; k < 3; ++k) {
      dot_partial_kernel<<<nblk, 256, 0, st>>>(M + j * nn2, M + k * nn2, nn2, part);
      sum_partials_kernel<<<1, 32, 0, st>>>(part, nblk, dots + 3 * j + k);
    }
  double h[9] = {};
  cudaMemcpyAsync(h, dots, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    set_last_error("a CUDA call failed", "egs_fisher_host");
    cleanup();
    return EGS_ERR_CUDA;
  }
  cleanup();
  // A (3 x 3, symmetric) and its inverse through a Cholesky factorisation
  double A[3][3];
  for (int j = 0; j < 3; ++j)
    for (int k = j; k < 3; ++k) A[j][k] = A[k][j] = 0.5 * h[3 * j + k];
  double L[3][3] = {};
  for (int j = 0; j < 3; ++j) {
    double s = A[j][j];
    for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
    if (!(s > 0.0)) {
      set_last_error("Fisher information not positive definite", "egs_fisher_host");
      return j + 1;
    }
    L[j][j] = std::sqrt(s);
    for (int i = j + 1; i < 3; ++i) {
      double t = A[i][j];
      for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
      L[i][j] = t / L[j][j];
    }
  }
  for (int c = 0; c < 3; ++c) {  // column c of A^-1: L L^T v = e_c
    double v[3] = {0, 0, 0};
    v[c] = 1.0;
    for (int i = 0; i < 3; ++i) {
      for (int k = 0; k < i; ++k) v[i] -= L[i][k] * v[k];
      v[i] /= L[i][i];
    }
    for (int i = 2; i >= 0; --i) {
      for (int k = i + 1; k < 3; ++k) v[i] -= L[k][i] * v[k];
      v[i] /= L[i][i];
    }
    for (int i = 0; i < 3; ++i) fisher_inverse[c * 3 + i] = v[i];
  }
  return EGS_OK;
}
