// Modified Bessel function of the second kind K_nu(x) and the Matern correlation
// built on it, in FP64 for sm_100a.
//
// Replaces the per-element call  gsl_sf_bessel_Knu(nu, dist)  made by
// UnivariateMaternStationary<T>::GenerateCovarianceMatrix
// (src/kernels/concrete/UnivariateMaternStationary.cpp:61-62).  GSL itself is not
// part of the reference tree; the method below is the published one it also uses:
//
//  * nu = n + mu with n = floor(nu + 1/2), |mu| <= 1/2;
//  * x <= 2: Temme's series (N. M. Temme, "On the numerical evaluation of the
//    modified Bessel function of the third kind", J. Comput. Phys. 19 (1975)
//    324-337) for K_mu and K_{mu+1};
//  * x > 2: the continued fraction CF2 evaluated with Steed's algorithm
//    (I. J. Thompson and A. R. Barnett, J. Comput. Phys. 64 (1986) 490-509;
//    Temme 1975 section 3) giving e^x K_mu and e^x K_{mu+1};
//  * upward recurrence K_{v+1} = K_{v-1} + (2v/x) K_v (stable for K) to reach nu.
//
// Half-integer nu has the closed form K_{1/2}(x) = sqrt(pi/2x) e^-x, from which
// the recurrence gives every n + 1/2 exactly; nu = 1/2 reduces the Matern to
// sigma^2 exp(-x).
#pragma once
#include <cstdint>
#include "rgamma_series.h"

namespace egs {

// 1/Gamma(1+mu) and 1/Gamma(1-mu) combinations used by Temme's series.
__device__ __forceinline__ void temme_gammas(double mu, double& gam1, double& gam2,
                                             double& gampl, double& gammi) {
  const double m2 = mu * mu;
  // even part -> gam2, odd part -> -gam1 (Horner in mu^2 from the top term down).
  double ev = 0.0, od = 0.0;
#pragma unroll
  for (int k = EGS_RGAMMA_NTERMS - 2; k >= 0; k -= 2) {
    ev = ev * m2 + egs_rgamma_coeff[k];
    od = od * m2 + egs_rgamma_coeff[k + 1];
  }
  gam2 = ev;
  gam1 = -od;
  gampl = gam2 - mu * gam1;  // 1/Gamma(1+mu)
  gammi = gam2 + mu * gam1;  // 1/Gamma(1-mu)
}

// Temme's series: K_mu(x) and K_{mu+1}(x) for 0 < x <= 2, |mu| <= 1/2.
__device__ __forceinline__ void k_temme_series(double mu, double x, double& kmu, double& kmu1) {
  const double half_x = 0.5 * x;
  const double ln2x = -log(half_x);   // ln(2/x)
  const double sig = mu * ln2x;       // sigma = mu ln(2/x)
  double gam1, gam2, gampl, gammi;
  temme_gammas(mu, gam1, gam2, gampl, gammi);
  // mu*pi / sin(mu*pi) -> 1 as mu -> 0
  const double fact = (fabs(mu) < 1e-15) ? 1.0 : (mu * M_PI) / sinpi(mu);
  // sinh(sigma)/sigma -> 1 as sigma -> 0
  double shs;
  if (fabs(sig) < 1e-4) {
    const double s2 = sig * sig;
    shs = 1.0 + s2 * (1.0 / 6.0 + s2 * (1.0 / 120.0));
  } else {
    shs = sinh(sig) / sig;
  }
  const double es = exp(sig);
  double f = fact * (gam1 * cosh(sig) + gam2 * shs * ln2x);
  double p = 0.5 * es / gampl;
  double q = 0.5 / (es * gammi);
  double c = 1.0;
  const double d = half_x * half_x;
  double sum = f;
  double sum1 = p;
  const double mu2 = mu * mu;
  for (int k = 1; k < 200; ++k) {
    const double dk = (double)k;
    f = (dk * f + p + q) / (dk * dk - mu2);
    c *= d / dk;
    p /= (dk - mu);
    q /= (dk + mu);
    const double t = c * f;
    sum += t;
    const double t1 = c * (p - dk * f);
    sum1 += t1;
    if (fabs(t) < 1e-17 * fabs(sum)) break;
  }
  kmu = sum;
  kmu1 = sum1 * (2.0 / x);
}

// Steed's evaluation of CF2: e^x K_mu(x) and e^x K_{mu+1}(x) for x > 2, |mu| <= 1/2.
// The continued fraction for the ratio K_{mu+1}/K_mu is summed by forward
// recurrences (Steed), and the auxiliary series S = sum C_i Q_i (Temme) gives
// K_mu itself as sqrt(pi/2x) / S.
__device__ __forceinline__ void k_steed_cf2_scaled(double mu, double x, double& ks_mu, double& ks_mu1) {
  const double a1 = 0.25 - mu * mu;
  double bi = 2.0 * (1.0 + x);   // b_1
  double di = 1.0 / bi;          // D_1
  double delta_h = di;           // h_1 - h_0
  double h = di;                 // partial value of the fraction
  double qprev = 0.0, qcur = 1.0; // Q_0, Q_1
  double ai = -a1;               // a_1 with the sign folded in
  double ci = a1;                // C_1
  double qsum = a1;              // sum C_i Q_i, starting at C_1 Q_1 with Q_1 = 1
  double s = 1.0 + qsum * delta_h;
  for (int i = 2; i < 2000; ++i) {
    ai -= 2.0 * (double)(i - 1);
    ci = -ai * ci / (double)i;
    const double qnext = (qprev - bi * qcur) / ai;
    qprev = qcur;
    qcur = qnext;
    qsum += ci * qnext;
    bi += 2.0;
    di = 1.0 / (bi + ai * di);
    delta_h = (bi * di - 1.0) * delta_h;
    h += delta_h;
    const double ds = qsum * delta_h;
    s += ds;
    if (fabs(ds) < 1e-17 * fabs(s)) break;
  }
  h *= a1;
  ks_mu = sqrt(M_PI / (2.0 * x)) / s;
  ks_mu1 = ks_mu * (mu + x + 0.5 - h) / x;
}

// Parameters of one Matern evaluation (constant over a generation launch).
struct MaternParams {
  double sigma2;     // theta[0]
  double beta;       // theta[1]
  double nu;         // theta[2]
  double con;        // sigma2 / (2^(nu-1) Gamma(nu))
  double mu;         // nu - n
  int n;             // floor(nu + 1/2)
  int kind;          // 0: nu == 1/2, 1: half-integer, 2: general
  int table;         // 1: general nu <= kKtabMaxNu, evaluated through the Chebyshev table below
  int pad_;
};

// K_nu(x) for kind 2 (general nu): Temme's series (x <= 2, unscaled) or Steed's
// CF2 (x > 2, scaled by e^x, *scaled = true), then the upward recurrence.
__device__ __forceinline__ double bessel_k_general(double x, const MaternParams& p, bool& scaled) {
  double k0, k1;
  if (x <= 2.0) {
    k_temme_series(p.mu, x, k0, k1);
    scaled = false;
  } else {
    k_steed_cf2_scaled(p.mu, x, k0, k1);
    scaled = true;
  }
  if (p.n == 0) return k0;
  double v = p.mu + 1.0;
  for (int j = 1; j < p.n; ++j) {
    const double k2 = k0 + (2.0 * v / x) * k1;
    k0 = k1;
    k1 = k2;
    v += 1.0;
  }
  return k1;
}

// Matern covariance for scaled distance x = d / beta > 0:
// con * x^nu * K_nu(x)   (UnivariateMaternStationary.cpp:61-62).
__device__ __forceinline__ double matern_positive(double x, const MaternParams& p) {
  if (p.kind == 0) {
    return p.sigma2 * exp(-x);
  }
  if (p.kind == 1) {
    // e^x sqrt(2x/pi) K_{j+1/2}(x): r0 = 1 (j=0), r1 = 1 + 1/x (j=1), upward recurrence.
    double r0 = 1.0, r1 = 1.0 + 1.0 / x;
    const int nh = p.n;  // nu = nh + 1/2 (n = floor(nu + 1/2) = nh + 1, mu = -1/2)
    // K_{nu} with nu = (n-1) + 1/2
    double rv;
    if (nh - 1 == 0) {
      rv = r0;
    } else {
      for (int j = 1; j < nh - 1; ++j) {
        const double r2 = r0 + (2.0 * (j + 0.5) / x) * r1;
        r0 = r1;
        r1 = r2;
      }
      rv = r1;
    }
    // con * x^nu * sqrt(pi/2x) e^-x * rv
    return p.con * sqrt(M_PI / (2.0 * x)) * exp(p.nu * log(x) - x) * rv;
  }
  bool scaled;
  const double knu = bessel_k_general(x, p, scaled);
  if (scaled) {
    return p.con * exp(p.nu * log(x) - x) * knu;
  }
  return p.con * pow(x, p.nu) * knu;
}

// ---------------------------------------------------------------------------
// Piecewise Chebyshev table of g(x) = e^x x^nu K_nu(x) for general nu.
//
// For one theta the generator evaluates the same K_nu at millions of distances;
// the series/continued-fraction evaluation above costs thousands of FP64
// operations per element (divisions, data-dependent trip counts that diverge
// inside a warp).  Instead, per theta, g is interpolated on half-octave
// intervals [2^e, 2^e sqrt2), [2^e sqrt2, 2^(e+1)) for 2^-20 <= x < 2^9 by
// Chebyshev series of degree 15 whose coefficients come from the evaluation
// above at the 16 Chebyshev points of each interval (one small launch per
// theta).  g is analytic except for its branch point at 0, which lies
// (3 + 2 sqrt2) half-widths from each interval's centre, so the series
// converge like (5.83 + sqrt(5.83^2 - 1))^-k ~ 11.6^-k: the interpolant is
// within a few 1e-15 (relative) of g for nu <= 8 (checked against 30-digit
// values).  An element then costs one table lookup, a 16-term Clenshaw sum and
// one exp.  Distances outside [2^-20, 2^9) and nu > 8 use the direct
// evaluation.
constexpr int kKtabDeg = 16;     // coefficients per interval
constexpr int kKtabStride = 17;  // padded row: lanes reading different intervals hit different banks
constexpr int kKtabELo = -20, kKtabEHi = 9;
constexpr int kKtabIntervals = 2 * (kKtabEHi - kKtabELo);
constexpr int kKtabDoubles = kKtabIntervals * kKtabStride;
constexpr double kKtabMaxNu = 8.0;
// t = x * 2^-e * S_h + C maps interval (e, h) onto [-1, 1]:
// h = 0: S = 2 / (sqrt2 - 1) = 2 + 2 sqrt2; h = 1: S = 2 + sqrt2; C = -(3 + 2 sqrt2) for both.
constexpr double kKtabS0 = 4.8284271247461900976, kKtabS1 = 3.4142135623730950488;
constexpr double kKtabC = -5.8284271247461900976;
constexpr long long kSqrt2Mantissa = 0x6A09E667F3BCDLL;  // fraction bits of fl(sqrt 2)

// e^x x^nu K_nu(x) by the direct evaluation (kind 2).
__device__ __forceinline__ double matern_g_direct(double x, const MaternParams& p) {
  bool scaled;
  const double knu = bessel_k_general(x, p, scaled);
  if (scaled) return exp(p.nu * log(x)) * knu;
  return exp(x) * pow(x, p.nu) * knu;
}

// Interval and local coordinate of x > 0; false outside the tabulated range.
__device__ __forceinline__ bool ktab_locate(double x, int& idx, double& t) {
  const long long bits = __double_as_longlong(x);
  const int e = (int)(bits >> 52) - 1023;
  if (e < kKtabELo || e >= kKtabEHi) return false;
  const int h = (bits & 0xFFFFFFFFFFFFFLL) >= kSqrt2Mantissa ? 1 : 0;
  idx = 2 * (e - kKtabELo) + h;
  const double scale = __longlong_as_double((long long)(1023 - e) << 52);  // 2^-e, exact
  t = fma(x, scale * (h ? kKtabS1 : kKtabS0), kKtabC);
  return true;
}

// Node j (Chebyshev point of the first kind) of interval idx.
__device__ __forceinline__ double ktab_node(int idx, int j) {
  const int e = idx / 2 + kKtabELo, h = idx & 1;
  const double t = cospi((j + 0.5) / kKtabDeg);
  const double scale = __longlong_as_double((long long)(1023 + e) << 52);  // 2^e, exact
  return (t - kKtabC) / (h ? kKtabS1 : kKtabS0) * scale;
}

// Clenshaw sum of one interval's Chebyshev series at t.
__device__ __forceinline__ double ktab_sum(const double* __restrict__ c, double t) {
  const double t2 = 2.0 * t;
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int k = kKtabDeg - 1; k >= 1; --k) {
    const double b0 = fma(t2, b1, c[k] - b2);
    b2 = b1;
    b1 = b0;
  }
  return fma(t, b1, c[0] - b2);
}

// Euclidean distance sqrt(dx^2 + dy^2) with dx = x2 - x1, dy = y2 - y1, rounded
// like the reference's sqrt(pow(dx,2) + pow(dy,2)) (no fused multiply-add;
// DistanceCalculationHelpers.cpp:49-57).
__device__ __forceinline__ double euclid_dist(double x1, double y1, double x2, double y2) {
  const double dx = __dsub_rn(x2, x1);
  const double dy = __dsub_rn(y2, y1);
  return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

// Full Matern entry: x = dist / beta; sigma2 where x == 0 (exact compare,
// UnivariateMaternStationary.cpp:59-62), else the function above.
__device__ __forceinline__ double matern_from_dist(double dist, const MaternParams& p) {
  const double x = __ddiv_rn(dist, p.beta);
  return (x == 0.0) ? p.sigma2 : matern_positive(x, p);
}

// The same entry through the Chebyshev table tab (kKtabDoubles, any address
// space) when p.table is set.
__device__ __forceinline__ double matern_from_dist_tab(double dist, const MaternParams& p,
                                                       const double* __restrict__ tab) {
  const double x = __ddiv_rn(dist, p.beta);
  if (x == 0.0) return p.sigma2;
  int idx;
  double t;
  if (p.table && ktab_locate(x, idx, t)) return p.con * (ktab_sum(tab + idx * kKtabStride, t) * exp(-x));
  return matern_positive(x, p);
}

}  // namespace egs
