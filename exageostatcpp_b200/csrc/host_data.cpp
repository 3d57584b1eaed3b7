// Host-side synthetic inputs of the reference's data generator, as C ABI calls.
//
//  * egs_generate_locations: LocationGenerator<T>::GenerateLocations / SortLocations
//    (src/data-generators/LocationGenerator.cpp:25-123) with the Morton helpers
//    SpreadBits / ReverseSpreadBits (src/helpers/ByteHandler.cpp:19-47).  Like the
//    reference it draws from the C library's srand()/rand() (std::srand(seed) at
//    src/api/ExaGeoStat.cpp:75-76), so the global rand() state advances exactly as
//    the reference's does.
//  * egs_shuffle_split: the random hold-out split of the prediction module,
//    PredictionHelpers<T>::PickRandomPoints / Shuffle
//    (src/prediction/PredictionHelpers.cpp:23-168) for one variable: a
//    Fisher-Yates pass that draws j = i + rand() / (RAND_MAX / (n - i) + 1)
//    (:146) from the same global rand() state, after which the first n_miss
//    entries are held out and the rest observed.
//  * egs_dlarnv_normal: LAPACK DLARNV with IDIST = 3 on top of DLARUV, called by
//    GenerateObservationsVector with ISEED = {seed, seed, seed, 1}
//    (src/linear-algebra-solvers/LinearAlgebraMethods.cpp:347-364).  DLARUV is a
//    multiplicative congruential generator modulo 2^48 with multiplier
//    33952834046453 (G. S. Fishman, Math. Comp. 54 (1990) 331-344); the i-th value of a
//    batch of up to 128 is seed * a^i mod 2^48, the seed then advances to the last
//    value.  DLARNV draws 2*il uniforms per batch of il <= 64 normals and applies
//    Box-Muller: sqrt(-2 log u1) cos(2 pi u2).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include "exageostat_b200.h"

namespace {

uint64_t spread_bits(uint64_t v) {
  v &= 0xffffull;
  v = (v ^ (v << 24)) & 0x000000ff000000ffull;
  v = (v ^ (v << 12)) & 0x000f000f000f000full;
  v = (v ^ (v << 6)) & 0x0303030303030303ull;
  v = (v ^ (v << 3)) & 0x1111111111111111ull;
  return v;
}

uint64_t reverse_spread_bits(uint64_t v) {
  v &= 0x1111111111111111ull;
  v = (v ^ (v >> 3)) & 0x0303030303030303ull;
  v = (v ^ (v >> 6)) & 0x000f000f000f000full;
  v = (v ^ (v >> 12)) & 0x000000ff000000ffull;
  v = (v ^ (v >> 24)) & 0x000000000000ffffull;
  return v;
}

double uniform_jitter(double lo, double hi) {
  const double r = (double)std::rand() / (double)(1.0 + RAND_MAX);
  return r * (hi - lo) + lo;
}

constexpr uint64_t kMask48 = (1ull << 48) - 1;
constexpr uint64_t kMultiplier = 33952834046453ull;

}  // namespace

extern "C" {

EGS_API int egs_generate_locations(int n, int seed, int reseed, double* x, double* y) {
  if (n <= 0 || !x || !y) return EGS_ERR_INVALID;
  if (reseed) std::srand((unsigned)seed);
  const int root_n = (int)std::ceil(std::sqrt((double)n));
  int index = 0;
  for (int i = 0; i < root_n && index < n; ++i) {
    for (int j = 0; j < root_n && index < n; ++j) {
      x[index] = ((i + 1) - 0.5 + uniform_jitter(-0.4, 0.4)) / root_n;
      y[index] = ((j + 1) - 0.5 + uniform_jitter(-0.4, 0.4)) / root_n;
      ++index;
    }
  }
  std::vector<uint64_t> code(n);
  for (int i = 0; i < n; ++i) {
    const uint16_t qx = (uint16_t)(x[i] * (double)UINT16_MAX + .5);
    const uint16_t qy = (uint16_t)(y[i] * (double)UINT16_MAX + .5);
    code[i] = (spread_bits(qy) << 1) + spread_bits(qx);
  }
  std::sort(code.begin(), code.end());
  for (int i = 0; i < n; ++i) {
    x[i] = (double)reverse_spread_bits(code[i]) / (double)UINT16_MAX;
    y[i] = (double)reverse_spread_bits(code[i] >> 1) / (double)UINT16_MAX;
  }
  return EGS_OK;
}

EGS_API int egs_dlarnv_normal(const int* iseed, int n, double* out) {
  if (!iseed || n < 0 || (n > 0 && !out)) return EGS_ERR_INVALID;
  for (int i = 0; i < 4; ++i)
    if (iseed[i] < 0 || iseed[i] > 4095) return EGS_ERR_INVALID;
  if ((iseed[3] & 1) == 0) return EGS_ERR_INVALID;  // LAPACK requires ISEED(4) odd
  uint64_t state = ((uint64_t)iseed[0] << 36) | ((uint64_t)iseed[1] << 24) | ((uint64_t)iseed[2] << 12) |
                   (uint64_t)iseed[3];
  const double two_pi = 6.28318530717958647692528676655900576839;
  const double r48 = 1.0 / (double)(1ull << 48);
  double u[128];
  for (int iv = 0; iv < n; iv += 64) {
    const int il = std::min(64, n - iv);
    uint64_t s = state;
    for (int i = 0; i < 2 * il; ++i) {
      s = (s * kMultiplier) & kMask48;  // seed * a^(i+1) mod 2^48
      u[i] = (double)s * r48;
    }
    state = s;
    for (int i = 0; i < il; ++i) out[iv + i] = std::sqrt(-2.0 * std::log(u[2 * i])) * std::cos(two_pi * u[2 * i + 1]);
  }
  return EGS_OK;
}

EGS_API int egs_shuffle_split(int n, int n_miss, const double* z, const double* x, const double* y,
                              double* z_obs, double* x_obs, double* y_obs, double* z_miss, double* x_miss,
                              double* y_miss) {
  if (n <= 0 || n_miss < 0 || n_miss > n || !z || !x || !y) return EGS_ERR_INVALID;
  if ((n - n_miss > 0 && (!z_obs || !x_obs || !y_obs)) || (n_miss > 0 && (!z_miss || !x_miss || !y_miss)))
    return EGS_ERR_INVALID;
  std::vector<double> sz(z, z + n), sx(x, x + n), sy(y, y + n);
  for (int i = 0; i + 1 < n; ++i) {
    const int j = i + std::rand() / (RAND_MAX / (n - i) + 1);
    std::swap(sz[i], sz[j]);
    std::swap(sx[i], sx[j]);
    std::swap(sy[i], sy[j]);
  }
  for (int i = 0; i < n_miss; ++i) {
    z_miss[i] = sz[i];
    x_miss[i] = sx[i];
    y_miss[i] = sy[i];
  }
  for (int i = n_miss; i < n; ++i) {
    z_obs[i - n_miss] = sz[i];
    x_obs[i - n_miss] = sx[i];
    y_obs[i - n_miss] = sy[i];
  }
  return EGS_OK;
}

}  // extern "C"
