// Per-row scales and the two splittings of a solved panel row used by the
// mixed-precision updates: FP16 hi/lo parts for the split-FP16 tcgen05 update
// and signed 7-bit slices for the Ozaki int8 products.  Shared by the slicing
// kernels (ozaki_band.cu) and the FP16 split of the DMMA form (split_gemm.cu).
#pragma once
#include <cuda_fp16.h>
#include <cstdint>

namespace egs {

constexpr int kOzSlices = 7;  // signed 7-bit slices per value (2^-49 of the row maximum)
// Slices of the off-band panel solve (FP32-stored rows times rows of L_kk^-1):
// 2^-42 of the row maxima.  The product with the inverse can cancel by the
// size of L_kk^-1's entries (10^4 to 10^5 for smooth kernels), which 2^-42
// still keeps below the FP32 rounding the solved rows get in storage.
constexpr int kOzPanelSlices = 6;

// FP16 split scale of a row with maximum m: inv_scale = 2^(e - 13) for
// 2^e <= m < 2^(e+1), so the scaled row lies below 2^14; rows whose maximum is
// 0 (or below 2^-120) get 0 and split to zeros; NaN or Inf rows get NaN.
__device__ __forceinline__ float f16_row_inv_scale(double m) {
  const long long bits = __double_as_longlong(m);
  const int e = (int)((bits >> 52) & 0x7FF) - 1023;
  if (e == 1024) return __int_as_float(0x7fc00000);  // NaN or Inf in the row: propagate
  if (!(m > 0.0) || e < -120) return 0.0f;
  return __int_as_float((e - 13 + 127) << 23);  // 2^(e-13), finite for e <= 140
}

// Ozaki row scale: 2^e with m < 2^e (the scaled row lies in (-1, 1)); 0 rows
// get 0, NaN rows NaN.
__device__ __forceinline__ double oz_row_scale(double m) {
  if (!(m > 0.0)) return (m == 0.0) ? 0.0 : __longlong_as_double(0x7ff8000000000000ll);
  const long long bits = __double_as_longlong(m);
  const int e = (int)((bits >> 52) & 0x7FF) - 1023;  // 2^e <= m < 2^(e+1) for normal m
  return (e >= 1023) ? __longlong_as_double(0x7ff8000000000000ll) : ldexp(1.0, e + 1);
}

// The first NP (at most seven) signed 7-bit slices of 16 scaled values
// (|v| < 1), one 16-byte store per slice: slice p (1..NP) of v is sign(v) * (floor(|v| 2^(7p)) mod 2^7),
// read off the truncated 49-bit fixed-point magnitude floor(|v| 2^49), which
// is the double's significand shifted by its exponent.  These are the values
// the repeated exact steps a_p = trunc(2^7 v), v <- 2^7 v - a_p give; the
// integer form keeps the slicing off the FP64 pipe.  Zero, subnormal and
// non-finite inputs give zero slices.
template <int NP = kOzSlices>
__device__ __forceinline__ void oz_emit_slices(const double (&v)[16], int8_t* dst, long long slice_stride) {
  static_assert(NP >= 1 && NP <= kOzSlices, "slices of the 49-bit magnitude");
  unsigned long long mag[16];
  unsigned neg = 0;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v[c]);
    const int ex = (int)((b >> 52) & 0x7FF);
    const unsigned long long sig = (b & 0xFFFFFFFFFFFFFull) | (1ull << 52);
    const int sh = 1026 - ex;  // |v| = sig 2^(ex - 1075), so floor(|v| 2^49) = sig >> (1026 - ex)
    mag[c] = (ex == 0 || ex > 1022 || sh > 52) ? 0ull : (sig >> sh);
    neg |= (unsigned)(b >> 63) << c;
  }
#pragma unroll
  for (int p = 1; p <= NP; ++p) {
    union {
      int8_t b[16];
      int4 q;
    } out;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int s = (int)((mag[c] >> (49 - 7 * p)) & 127u);
      out.b[c] = (int8_t)(((neg >> c) & 1u) ? -s : s);
    }
    *reinterpret_cast<int4*>(dst + (p - 1) * slice_stride) = out.q;
  }
}

// hi = fp16(v), lo = fp16(v - hi) of 16 scaled values, two 16-byte stores each.
__device__ __forceinline__ void f16_emit_split(const double (&v)[16], __half* hi, __half* lo) {
  union {
    __half h[16];
    int4 q[2];
  } H, L;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const __half h = __double2half(v[c]);
    H.h[c] = h;
    L.h[c] = __double2half(v[c] - (double)__half2float(h));
  }
  reinterpret_cast<int4*>(hi)[0] = H.q[0];
  reinterpret_cast<int4*>(hi)[1] = H.q[1];
  reinterpret_cast<int4*>(lo)[0] = L.q[0];
  reinterpret_cast<int4*>(lo)[1] = L.q[1];
}

}  // namespace egs
