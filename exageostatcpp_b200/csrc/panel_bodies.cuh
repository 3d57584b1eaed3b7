// Device bodies of the panel, solve and reduction kernels, shared by the
// single-problem kernels (potrf.cu) and the batched kernels (batch.cu).  Each
// body works on one tile (or one 64x64 block) given by pointers, so a kernel
// only has to locate its tile.
#pragma once
#include "common.cuh"

namespace egs {

constexpr int kNB = 64;  // inner block width of the panel factorisation

__device__ __forceinline__ double block_sum_256(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  const double out = red[0];
  __syncthreads();
  return out;
}

// Cholesky of the 64x64 block at T (ld ts), blocked by 16 columns.  Every
// thread of the block (NTHR, whole warps, at least two) takes part in moving
// the block between global and shared memory, with all loads issued before any
// is used.  For each 16-column block: (1) warp 0 factors the 16 x 16 diagonal
// block in registers (lane l holds row l; the pivot and the scaled column are
// exchanged with shuffles, so the 16 dependent pivot steps need no block-wide
// barrier); (2) one thread per row below it solves that row against the block
// (x_j = (a_j - sum_{q<j} x_q l_jq) / l_jj); (3) all threads update the rest
// of the 64 x 64 block with the 16 new columns.  Every element receives its
// multiply-adds in the same order (columns ascending) and every column the
// same scaling (by the correctly rounded reciprocal of the correctly rounded
// square root) as in the column-by-column right-looking factorisation, so the
// result is the same bit for bit; only the barriers are fewer (3 per 16
// columns instead of 2 per column).  info records the 1-based global column
// (gcol0 + j + 1) of the first pivot that is not positive (or NaN).
template <int NTHR>
__device__ __forceinline__ void potrf64_body(double* __restrict__ T, int ts, int gcol0, int* __restrict__ info) {
  static_assert(NTHR % 32 == 0 && NTHR >= 64 && NTHR <= 1024, "whole warps, at least two");
  constexpr int kSB = 16;  // sub-block width
  __shared__ double S[kNB][kNB + 1];
  __shared__ double pinv[kNB];  // 1 / L_jj
  constexpr int per = kNB * kNB / NTHR;
  {
    // column-major block: element e = c * 64 + r; all loads issued first
    double v[per];
#pragma unroll
    for (int q = 0; q < per; ++q) {
      const int e = q * NTHR + threadIdx.x;
      const int r = e & (kNB - 1), c = e >> 6;
      v[q] = (r >= c) ? T[(long long)c * ts + r] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < per; ++q) {
      const int e = q * NTHR + threadIdx.x;
      S[e & (kNB - 1)][e >> 6] = v[q];
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll 1
  for (int c0 = 0; c0 < kNB; c0 += kSB) {
    // (1) the diagonal sub-block, one warp, in registers
    if (warp == 0) {
      const int l = lane < kSB ? lane : kSB - 1;  // lanes 16..31 shadow lane 15 and write nothing
      double a[kSB];
#pragma unroll
      for (int q = 0; q < kSB; ++q) a[q] = (q <= l) ? S[c0 + l][c0 + q] : 0.0;
#pragma unroll
      for (int j = 0; j < kSB; ++j) {
        const double d = __shfl_sync(0xffffffffu, a[j], j);
        if (lane == j && !(d > 0.0)) atomicCAS(info, 0, gcol0 + c0 + j + 1);
        const double ljj = sqrt(d);
        const double inv = __drcp_rn(ljj);  // correctly rounded, as 1.0 / ljj
        if (l > j) a[j] *= inv;
        if (l == j) a[j] = ljj;
        if (lane == j) pinv[c0 + j] = inv;
#pragma unroll
        for (int c = 0; c < kSB; ++c) {
          if (c > j) {
            const double lcj = __shfl_sync(0xffffffffu, a[j], c);
            if (l >= c) a[c] = fma(-a[j], lcj, a[c]);
          }
        }
      }
      if (lane < kSB) {
#pragma unroll
        for (int q = 0; q < kSB; ++q)
          if (q <= lane) S[c0 + lane][c0 + q] = a[q];
      }
    }
    __syncthreads();
    const int rest = kNB - c0 - kSB;  // rows (and columns) after this sub-block
    if (rest == 0) break;
    // (2) the rows below the sub-block, one thread per row
    if ((int)threadIdx.x < rest) {
      const int r = c0 + kSB + threadIdx.x;
      double x[kSB];
#pragma unroll
      for (int j = 0; j < kSB; ++j) {
        double v = S[r][c0 + j];
#pragma unroll
        for (int q = 0; q < kSB; ++q)
          if (q < j) v = fma(-x[q], S[c0 + j][c0 + q], v);
        x[j] = v * pinv[c0 + j];
      }
#pragma unroll
      for (int j = 0; j < kSB; ++j) S[r][c0 + j] = x[j];
    }
    __syncthreads();
    // (3) the rest of the block: S(r, c) -= sum_q L(r, q) L(c, q), c0+16 <= c <= r
    const int cnt = rest * (rest + 1) / 2;
    for (int e = threadIdx.x; e < cnt; e += NTHR) {
      // e -> (r, c) with c <= r in the lower triangle of the rest, rows first
      int rr = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while (rr * (rr + 1) / 2 > e) --rr;
      while ((rr + 1) * (rr + 2) / 2 <= e) ++rr;
      const int cc = e - rr * (rr + 1) / 2;
      const int r = c0 + kSB + rr, c = c0 + kSB + cc;
      double v = S[r][c];
#pragma unroll
      for (int q = 0; q < kSB; ++q) v = fma(-S[r][c0 + q], S[c][c0 + q], v);
      S[r][c] = v;
    }
    __syncthreads();
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < per; ++q) {
    const int e = q * NTHR + threadIdx.x;
    const int r = e & (kNB - 1), c = e >> 6;
    if (r >= c) T[(long long)c * ts + r] = S[r][c];
  }
}

// X := A * L^-T for the 64 columns [col0, col0+64) of row `row` of tile A
// (ld ts); L is the factored 64x64 diagonal block at (col0, col0) of tile TL.
// Called by every thread of a 128-thread block (rows past ts just return).
// Right-looking: once x_c is final, it is applied to every later column, so
// the multiply-adds of a step are independent; each x_c still receives its
// terms in the order q = 0 .. c-1, as in forward substitution.
template <int NTHR>
__device__ __forceinline__ void trsm_rows_body(double* __restrict__ A, const double* __restrict__ TL, int ts,
                                               int row, int col0) {
  __shared__ __align__(16) double LT[kNB][kNB];  // LT[c][r] = L(r, c): column c of L
  __shared__ double invd[kNB];
  {
    // the 64 x 64 block, all loads issued before any is used
    constexpr int per = kNB * kNB / NTHR;
    double v[per];
#pragma unroll
    for (int q = 0; q < per; ++q) {
      const int e = q * NTHR + threadIdx.x;
      const int rr = e & (kNB - 1), c = e >> 6;
      v[q] = (rr >= c) ? TL[(long long)(col0 + c) * ts + col0 + rr] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < per; ++q) {
      const int e = q * NTHR + threadIdx.x;
      LT[e >> 6][e & (kNB - 1)] = v[q];
    }
  }
  __syncthreads();
  if (threadIdx.x < kNB) invd[threadIdx.x] = 1.0 / LT[threadIdx.x][threadIdx.x];
  __syncthreads();
  if (row >= ts) return;
  double* a = A + (long long)col0 * ts + row;
  double x[kNB];
#pragma unroll
  for (int c = 0; c < kNB; ++c) x[c] = a[(long long)c * ts];
#pragma unroll
  for (int c = 0; c < kNB; ++c) {
    x[c] *= invd[c];
    const double xc = x[c];
    if (c + 1 < kNB && ((c + 1) & 1)) x[c + 1] = fma(-xc, LT[c][c + 1], x[c + 1]);
#pragma unroll
    for (int q = (c + 2) & ~1; q < kNB; q += 2) {
      const double2 l2 = *reinterpret_cast<const double2*>(&LT[c][q]);
      x[q] = fma(-xc, l2.x, x[q]);
      x[q + 1] = fma(-xc, l2.y, x[q + 1]);
    }
  }
#pragma unroll
  for (int c = 0; c < kNB; ++c) a[(long long)c * ts] = x[c];
}

// Forward substitution on one diagonal tile T: zk := T^-1 zk (ts entries).
// Dynamic shared memory: ts doubles.
__device__ __forceinline__ void trsv_diag_body(const double* __restrict__ T, int ts, double* __restrict__ zk) {
  extern __shared__ double zs[];  // ts
  __shared__ double B[kNB][kNB + 1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int r = tid; r < ts; r += blockDim.x) zs[r] = zk[r];
  for (int kb = 0; kb < ts; kb += kNB) {
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
      const int rr = e % kNB, c = e / kNB;
      B[rr][c] = (rr >= c) ? T[(long long)(kb + c) * ts + kb + rr] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      double z0 = zs[kb + lane], z1 = zs[kb + 32 + lane];
      for (int c = 0; c < kNB; ++c) {
        double zc;
        if (c < 32) {
          if (lane == c) z0 = z0 / B[c][c];
          zc = __shfl_sync(0xffffffffu, z0, c);
        } else {
          if (lane == c - 32) z1 = z1 / B[c][c];
          zc = __shfl_sync(0xffffffffu, z1, c - 32);
        }
        if (lane > c) z0 = fma(-B[lane][c], zc, z0);
        if (lane + 32 > c) z1 = fma(-B[lane + 32][c], zc, z1);
      }
      zs[kb + lane] = z0;
      zs[kb + 32 + lane] = z1;
    }
    __syncthreads();
    for (int r = kb + kNB + tid; r < ts; r += blockDim.x) {
      const double* col = T + (long long)kb * ts + r;
      double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
#pragma unroll 4
      for (int c = 0; c < kNB; c += 4) {
        acc0 = fma(col[(long long)c * ts], zs[kb + c], acc0);
        acc1 = fma(col[(long long)(c + 1) * ts], zs[kb + c + 1], acc1);
        acc2 = fma(col[(long long)(c + 2) * ts], zs[kb + c + 2], acc2);
        acc3 = fma(col[(long long)(c + 3) * ts], zs[kb + c + 3], acc3);
      }
      zs[r] -= (acc0 + acc1) + (acc2 + acc3);
    }
    __syncthreads();
  }
  for (int r = tid; r < ts; r += blockDim.x) zk[r] = zs[r];
}

// zi -= T zk for the 64 rows of block rblk of tile T (256 threads = 64 rows x
// 4 column groups, fixed reduction order, FP64 arithmetic whatever the tile's
// storage type).  Dynamic shared memory: ts doubles.
template <typename Tile>
__device__ __forceinline__ void gemv_panel_body(const Tile* __restrict__ T, int ts, const double* __restrict__ zk,
                                                double* __restrict__ zi, int rblk) {
  extern __shared__ double zks[];  // ts
  __shared__ double red[4][kNB];
  for (int c = threadIdx.x; c < ts; c += blockDim.x) zks[c] = zk[c];
  __syncthreads();
  const int rl = threadIdx.x % kNB, g = threadIdx.x / kNB;
  const int r = rblk * kNB + rl;
  double acc = 0.0;
  if (r < ts) {
    for (int c = g; c < ts; c += 4) acc = fma((double)T[(long long)c * ts + r], zks[c], acc);
  }
  red[g][rl] = acc;
  __syncthreads();
  if (g == 0 && r < ts) zi[r] -= ((red[0][rl] + red[1][rl]) + red[2][rl]) + red[3][rl];
}

// Sum over the first `rows` diagonal entries of tile T of log L_rr (L_rr > 0
// only, dmdet-codelet.cpp:76-77); 256 threads.
__device__ __forceinline__ double logdet_tile_body(const double* __restrict__ T, int ts, int rows) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const double d = T[(long long)r * ts + r];
    if (d > 0.0) acc += log(d);
  }
  return block_sum_256(acc, red);
}

// result[0..3] = (log-likelihood, log|C|, Z^T C^-1 Z, info) of one problem
// (ChameleonImplementation.cpp:188-192, :257-265); 256 threads, fixed order.
__device__ __forceinline__ void finalize_body(const double* __restrict__ partial, int nt, const double* __restrict__ z,
                                              int n, double* __restrict__ result, const int* __restrict__ info) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) acc = fma(z[r], z[r], acc);
  const double dot = block_sum_256(acc, red);
  if (threadIdx.x == 0) {
    double det = 0.0;
    for (int k = 0; k < nt; ++k) det += partial[k];
    const double logdet = 2.0 * det;
    const double pi = 3.141592653589793;
    const double nn = (double)n;
    result[0] = -0.5 * dot - 0.5 * logdet - (double)(nn / 2.0) * log(2.0 * pi);
    result[1] = logdet;
    result[2] = dot;
    result[3] = (double)(info ? *info : 0);
  }
}

}  // namespace egs
