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

// Cholesky of the 64x64 block at T (ld ts).  Every thread of the block (NTHR,
// whole warps) takes part in moving the block between global and shared memory,
// with all loads issued before any is used.  Up to eight warps factor it; lane
// l of each owns rows l and l + 32, and warp w the columns c with c % CW == w.
// At step j every warp scales column j with the reciprocal pivot and applies
// the rank-1 update to its columns c > j; the owner of column j + 1 updates
// that column first and computes the next pivot's square root and reciprocal
// before the step's barrier, so no warp waits on them after it.  Warp 0 stores
// the scaled column j after the barrier (no warp reads it again).  info
// records the 1-based global column (gcol0 + j + 1) of the first pivot that is
// not positive (or NaN).
template <int NTHR>
__device__ __forceinline__ void potrf64_body(double* __restrict__ T, int ts, int gcol0, int* __restrict__ info) {
  static_assert(NTHR % 32 == 0 && NTHR >= 32 && NTHR <= 1024, "whole warps");
  __shared__ double S[kNB][kNB + 1];
  __shared__ double piv[kNB], pinv[kNB];  // L_jj and 1 / L_jj
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
  if (threadIdx.x == 0) {
    const double d = S[0][0];
    if (!(d > 0.0)) atomicCAS(info, 0, gcol0 + 1);
    const double ljj = sqrt(d);
    piv[0] = ljj;
    pinv[0] = __drcp_rn(ljj);  // correctly rounded, as 1.0 / ljj
  }
  __syncthreads();
  constexpr int CW = NTHR / 32 < 8 ? NTHR / 32 : 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = lane, r1 = lane + 32;
  for (int j = 0; j < kNB; ++j) {
    double l0 = 0.0, l1 = 0.0;
    if (warp < CW) {
      const double inv = pinv[j];
      l0 = (r0 > j) ? S[r0][j] * inv : 0.0;
      l1 = (r1 > j) ? S[r1][j] * inv : 0.0;
      // first column of this warp after j
      int c1 = j + 1 + ((warp - (j + 1)) % CW + CW) % CW;
      if (c1 == j + 1 && c1 < kNB) {
        const double lcj = S[c1][j] * inv;
        if (r0 >= c1) S[r0][c1] = fma(-l0, lcj, S[r0][c1]);
        if (r1 >= c1) S[r1][c1] = fma(-l1, lcj, S[r1][c1]);
        __syncwarp();
        if (lane == 0) {
          const double d = S[c1][c1];
          if (!(d > 0.0)) atomicCAS(info, 0, gcol0 + c1 + 1);
          const double ljj = sqrt(d);
          piv[c1] = ljj;
          pinv[c1] = __drcp_rn(ljj);
        }
        c1 += CW;
      }
#pragma unroll 4
      for (int c = c1; c < kNB; c += CW) {
        const double lcj = S[c][j] * inv;
        if (r0 >= c) S[r0][c] = fma(-l0, lcj, S[r0][c]);
        if (r1 >= c) S[r1][c] = fma(-l1, lcj, S[r1][c]);
      }
    }
    __syncthreads();
    if (warp == 0) {
      if (r0 > j) S[r0][j] = l0;
      if (r1 > j) S[r1][j] = l1;
      if (r0 == j) S[r0][j] = piv[j];
      if (r1 == j) S[r1][j] = piv[j];
    }
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
