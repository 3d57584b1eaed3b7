// Panel-level building blocks of the tiled Cholesky path on sm_100a: the 64x64
// diagonal-block factorisation, the row-parallel triangular solve of a 64-column
// block, the single right-hand-side forward/backward substitution over tiles,
// and the deterministic reductions that turn the factor into the log-likelihood.
//
// Reference counterparts:
//   CHAMELEON_dpotrf_Tile            ChameleonDense.cpp:25-37   (panel part; the trailing
//                                                                update is dgemm_tma.cu)
//   CHAMELEON_dtrsm_Tile (Z := L^-1 Z) ChameleonImplementation.cpp:337-347
//   DMDETCodelet::core_dmdet          dmdet-codelet.cpp:73-80   (sum of log L_kk, L_kk > 0)
//   DDOTPCodelet::cl_ddotp_function   ddotp-codelet.cpp:63-72   (Z^T Z)
//   log-likelihood assembly           ChameleonImplementation.cpp:257-265
//   DMSECodelet                       dmse-codelet.cpp:60-73    (sum (zhat - z)^2)
// Every reduction uses a fixed summation order, so a result does not depend on
// what else runs on the GPU.
#include <cmath>
#include "common.cuh"
#include "kernels.cuh"
#include "panel_bodies.cuh"

namespace egs {

// Cholesky of the 64x64 diagonal block at (off, off) of one tile (potrf64_body).
__global__ void __launch_bounds__(256)
potrf_diag_block_kernel(double* __restrict__ tiles, int ts, long long slot, int off, int col_base,
                        int* __restrict__ info) {
  potrf64_body<256>(tiles + slot * (long long)ts * ts + (long long)off * ts + off, ts, col_base + off, info);
}

void launch_potrf_diag_block(double* tiles, int ts, long long slot, int off, int col_base, int* info,
                             cudaStream_t st) {
  potrf_diag_block_kernel<<<1, 256, 0, st>>>(tiles, ts, slot, off, col_base, info);
}

// X := A * L^-T for the 64-column block [col0, col0+64) of ntiles consecutive
// tiles starting at slot0: rows [row0_first, ts) of the first tile and rows
// [row0, ts) of the others; L is the factored 64x64 diagonal block at (col0,
// col0) of tile lslot (trsm_rows_body).
__global__ void __launch_bounds__(128)
trsm_rows_kernel(double* __restrict__ tiles, int ts, long long slot0, int grid_row0, int row0_first, int row0,
                 int col0, long long lslot) {
  const int lo = blockIdx.y == 0 ? row0_first : row0;
  int row = grid_row0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (row < lo) row = ts;  // takes part in loading L only
  trsm_rows_body<128>(tiles + (slot0 + blockIdx.y) * (long long)ts * ts, tiles + lslot * (long long)ts * ts, ts,
                      row, col0);
}

void launch_trsm_rows(double* tiles, int ts, long long slot0, int ntiles, int row0, int col0,
                      long long lslot, cudaStream_t st) {
  launch_trsm_rows_panel(tiles, ts, slot0, ntiles, row0, row0, col0, lslot, st);
}

void launch_trsm_rows_panel(double* tiles, int ts, long long slot0, int ntiles, int row0_first, int row0, int col0,
                            long long lslot, cudaStream_t st) {
  if (ntiles <= 0) return;
  if (ntiles == 1) row0 = row0_first;
  const int first = row0 < row0_first ? row0 : row0_first;
  const int rows = ts - first;
  if (rows <= 0) return;
  const int threads = 128;
  trsm_rows_kernel<<<dim3((rows + threads - 1) / threads, ntiles), threads, 0, st>>>(tiles, ts, slot0, first,
                                                                                    row0_first, row0, col0, lslot);
}

// Forward substitution on one diagonal tile: z_k := L_kk^-1 z_k (trsv_diag_body).
__global__ void __launch_bounds__(1024)
trsv_diag_kernel(const double* __restrict__ tiles, int ts, long long slot, double* __restrict__ zk) {
  trsv_diag_body(tiles + slot * (long long)ts * ts, ts, zk);
}

void launch_trsv_diag(const double* tiles, int ts, long long slot, double* zk, cudaStream_t st) {
  trsv_diag_kernel<<<1, 1024, ts * sizeof(double), st>>>(tiles, ts, slot, zk);
}

// z_i -= L_ik z_k for every tile row i > k (gemv_panel_body).
__global__ void __launch_bounds__(256)
gemv_panel_kernel(const double* __restrict__ tiles, int ts, int nt, int k, double* __restrict__ z) {
  const int i = k + 1 + blockIdx.y;
  gemv_panel_body(tiles + tile_slot(i, k, nt) * (long long)ts * ts, ts, z + (long long)k * ts,
                  z + (long long)i * ts, blockIdx.x);
}

void launch_gemv_panel(const double* tiles, int ts, int nt, int k, double* z, cudaStream_t st) {
  if (k >= nt - 1) return;
  gemv_panel_kernel<<<dim3((ts + kNB - 1) / kNB, nt - 1 - k), 256, ts * sizeof(double), st>>>(tiles, ts, nt,
                                                                                          k, z);
}

// ---------------------------------------------------------------------------
// Backward substitution on one diagonal tile: z_k := L_kk^-T z_k.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
trsv_t_diag_kernel(const double* __restrict__ tiles, int ts, long long slot, double* __restrict__ zk) {
  extern __shared__ double zs[];
  __shared__ double B[kNB][kNB + 1];
  const double* T = tiles + slot * (long long)ts * ts;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int r = tid; r < ts; r += blockDim.x) zs[r] = zk[r];
  for (int kb = ts - kNB; kb >= 0; kb -= kNB) {
    for (int e = tid; e < kNB * kNB; e += blockDim.x) {
      const int rr = e % kNB, c = e / kNB;
      B[rr][c] = (rr >= c) ? T[(long long)(kb + c) * ts + kb + rr] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      double z0 = zs[kb + lane], z1 = zs[kb + 32 + lane];
      for (int c = kNB - 1; c >= 0; --c) {
        double zc;
        if (c >= 32) {
          if (lane == c - 32) z1 = z1 / B[c][c];
          zc = __shfl_sync(0xffffffffu, z1, c - 32);
        } else {
          if (lane == c) z0 = z0 / B[c][c];
          zc = __shfl_sync(0xffffffffu, z0, c);
        }
        // rows r < c: z_r -= L[c][r] x_c
        if (lane < c) z0 = fma(-B[c][lane], zc, z0);
        if (lane + 32 < c) z1 = fma(-B[c][lane + 32], zc, z1);
      }
      zs[kb + lane] = z0;
      zs[kb + 32 + lane] = z1;
    }
    __syncthreads();
    // rows r < kb: z_r -= sum_c L[kb+c][r] x[kb+c]; column r of L is contiguous in rows.
    for (int r = warp; r < kb; r += blockDim.x / 32) {
      const double* col = T + (long long)r * ts + kb;
      double acc = fma(col[lane], zs[kb + lane], col[lane + 32] * zs[kb + lane + 32]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) zs[r] -= acc;
    }
    __syncthreads();
  }
  for (int r = tid; r < ts; r += blockDim.x) zk[r] = zs[r];
}

void launch_trsv_t_diag(const double* tiles, int ts, long long slot, double* zk, cudaStream_t st) {
  trsv_t_diag_kernel<<<1, 256, ts * sizeof(double), st>>>(tiles, ts, slot, zk);
}

// z_i -= L_ki^T z_k for every tile column i < k (tile (k, i) is stored).  One warp per column.
__global__ void __launch_bounds__(256)
gemv_t_panel_kernel(const double* __restrict__ tiles, int ts, int nt, int k, double* __restrict__ z) {
  const int i = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + warp;
  if (c >= ts) return;
  const double* col = tiles + tile_slot(k, i, nt) * (long long)ts * ts + (long long)c * ts;
  const double* zk = z + (long long)k * ts;
  double acc = 0.0;
  for (int r = lane; r < ts; r += 32) acc = fma(col[r], zk[r], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) z[(long long)i * ts + c] -= acc;
}

void launch_gemv_t_panel(const double* tiles, int ts, int nt, int k, double* z, cudaStream_t st) {
  if (k <= 0) return;
  gemv_t_panel_kernel<<<dim3((ts + 7) / 8, k), 256, 0, st>>>(tiles, ts, nt, k, z);
}

// ---------------------------------------------------------------------------
// Deterministic reductions.
// ---------------------------------------------------------------------------
// partial[k] = sum over the real rows of diagonal tile k of log L_rr.
__global__ void __launch_bounds__(256)
logdet_partials_kernel(const double* __restrict__ tiles, int ts, int nt, int n, double* __restrict__ partial) {
  const int k = blockIdx.x;
  const int rows = min(ts, n - k * ts);
  const double s = logdet_tile_body(tiles + tile_slot(k, k, nt) * (long long)ts * ts, ts, rows);
  if (threadIdx.x == 0) partial[k] = s;
}

void launch_logdet_partials(const double* tiles, int ts, int nt, int n, double* partial, cudaStream_t st) {
  logdet_partials_kernel<<<nt, 256, 0, st>>>(tiles, ts, nt, n, partial);
}

// result = (log-likelihood, log|C|, Z^T C^-1 Z after the solve, info) (finalize_body).
__global__ void __launch_bounds__(256)
finalize_kernel(const double* __restrict__ partial, int nt, const double* __restrict__ z, int n,
                double* __restrict__ result, const int* __restrict__ info) {
  finalize_body(partial, nt, z, n, result, info);
}

void launch_finalize(const double* partial, int nt, const double* z, int n, double* result, const int* info,
                     cudaStream_t st) {
  finalize_kernel<<<1, 256, 0, st>>>(partial, nt, z, n, result, info);
}

// out[0] = sum (a - b)^2 (DMSECodelet, dmse-codelet.cpp:60-73), fixed order.
__global__ void __launch_bounds__(256)
sumsq_diff_kernel(const double* __restrict__ a, const double* __restrict__ b, int n, double* __restrict__ out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double d = a[r] - b[r];
    acc = fma(d, d, acc);
  }
  const double s = block_sum_256(acc, red);
  if (threadIdx.x == 0) out[0] = s;
}

void launch_sumsq_diff(const double* a, const double* b, int n, double* out, cudaStream_t st) {
  sumsq_diff_kernel<<<1, 256, 0, st>>>(a, b, n, out);
}

}  // namespace egs

namespace egs {

// out[j] = sum_i A[i + j*lda] * w[i] for j < cols (A is rows x cols column-major):
// the kriging product Zmiss = C12 * Zobs with C12 stored transposed (obs x miss,
// LinearAlgebraMethods.cpp:552).  One warp per output, fixed reduction order.
__global__ void __launch_bounds__(256)
gemv_t_block_kernel(const double* __restrict__ a, long long lda, int rows, int cols, const double* __restrict__ w,
                    double* __restrict__ out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * 8 + warp;
  if (j >= cols) return;
  const double* col = a + (long long)j * lda;
  double acc = 0.0;
  for (int i = lane; i < rows; i += 32) acc = fma(col[i], w[i], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[j] = acc;
}

void launch_gemv_t_block(const double* a, long long lda, int rows, int cols, const double* w, double* out,
                         cudaStream_t st) {
  if (cols <= 0) return;
  gemv_t_block_kernel<<<(cols + 7) / 8, 256, 0, st>>>(a, lda, rows, cols, w, out);
}

}  // namespace egs

namespace egs {

// part[slot(i, j)][r] = sum_c L_ij[r][c] e_j[c] over the stored lower tiles (only
// c <= r inside a diagonal tile): the tile products of Z = L e
// (dtrmm in GenerateObservationsVector, LinearAlgebraMethods.cpp:400).
__global__ void __launch_bounds__(256)
trmv_tile_kernel(const double* __restrict__ tiles, int ts, int nt, const double* __restrict__ e,
                 double* __restrict__ part) {
  __shared__ double red[4][kNB];
  const long long slot = blockIdx.y;
  // slot -> (i, j)
  int j = 0;
  while (j < nt - 1 && tile_slot(j + 1, j + 1, nt) <= slot) ++j;
  const int i = j + (int)(slot - tile_slot(j, j, nt));
  const double* T = tiles + slot * (long long)ts * ts;
  const double* ej = e + (long long)j * ts;
  const int rl = threadIdx.x % kNB, g = threadIdx.x / kNB;
  const int r = blockIdx.x * kNB + rl;
  double acc = 0.0;
  if (r < ts) {
    const int cend = (i == j) ? r + 1 : ts;
    for (int c = g; c < cend; c += 4) acc = fma(T[(long long)c * ts + r], ej[c], acc);
  }
  red[g][rl] = acc;
  __syncthreads();
  if (g == 0 && r < ts) part[slot * ts + r] = ((red[0][rl] + red[1][rl]) + red[2][rl]) + red[3][rl];
}

// z[i*ts + r] = sum_{j <= i} part[slot(i, j)][r], j ascending (fixed order).
__global__ void __launch_bounds__(256)
trmv_reduce_kernel(const double* __restrict__ part, int ts, int nt, double* __restrict__ z) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)nt * ts) return;
  const int i = (int)(g / ts), r = (int)(g - (long long)i * ts);
  double acc = 0.0;
  for (int j = 0; j <= i; ++j) acc += part[tile_slot(i, j, nt) * ts + r];
  z[g] = acc;
}

void launch_trmv(const double* tiles, int ts, int nt, const double* e, double* part, double* z, cudaStream_t st) {
  const long long nslots = lower_tiles(nt);  // <= 65535 is checked by the caller
  trmv_tile_kernel<<<dim3((ts + kNB - 1) / kNB, (unsigned)nslots), 256, 0, st>>>(tiles, ts, nt, e, part);
  const long long total = (long long)nt * ts;
  trmv_reduce_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(part, ts, nt, z);
}

}  // namespace egs

namespace egs {

// out = L^T w for the lower tiled factor (global row r = j ts + c):
// out[r] = sum_{i > j} (column c of tile (i, j)) . w_i + sum_{rr >= c} L_jj(rr, c) w_j(rr);
// one warp per output element, fixed summation order.
__global__ void __launch_bounds__(256)
trmv_t_kernel(const double* __restrict__ tiles, int ts, int nt, const double* __restrict__ w,
              double* __restrict__ out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.y, c = blockIdx.x * 8 + warp;
  if (c >= ts) return;
  double acc = 0.0;
  for (int i = j; i < nt; ++i) {
    const double* col = tiles + tile_slot(i, j, nt) * (long long)ts * ts + (long long)c * ts;
    const double* wi = w + (long long)i * ts;
    for (int rr = (i == j ? c : 0) + lane; rr < ts; rr += 32) acc = fma(col[rr], wi[rr], acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[(long long)j * ts + c] = acc;
}

void launch_trmv_t(const double* tiles, int ts, int nt, const double* w, double* out, cudaStream_t st) {
  trmv_t_kernel<<<dim3((ts + 7) / 8, nt), 256, 0, st>>>(tiles, ts, nt, w, out);
}

// out[slot] = a . b over n entries (one block, fixed order).
__global__ void __launch_bounds__(256)
dot_kernel(const double* __restrict__ a, const double* __restrict__ b, int n, double* __restrict__ out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) acc = fma(a[i], b[i], acc);
  const double s = block_sum_256(acc, red);
  if (threadIdx.x == 0) *out = s;
}

void launch_dot(const double* a, const double* b, int n, double* out, cudaStream_t st) {
  dot_kernel<<<1, 256, 0, st>>>(a, b, n, out);
}

}  // namespace egs
