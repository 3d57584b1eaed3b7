// Kernels of the mixed-precision log-likelihood evaluation (FP64 band, FP32
// off-band tiles), sm_100a.
//
// Storage of one problem (nt tile rows of ts, band b >= 0 tile rows kept FP64):
//   band pool  FP64 tiles (i, j), 0 <= i - j <= b, at slot j*(b+1) + (i-j);
//   off pool   FP32 tiles (i, j), i - j > b, at tile_slot(i-b-1, j, nt-b-1);
//   W          FP64 workspace of one tile column: W[t] = tile (k+t, k), plus
//              W[nt-k] = identity, which the panel solve turns into L_kk^-T;
//   inv pool   FP64 L_kk^-T of every diagonal tile (upper triangular).
// The step-k host sequence (capi.cu) gathers column k into W (FP32 tiles
// widened), factors and solves it there with the FP64 kernels, scatters it back
// (off-band tiles rounded to FP32), splits it for the FP16 tensor-core update
// (split_gemm.cu) and runs the FP64 band update with the DMMA kernel.
//
// Solves: the diagonal blocks are applied through their explicit inverses
// (a many-block matrix-vector product instead of a sequential substitution),
// the off-diagonal tiles are read in FP64 (band) or FP32 (off-band) with FP64
// arithmetic; one step of iterative
// refinement uses the residual r = z - C v with C regenerated on the fly in
// FP64 (matern_residual_kernel), so the quadratic form z^T C^-1 z keeps FP64
// accuracy up to the factor's conditioning.
#include <cuda_fp16.h>
#include "common.cuh"
#include "kernels.cuh"
#include "matern_tile.cuh"
#include "panel_bodies.cuh"

namespace egs {

__host__ __device__ __forceinline__ long long band_slot(int i, int j, int b) { return (long long)j * (b + 1) + (i - j); }
__host__ __device__ __forceinline__ long long off_slot(int i, int j, int nt, int b) {
  return tile_slot(i - b - 1, j, nt - b - 1);
}

// ---------------------------------------------------------------------------
// Generation: tinfo[t] = (i, j, 0 band / 1 off, slot)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kGenThreads)
matern_mixed_kernel(double* __restrict__ band, float* __restrict__ off, const double* __restrict__ x,
                    const double* __restrict__ y, int n, int ts, const int4* __restrict__ tinfo, long long t0,
                    const MaternParams* __restrict__ pp, const double* __restrict__ ktab) {
  __shared__ double stab[kKtabDoubles];
  const MaternParams p = *pp;
  stage_ktab(stab, ktab, p);
  const int4 ti = tinfo[t0 + blockIdx.y];
  const long long pair0 = (long long)blockIdx.x * kGenPairsPerBlock;
  const long long base = (long long)ti.w * ts * ts;
  if (ti.z == 0) {
    matern_tile_pairs(band + base, x, y, n, ts, ti.x, ti.y, pair0, p, stab);
  } else {
    matern_tile_pairs(off + base, x, y, n, ts, ti.x, ti.y, pair0, p, stab);
  }
}

void launch_matern_mixed(double* band, float* off, const double* x, const double* y, int n, int ts,
                         const int4* tinfo, long long ntiles, const MaternParams* params, double* ktab,
                         cudaStream_t st) {
  launch_matern_ktab(params, ktab, 1, st);
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + kGenPairsPerBlock - 1) / kGenPairsPerBlock);
  for (long long t0 = 0; t0 < ntiles; t0 += 65535) {
    const unsigned gy = (unsigned)((ntiles - t0) < 65535 ? (ntiles - t0) : 65535);
    matern_mixed_kernel<<<dim3(gx, gy), kGenThreads, 0, st>>>(band, off, x, y, n, ts, tinfo, t0, params, ktab);
  }
}

// ---------------------------------------------------------------------------
// Column k <-> W
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
gather_column_kernel(const double* __restrict__ band, const float* __restrict__ off, double* __restrict__ W, int ts,
                     int nt, int b, int k) {
  const int t = blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  double2 v;
  if (t == nt - k) {
    // identity tile below the column: the panel solve makes it L_kk^-T
    const long long c = e / ts, r = e - c * ts;
    v = make_double2(r == c ? 1.0 : 0.0, r + 1 == c ? 1.0 : 0.0);
  } else if (t <= b) {
    v = *reinterpret_cast<const double2*>(band + band_slot(k + t, k, b) * ts * ts + e);
  } else {
    const float2 f = *reinterpret_cast<const float2*>(off + off_slot(k + t, k, nt, b) * ts * ts + e);
    v = make_double2(f.x, f.y);
  }
  *reinterpret_cast<double2*>(W + (long long)t * ts * ts + e) = v;
}

__global__ void __launch_bounds__(256)
scatter_column_kernel(const double* __restrict__ W, double* __restrict__ band, float* __restrict__ off,
                      double* __restrict__ inv, int ts, int nt, int b, int k) {
  const int t = blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  const double2 v = *reinterpret_cast<const double2*>(W + (long long)t * ts * ts + e);
  if (t == nt - k) {
    *reinterpret_cast<double2*>(inv + (long long)k * ts * ts + e) = v;
  } else if (t <= b) {
    *reinterpret_cast<double2*>(band + band_slot(k + t, k, b) * ts * ts + e) = v;
  } else {
    *reinterpret_cast<float2*>(off + off_slot(k + t, k, nt, b) * ts * ts + e) = make_float2((float)v.x, (float)v.y);
  }
}

// W[0 .. nt-k-1] = tile column k (FP32 tiles widened), W[nt-k] = identity.
void launch_gather_column(const double* band, const float* off, double* W, int ts, int nt, int b, int k,
                          cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  gather_column_kernel<<<dim3(gx, nt - k + 1), 256, 0, st>>>(band, off, W, ts, nt, b, k);
}

// Tile column k back to the pools (off-band tiles rounded to FP32) and
// W[nt-k] = L_kk^-T to inv slot k.
void launch_scatter_column(const double* W, double* band, float* off, double* inv, int ts, int nt, int b, int k,
                           cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  scatter_column_kernel<<<dim3(gx, nt - k + 1), 256, 0, st>>>(W, band, off, inv, ts, nt, b, k);
}

// Short panel of the Ozaki form: W2[0 .. nb] = tiles (k .. k+nb, k) from the
// FP64 band pool, W2[nb+1] = identity (nb = min(b, nt-k-1)).
__global__ void __launch_bounds__(256)
gather_panel_kernel(const double* __restrict__ band, double* __restrict__ W2, int ts, int b, int nb, int k) {
  const int t = blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  double2 v;
  if (t == nb + 1) {
    const long long c = e / ts, r = e - c * ts;
    v = make_double2(r == c ? 1.0 : 0.0, r + 1 == c ? 1.0 : 0.0);
  } else {
    v = *reinterpret_cast<const double2*>(band + band_slot(k + t, k, b) * ts * ts + e);
  }
  *reinterpret_cast<double2*>(W2 + (long long)t * ts * ts + e) = v;
}

// W2[0 .. nb] back to the band pool (and W2[1 .. nb] into W[1 .. nb] for the
// split and slicing of the whole panel); W2[nb+1] = L_kk^-T to inverse slot k.
__global__ void __launch_bounds__(256)
scatter_panel_kernel(const double* __restrict__ W2, double* __restrict__ band, double* __restrict__ inv,
                     double* __restrict__ W, int ts, int b, int nb, int k) {
  const int t = blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  const double2 v = *reinterpret_cast<const double2*>(W2 + (long long)t * ts * ts + e);
  if (t == nb + 1) {
    *reinterpret_cast<double2*>(inv + (long long)k * ts * ts + e) = v;
  } else {
    *reinterpret_cast<double2*>(band + band_slot(k + t, k, b) * ts * ts + e) = v;
    if (t > 0) *reinterpret_cast<double2*>(W + (long long)t * ts * ts + e) = v;
  }
}

// Off-band tiles W[nb+1 .. nt-k-1] = (k+nb+1 .. nt-1, k) rounded into the FP32 pool.
__global__ void __launch_bounds__(256)
scatter_offband_kernel(const double* __restrict__ W, float* __restrict__ off, int ts, int nt, int b, int nb, int k) {
  const int t = nb + 1 + blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  const double2 v = *reinterpret_cast<const double2*>(W + (long long)t * ts * ts + e);
  *reinterpret_cast<float2*>(off + off_slot(k + t, k, nt, b) * ts * ts + e) = make_float2((float)v.x, (float)v.y);
}

void launch_gather_panel(const double* band, double* W2, int ts, int b, int nb, int k, cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  gather_panel_kernel<<<dim3(gx, nb + 2), 256, 0, st>>>(band, W2, ts, b, nb, k);
}

void launch_scatter_panel(const double* W2, double* band, double* inv, double* W, int ts, int b, int nb, int k,
                          cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  scatter_panel_kernel<<<dim3(gx, nb + 2), 256, 0, st>>>(W2, band, inv, W, ts, b, nb, k);
}

void launch_scatter_offband(const double* W, float* off, int ts, int nt, int b, int nb, int k, cudaStream_t st) {
  const int count = nt - k - 1 - nb;
  if (count <= 0) return;
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  scatter_offband_kernel<<<dim3(gx, count), 256, 0, st>>>(W, off, ts, nt, b, nb, k);
}

const float* offband_tile(const float* off, int ts, int nt, int b, int i, int k) {
  return off + off_slot(i, k, nt, b) * (long long)ts * ts;
}

// ---------------------------------------------------------------------------
// Reductions and solves
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
logdet_band_kernel(const double* __restrict__ band, int ts, int b, int n, double* __restrict__ partial) {
  const int k = blockIdx.x;
  const int rows = min(ts, n - k * ts);
  const double s = logdet_tile_body(band + band_slot(k, k, b) * (long long)ts * ts, ts, rows);
  if (threadIdx.x == 0) partial[k] = s;
}

void launch_logdet_band(const double* band, int ts, int nt, int b, int n, double* partial, cudaStream_t st) {
  logdet_band_kernel<<<nt, 256, 0, st>>>(band, ts, b, n, partial);
}

// z_i -= L_ik z_k for every tile row i > k, with z_k read from zk; blocks of
// the first target row also store zk into z (the solved segment k).
__global__ void __launch_bounds__(256)
gemv_mixed_kernel(const double* __restrict__ band, const float* __restrict__ off, int ts, int nt, int b, int k,
                  const double* __restrict__ zk, double* __restrict__ z) {
  const int i = k + 1 + blockIdx.y;
  double* zi = z + (long long)i * ts;
  if (blockIdx.y == 0) {
    const int r = blockIdx.x * kNB + threadIdx.x;
    if (threadIdx.x < kNB && r < ts) z[(long long)k * ts + r] = zk[r];
  }
  if (i - k <= b) {
    gemv_panel_body(band + band_slot(i, k, b) * (long long)ts * ts, ts, zk, zi, blockIdx.x);
  } else {
    gemv_panel_body(off + off_slot(i, k, nt, b) * (long long)ts * ts, ts, zk, zi, blockIdx.x);
  }
}

// z_i -= L_ki^T z_k for every tile column i < k; one warp per column of tile (k, i).
template <typename Tile>
__device__ __forceinline__ double col_dot(const Tile* __restrict__ col, const double* __restrict__ zk, int ts,
                                          int lane) {
  double acc = 0.0;
  for (int r = lane; r < ts; r += 32) acc = fma((double)col[r], zk[r], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

__global__ void __launch_bounds__(256)
gemv_t_mixed_kernel(const double* __restrict__ band, const float* __restrict__ off, int ts, int nt, int b, int k,
                    const double* __restrict__ zk, double* __restrict__ z) {
  const int i = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + warp;
  if (c >= ts) return;
  if (i == 0 && lane == 0) z[(long long)k * ts + c] = zk[c];
  double acc;
  if (k - i <= b) {
    acc = col_dot(band + band_slot(k, i, b) * (long long)ts * ts + (long long)c * ts, zk, ts, lane);
  } else {
    acc = col_dot(off + off_slot(k, i, nt, b) * (long long)ts * ts + (long long)c * ts, zk, ts, lane);
  }
  if (lane == 0) z[(long long)i * ts + c] -= acc;
}

// out = L_kk^-1 in = X^T in with X = L_kk^-T (upper triangular, column-major):
// out[i] = sum_{j <= i} X[j, i] in[j]; one warp per output (a contiguous column).
__global__ void __launch_bounds__(256)
inv_apply_t_kernel(const double* __restrict__ X, int ts, const double* __restrict__ in, double* __restrict__ out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 8 + warp;
  if (i >= ts) return;
  const double* col = X + (long long)i * ts;
  double acc = 0.0;
  for (int j = lane; j <= i; j += 32) acc = fma(col[j], in[j], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) out[i] = acc;
}

// out = L_kk^-T in = X in: out[i] = sum_{j >= i} X[i, j] in[j]; 64 rows x 4
// column groups per block, fixed reduction order.  Dynamic shared memory: ts doubles.
__global__ void __launch_bounds__(256)
inv_apply_kernel(const double* __restrict__ X, int ts, const double* __restrict__ in, double* __restrict__ out) {
  extern __shared__ double ins[];
  __shared__ double red[4][kNB];
  for (int c = threadIdx.x; c < ts; c += blockDim.x) ins[c] = in[c];
  __syncthreads();
  const int rl = threadIdx.x & (kNB - 1), g = threadIdx.x / kNB;
  const int i = blockIdx.x * kNB + rl;
  // four interleaved sums per thread keep sixteen loads in flight; the column
  // order within each sum and the final combination are fixed
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  if (i < ts) {
    const double* xr = X + i;
    int j = blockIdx.x * kNB + g;
    for (; j + 12 < ts; j += 16) {
      const double x0 = (j >= i) ? xr[(long long)j * ts] : 0.0;
      const double x1 = (j + 4 >= i) ? xr[(long long)(j + 4) * ts] : 0.0;
      const double x2 = (j + 8 >= i) ? xr[(long long)(j + 8) * ts] : 0.0;
      const double x3 = (j + 12 >= i) ? xr[(long long)(j + 12) * ts] : 0.0;
      a0 = fma(x0, ins[j], a0);
      a1 = fma(x1, ins[j + 4], a1);
      a2 = fma(x2, ins[j + 8], a2);
      a3 = fma(x3, ins[j + 12], a3);
    }
    for (; j < ts; j += 4)
      if (j >= i) a0 = fma(xr[(long long)j * ts], ins[j], a0);
  }
  red[g][rl] = (a0 + a1) + (a2 + a3);
  __syncthreads();
  if (g == 0 && i < ts) out[i] = ((red[0][rl] + red[1][rl]) + red[2][rl]) + red[3][rl];
}

__global__ void add_inplace_kernel(double* __restrict__ a, const double* __restrict__ b, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] += b[i];
}

void launch_add_inplace(double* a, const double* b, int n, cudaStream_t st) {
  add_inplace_kernel<<<(n + 255) / 256, 256, 0, st>>>(a, b, n);
}

__global__ void copy_segment_kernel(const double* __restrict__ src, double* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

// v := (L L^T)^-1 v with the mixed factor; tmp holds ts doubles.
void launch_mixed_solve(const double* band, const float* off, const double* inv, int ts, int nt, int b, double* v,
                        double* tmp, cudaStream_t st, long long* launches) {
  const long long ts2 = (long long)ts * ts;
  for (int k = 0; k < nt; ++k) {
    inv_apply_t_kernel<<<(ts + 7) / 8, 256, 0, st>>>(inv + k * ts2, ts, v + (long long)k * ts, tmp);
    if (k < nt - 1) {
      gemv_mixed_kernel<<<dim3((ts + kNB - 1) / kNB, nt - 1 - k), 256, ts * sizeof(double), st>>>(band, off, ts, nt,
                                                                                                 b, k, tmp, v);
    } else {
      copy_segment_kernel<<<(ts + 255) / 256, 256, 0, st>>>(tmp, v + (long long)k * ts, ts);
    }
    *launches += 2;
  }
  for (int k = nt - 1; k >= 0; --k) {
    inv_apply_kernel<<<(ts + kNB - 1) / kNB, 256, ts * sizeof(double), st>>>(inv + k * ts2, ts, v + (long long)k * ts,
                                                                               tmp);
    if (k > 0) {
      gemv_t_mixed_kernel<<<dim3((ts + 7) / 8, k), 256, 0, st>>>(band, off, ts, nt, b, k, tmp, v);
    } else {
      copy_segment_kernel<<<(ts + 255) / 256, 256, 0, st>>>(tmp, v, ts);
    }
    *launches += 2;
  }
}

// ---------------------------------------------------------------------------
// Refinement residual r = z - C(theta) v, C regenerated in FP64.
// C is symmetric, so every pair i > j is evaluated once and used twice: for row
// i (C(i, j) v_j) and for column j (C(i, j) v_i).  The lower triangle of
// 256-row blocks is covered by square super-blocks of 1 .. kResSuper blocks a
// side (res_side), one CTA each.  A thread owns row i of the current row block: its row sum
// stays in a register across the super-block's column blocks, and the column
// sums are formed by warp butterflies and a fixed-order sum over the warps,
// kept per column block in shared memory by the thread that owns the column.  Super-block
// partials go to rowpart[sbj][i] and colpart[sbi][j]; the reduce kernel adds
// them in a fixed order.  Only the n real rows / columns take part.
// ---------------------------------------------------------------------------
constexpr int kResBlk = 256;    // rows (and columns) per block = threads per CTA
constexpr int kResSuper = 8;    // most blocks per super-block side

__host__ __device__ __forceinline__ int res_blocks(int n) { return (n + kResBlk - 1) / kResBlk; }
// Blocks per super-block side: as many as keep at least ~24 super-blocks per
// side (hundreds of CTAs), at most kResSuper.
__host__ __device__ __forceinline__ int res_side(int n) {
  const int s = res_blocks(n) / 24;
  return s < 1 ? 1 : (s > kResSuper ? kResSuper : s);
}
__host__ __device__ __forceinline__ int res_supers(int n) { return (res_blocks(n) + res_side(n) - 1) / res_side(n); }

__global__ void __launch_bounds__(kResBlk, 3)
matern_residual_partial_kernel(const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ v, int n, const MaternParams* __restrict__ pp,
                               const double* __restrict__ ktab, double* __restrict__ rowpart,
                               double* __restrict__ colpart) {
  __shared__ double stab[kKtabDoubles];
  __shared__ double xs[kResBlk], ys[kResBlk], vs[kResBlk];
  __shared__ double red[kResBlk / 32][kResBlk];
  __shared__ double colacc[kResSuper][kResBlk];  // column sums of each column block (thread = column)
  const MaternParams p = *pp;
  stage_ktab(stab, ktab, p);
  // super-block (sbi, sbj), sbj <= sbi, from the linear index
  const int L = blockIdx.x;
  int sbi = (int)((sqrt(8.0 * (double)L + 1.0) - 1.0) * 0.5);
  while ((sbi + 1) * (sbi + 2) / 2 <= L) ++sbi;
  while (sbi * (sbi + 1) / 2 > L) --sbi;
  const int sbj = L - sbi * (sbi + 1) / 2;
  const int nb = res_blocks(n), side = res_side(n);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int bj0 = sbj * side, bj1 = min(nb, bj0 + side);
  const int bi0 = sbi * side, bi1 = min(nb, bi0 + side);
#pragma unroll
  for (int q = 0; q < kResSuper; ++q) colacc[q][t] = 0.0;
  for (int bi = bi0; bi < bi1; ++bi) {
    const int i = bi * kResBlk + t;
    const bool row = i < n;
    const double xi = row ? x[i] : 0.0, yi = row ? y[i] : 0.0, vi = row ? v[i] : 0.0;
    double racc = 0.0;
#pragma unroll 1
    for (int q = 0; q < side; ++q) {
      const int bj = bj0 + q;
      if (bj >= bj1 || bj > bi) break;  // uniform over the CTA
      const int jb = bj * kResBlk;
      __syncthreads();  // previous column block done with xs / ys / vs / red
      if (jb + t < n) {
        xs[t] = x[jb + t];
        ys[t] = y[jb + t];
        vs[t] = v[jb + t];
      } else {
        xs[t] = ys[t] = vs[t] = 0.0;
      }
      __syncthreads();
      const bool diag = (bj == bi);
      const int m = min(kResBlk, n - jb);
      for (int jj = 0; jj < m; ++jj) {
        double c = 0.0;
        if (row && (!diag || jj <= t)) c = matern_from_dist_tab(euclid_dist(xi, yi, xs[jj], ys[jj]), p, stab);
        racc = fma(c, vs[jj], racc);
        // column jj gets C(i, jj) v_i from every row i below it (i > j)
        double cc = (!diag || jj < t) ? c * vi : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cc += __shfl_xor_sync(0xffffffffu, cc, o);
        if (lane == 0) red[warp][jj] = cc;
      }
      __syncthreads();
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < kResBlk / 32; ++w) sum += red[w][t];
      colacc[q][t] += sum;
    }
    if (row) rowpart[(long long)sbj * n + i] = racc;
  }
  for (int q = 0; q < side; ++q) {
    const int j = (bj0 + q) * kResBlk + t;
    if (bj0 + q < bj1 && j < n) colpart[(long long)sbi * n + j] = colacc[q][t];
  }
}

// r_i = z_i - (row partials of super-block columns 0 .. sb(i) + column partials
// of super-block rows sb(i) .. ns-1), each in a fixed order; padding rows get 0.
__global__ void __launch_bounds__(256)
residual_reduce_kernel(const double* __restrict__ z, const double* __restrict__ rowpart,
                       const double* __restrict__ colpart, int n, int np, double* __restrict__ r) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= np) return;
  if (i >= n) {
    r[i] = 0.0;
    return;
  }
  const int sb = (i / kResBlk) / res_side(n), ns = res_supers(n);
  double a = 0.0, b = 0.0;
  for (int q = 0; q <= sb; ++q) a += rowpart[(long long)q * n + i];
  for (int q = sb; q < ns; ++q) b += colpart[(long long)q * n + i];
  r[i] = z[i] - (a + b);
}

long long residual_scratch_doubles(int n) { return 2LL * res_supers(n) * n; }

void launch_matern_residual(const double* x, const double* y, const double* z, const double* v, int n, int np,
                            const MaternParams* params, const double* ktab, double* scratch, double* r,
                            cudaStream_t st) {
  const int ns = res_supers(n);
  double* rowpart = scratch;
  double* colpart = scratch + (long long)ns * n;
  const unsigned grid = (unsigned)((long long)ns * (ns + 1) / 2);
  matern_residual_partial_kernel<<<grid, kResBlk, 0, st>>>(x, y, v, n, params, ktab, rowpart, colpart);
  residual_reduce_kernel<<<(np + 255) / 256, 256, 0, st>>>(z, rowpart, colpart, n, np, r);
}

// result = (loglik, logdet, z^T (v + w), info) with the refined solution v + w.
__global__ void __launch_bounds__(256)
finalize_mixed_kernel(const double* __restrict__ partial, int nt, const double* __restrict__ z,
                      const double* __restrict__ v, const double* __restrict__ w, int n, double* __restrict__ result,
                      const int* __restrict__ info) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) acc = fma(z[r], v[r] + w[r], acc);
  const double dot = block_sum_256(acc, red);
  if (threadIdx.x == 0) {
    double det = 0.0;
    for (int k = 0; k < nt; ++k) det += partial[k];
    const double logdet = 2.0 * det;
    const double pi = 3.141592653589793;
    result[0] = -0.5 * dot - 0.5 * logdet - ((double)n / 2.0) * log(2.0 * pi);
    result[1] = logdet;
    result[2] = dot;
    result[3] = (double)(info ? *info : 0);
  }
}

void launch_finalize_mixed(const double* partial, int nt, const double* z, const double* v, const double* w, int n,
                           double* result, const int* info, cudaStream_t st) {
  finalize_mixed_kernel<<<1, 256, 0, st>>>(partial, nt, z, v, w, n, result, info);
}

}  // namespace egs
