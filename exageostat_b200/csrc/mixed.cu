// Kernels of the mixed-precision log-likelihood evaluation (FP64 band, FP32
// off-band tiles), sm_100a.
//
// Storage of one problem (nt tile rows of ts, band b >= 0 tile rows kept FP64):
//   band pool  FP64 tiles (i, j), 0 <= i - j <= b, at slot j*(b+1) + (i-j);
//   off pool   FP32 tiles (i, j), i - j > b, at tile_slot(i-b-1, j, nt-b-1);
//   W          FP64 workspace of one tile column: W[t] = tile (k+t, k).
// The step-k host sequence (capi.cu) gathers column k into W (FP32 tiles
// widened), factors and solves it there with the FP64 kernels, scatters it back
// (off-band tiles rounded to FP32), splits it for the FP16 tensor-core update
// (split_gemm.cu) and runs the FP64 band update with the DMMA kernel.
//
// Solves: forward and backward substitution read the band tiles in FP64 and
// the off-band tiles in FP32 with FP64 arithmetic; one step of iterative
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
  if (t <= b) {
    v = *reinterpret_cast<const double2*>(band + band_slot(k + t, k, b) * ts * ts + e);
  } else {
    const float2 f = *reinterpret_cast<const float2*>(off + off_slot(k + t, k, nt, b) * ts * ts + e);
    v = make_double2(f.x, f.y);
  }
  *reinterpret_cast<double2*>(W + (long long)t * ts * ts + e) = v;
}

__global__ void __launch_bounds__(256)
scatter_column_kernel(const double* __restrict__ W, double* __restrict__ band, float* __restrict__ off, int ts,
                      int nt, int b, int k) {
  const int t = blockIdx.y;
  const long long e = ((long long)blockIdx.x * 256 + threadIdx.x) * 2;
  if (e >= (long long)ts * ts) return;
  const double2 v = *reinterpret_cast<const double2*>(W + (long long)t * ts * ts + e);
  if (t <= b) {
    *reinterpret_cast<double2*>(band + band_slot(k + t, k, b) * ts * ts + e) = v;
  } else {
    *reinterpret_cast<float2*>(off + off_slot(k + t, k, nt, b) * ts * ts + e) = make_float2((float)v.x, (float)v.y);
  }
}

void launch_gather_column(const double* band, const float* off, double* W, int ts, int nt, int b, int k,
                          cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  gather_column_kernel<<<dim3(gx, nt - k), 256, 0, st>>>(band, off, W, ts, nt, b, k);
}

void launch_scatter_column(const double* W, double* band, float* off, int ts, int nt, int b, int k,
                           cudaStream_t st) {
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + 255) / 256);
  scatter_column_kernel<<<dim3(gx, nt - k), 256, 0, st>>>(W, band, off, ts, nt, b, k);
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

// z_i -= L_ik z_k for every tile row i > k.
__global__ void __launch_bounds__(256)
gemv_mixed_kernel(const double* __restrict__ band, const float* __restrict__ off, int ts, int nt, int b, int k,
                  double* __restrict__ z) {
  const int i = k + 1 + blockIdx.y;
  const double* zk = z + (long long)k * ts;
  double* zi = z + (long long)i * ts;
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
                    double* __restrict__ z) {
  const int i = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * 8 + warp;
  if (c >= ts) return;
  const double* zk = z + (long long)k * ts;
  double acc;
  if (k - i <= b) {
    acc = col_dot(band + band_slot(k, i, b) * (long long)ts * ts + (long long)c * ts, zk, ts, lane);
  } else {
    acc = col_dot(off + off_slot(k, i, nt, b) * (long long)ts * ts + (long long)c * ts, zk, ts, lane);
  }
  if (lane == 0) z[(long long)i * ts + c] -= acc;
}

// v := (L L^T)^-1 v with the mixed factor.
void launch_mixed_solve(const double* band, const float* off, int ts, int nt, int b, double* v, cudaStream_t st,
                        long long* launches) {
  for (int k = 0; k < nt; ++k) {
    launch_trsv_diag(band, ts, band_slot(k, k, b), v + (long long)k * ts, st);
    ++*launches;
    if (k < nt - 1) {
      gemv_mixed_kernel<<<dim3((ts + kNB - 1) / kNB, nt - 1 - k), 256, ts * sizeof(double), st>>>(band, off, ts, nt,
                                                                                                 b, k, v);
      ++*launches;
    }
  }
  for (int k = nt - 1; k >= 0; --k) {
    launch_trsv_t_diag(band, ts, band_slot(k, k, b), v + (long long)k * ts, st);
    ++*launches;
    if (k > 0) {
      gemv_t_mixed_kernel<<<dim3((ts + 7) / 8, k), 256, 0, st>>>(band, off, ts, nt, b, k, v);
      ++*launches;
    }
  }
}

// ---------------------------------------------------------------------------
// Refinement residual r = z - C(theta) v, C regenerated in FP64.
// Block (row block of 256 rows, column split s): partial[s][i] = sum over the
// columns of split s of C(i, j) v_j, in a fixed order; the reduce kernel adds
// the splits in order.  Only the n real rows / columns take part.
// ---------------------------------------------------------------------------
constexpr int kResSplits = 8;
constexpr int kResChunk = 256;

__global__ void __launch_bounds__(256)
matern_residual_partial_kernel(const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ v, int n, const MaternParams* __restrict__ pp,
                               const double* __restrict__ ktab, double* __restrict__ partial) {
  __shared__ double stab[kKtabDoubles];
  __shared__ double xs[kResChunk], ys[kResChunk], vs[kResChunk];
  const MaternParams p = *pp;
  stage_ktab(stab, ktab, p);
  const int i = blockIdx.x * 256 + threadIdx.x;
  const int per = (n + kResSplits - 1) / kResSplits;
  const int j0 = blockIdx.y * per, j1 = min(n, j0 + per);
  const bool row = i < n;
  const double xi = row ? x[i] : 0.0, yi = row ? y[i] : 0.0;
  double acc = 0.0;
  for (int jc = j0; jc < j1; jc += kResChunk) {
    const int m = min(kResChunk, j1 - jc);
    __syncthreads();
    if (threadIdx.x < m) {
      xs[threadIdx.x] = x[jc + threadIdx.x];
      ys[threadIdx.x] = y[jc + threadIdx.x];
      vs[threadIdx.x] = v[jc + threadIdx.x];
    }
    __syncthreads();
    if (row) {
      for (int q = 0; q < m; ++q) acc = fma(matern_from_dist_tab(euclid_dist(xi, yi, xs[q], ys[q]), p, stab), vs[q], acc);
    }
  }
  if (row) partial[(long long)blockIdx.y * n + i] = acc;
}

__global__ void __launch_bounds__(256)
residual_reduce_kernel(const double* __restrict__ z, const double* __restrict__ partial, int n, int np,
                       double* __restrict__ r) {
  const int i = blockIdx.x * 256 + threadIdx.x;
  if (i >= np) return;
  if (i >= n) {
    r[i] = 0.0;
    return;
  }
  double s = 0.0;
  for (int q = 0; q < kResSplits; ++q) s += partial[(long long)q * n + i];
  r[i] = z[i] - s;
}

long long residual_scratch_doubles(int n) { return (long long)kResSplits * n; }

void launch_matern_residual(const double* x, const double* y, const double* z, const double* v, int n, int np,
                            const MaternParams* params, const double* ktab, double* scratch, double* r,
                            cudaStream_t st) {
  matern_residual_partial_kernel<<<dim3((n + 255) / 256, kResSplits), 256, 0, st>>>(x, y, v, n, params, ktab,
                                                                                     scratch);
  residual_reduce_kernel<<<(np + 255) / 256, 256, 0, st>>>(z, scratch, n, np, r);
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
