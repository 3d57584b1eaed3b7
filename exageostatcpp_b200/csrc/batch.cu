// Batched log-likelihood evaluation of many independent problems ("regional"
// likelihoods of uneven N) on one GPU.
//
// Each problem is the reference's ExaGeoStatMLETile evaluation
// (src/linear-algebra-solvers/concrete/chameleon/ChameleonImplementation.cpp:35-327)
// with its own locations, observations and theta.  Instead of one sequence of
// launches per problem, every stage runs once for all problems:
//
//  * one pool holds every problem's lower tiles (common tile size ts), one 3-D
//    TMA tensor map covers the pool, and per-problem tables give each problem's
//    first tile slot, location offset and tile count;
//  * problems are ordered by tile count (descending), so the problems still
//    active at factorisation step k are a prefix of that order;
//  * step k launches the 64x64 diagonal potrf, the row solves and the
//    tensor-core updates for all active problems at once; the DMMA update runs
//    a precomputed job table (one job per problem) through the batched mode of
//    dgemm_update_kernel;
//  * the whole evaluation of all problems is captured once as a CUDA graph and
//    replayed for every new set of theta (one graph launch per optimiser step).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <numeric>
#include <string>
#include <vector>
#include "common.cuh"
#include "kernels.cuh"
#include "matern_tile.cuh"
#include "panel_bodies.cuh"

namespace egs {

// ---------------------------------------------------------------------------
// Batched kernels
// ---------------------------------------------------------------------------

// Matern tiles of every problem: tinfo[t] = (problem, i, j) of pool slot t;
// block (x, y) generates pairs [x * kGenPairsPerBlock, ...) of slot t0 + y.
__global__ void __launch_bounds__(kGenThreads)
matern_batch_kernel(double* __restrict__ tiles, const double* __restrict__ x, const double* __restrict__ y,
                    const int4* __restrict__ tinfo, long long t0, int ts, const MaternParams* __restrict__ params,
                    const double* __restrict__ ktab, const long long* __restrict__ loc_base,
                    const int* __restrict__ nvec) {
  __shared__ double stab[kKtabDoubles];
  const long long t = t0 + blockIdx.y;
  const int4 ti = tinfo[t];
  const int p = ti.x;
  const MaternParams prm = params[p];
  stage_ktab(stab, ktab + (long long)p * kKtabDoubles, prm);
  matern_tile_pairs(tiles + t * (long long)ts * ts, x + loc_base[p], y + loc_base[p], nvec[p], ts, ti.y, ti.z,
                    (long long)blockIdx.x * kGenPairsPerBlock, prm, stab);
}

__global__ void __launch_bounds__(256)
potrf_batch_kernel(double* __restrict__ tiles, int ts, int k, int kb, const long long* __restrict__ tile_base,
                   const int* __restrict__ ntv, int* __restrict__ info) {
  const int p = blockIdx.x;
  const long long slot = tile_base[p] + tile_slot(k, k, ntv[p]);
  potrf64_body<256>(tiles + slot * (long long)ts * ts + (long long)kb * ts + kb, ts, k * ts + kb, info + p);
}

// panel = 0: rows [row0, ts) of the diagonal tile; panel = 1: all rows of tiles k+1.. of each problem.
__global__ void __launch_bounds__(128)
trsm_batch_kernel(double* __restrict__ tiles, int ts, int k, int row0, int col0, int panel,
                  const long long* __restrict__ tile_base, const int* __restrict__ ntv) {
  const int p = blockIdx.z;
  const int nt = ntv[p];
  const int ntl = panel ? nt - k - 1 : 1;
  if ((int)blockIdx.y >= ntl) return;
  const long long sl = tile_base[p] + tile_slot(k, k, nt);
  const long long sa = panel ? tile_base[p] + tile_slot(k + 1 + blockIdx.y, k, nt) : sl;
  trsm_rows_body<128>(tiles + sa * (long long)ts * ts, tiles + sl * (long long)ts * ts, ts,
                 row0 + blockIdx.x * blockDim.x + threadIdx.x, col0);
}

__global__ void __launch_bounds__(256)
logdet_batch_kernel(const double* __restrict__ tiles, int ts, const long long* __restrict__ tile_base,
                    const int* __restrict__ ntv, const int* __restrict__ nvec, double* __restrict__ partial,
                    const long long* __restrict__ partial_base) {
  const int p = blockIdx.y, k = blockIdx.x;
  if (k >= ntv[p]) return;
  const int rows = min(ts, nvec[p] - k * ts);
  const double s =
      logdet_tile_body(tiles + (tile_base[p] + tile_slot(k, k, ntv[p])) * (long long)ts * ts, ts, rows);
  if (threadIdx.x == 0) partial[partial_base[p] + k] = s;
}

__global__ void __launch_bounds__(1024)
trsv_batch_kernel(const double* __restrict__ tiles, int ts, int k, const long long* __restrict__ tile_base,
                  const int* __restrict__ ntv, double* __restrict__ z, const long long* __restrict__ loc_base) {
  const int p = blockIdx.x;
  trsv_diag_body(tiles + (tile_base[p] + tile_slot(k, k, ntv[p])) * (long long)ts * ts, ts,
                 z + loc_base[p] + (long long)k * ts);
}

__global__ void __launch_bounds__(256)
gemv_batch_kernel(const double* __restrict__ tiles, int ts, int k, const long long* __restrict__ tile_base,
                  const int* __restrict__ ntv, double* __restrict__ z, const long long* __restrict__ loc_base) {
  const int p = blockIdx.z;
  const int i = k + 1 + blockIdx.y;
  if (i >= ntv[p]) return;
  double* zp = z + loc_base[p];
  gemv_panel_body(tiles + (tile_base[p] + tile_slot(i, k, ntv[p])) * (long long)ts * ts, ts,
                  zp + (long long)k * ts, zp + (long long)i * ts, blockIdx.x);
}

__global__ void __launch_bounds__(256)
finalize_batch_kernel(const double* __restrict__ partial, const long long* __restrict__ partial_base,
                      const int* __restrict__ ntv, const double* __restrict__ z,
                      const long long* __restrict__ loc_base, const int* __restrict__ nvec,
                      double* __restrict__ result, const int* __restrict__ info) {
  const int p = blockIdx.x;
  finalize_body(partial + partial_base[p], ntv[p], z + loc_base[p], nvec[p], result + 4 * (long long)p, info + p);
}

}  // namespace egs

using namespace egs;

struct egs_batch {
  int B = 0, ts = 0, nt_max = 0;
  std::vector<int> n, nt, order;  // order[p] = caller index of sorted problem p
  std::vector<int> active;        // active[k] = number of problems with more than k tile rows
  std::vector<long long> tile_base, loc_base, partial_base;
  long long total_tiles = 0, total_loc = 0, total_partial = 0, bytes = 0;
  double *tiles = nullptr, *x = nullptr, *y = nullptr, *z = nullptr, *zcpy = nullptr;
  double *partial = nullptr, *result = nullptr;
  int *info = nullptr, *err = nullptr, *d_n = nullptr, *d_nt = nullptr;
  long long *d_tile_base = nullptr, *d_loc_base = nullptr, *d_partial_base = nullptr;
  int4* d_tinfo = nullptr;
  MaternParams *d_params = nullptr, *h_params = nullptr;
  double* d_ktab = nullptr;  // B Chebyshev tables of K_nu
  double* h_result = nullptr;
  int *h_info = nullptr, *h_err = nullptr;
  GemmDesc* d_jobs = nullptr;
  long long* d_begin = nullptr;
  struct Launch {
    long long job_off, begin_off;
    int njobs;
    long long total;
  };
  std::vector<Launch> diag_launch, panel_launch, trail_launch;  // indexed by (k, kb) or k
  alignas(64) unsigned char tmap[128];
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long evals = 0;
  long long launches_per_eval = 0;
};

namespace {

constexpr int kBatchInner = 64;

int check(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), where);
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

template <typename T>
int balloc(egs_batch* b, T** p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    set_last_error(cudaGetErrorString(e), "egs_batch_create");
    return e == cudaErrorMemoryAllocation ? EGS_ERR_OOM : EGS_ERR_CUDA;
  }
  b->bytes += (long long)(count * sizeof(T));
  return EGS_OK;
}

void free_batch(egs_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  void* dev[] = {b->tiles, b->x, b->y, b->z, b->zcpy, b->partial, b->result, b->info, b->err, b->d_n, b->d_nt,
                 b->d_tile_base, b->d_loc_base, b->d_partial_base, b->d_tinfo, b->d_params, b->d_ktab,
                 b->d_jobs, b->d_begin};
  for (void* p : dev) cudaFree(p);
  cudaFreeHost(b->h_params);
  cudaFreeHost(b->h_result);
  cudaFreeHost(b->h_info);
  cudaFreeHost(b->h_err);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

GemmDesc job_desc(const egs_batch* b, int p, int M, int N, int K, int a_row0, int a_col0, int a_tcol, int b_row0,
                  int b_col0, int b_tcol, int c_row0, int c_col0, int lower) {
  GemmDesc d{};
  d.M = M;
  d.N = N;
  d.K = K;
  d.a_row0 = a_row0;
  d.a_col0 = a_col0;
  d.a_tcol = a_tcol;
  d.b_row0 = b_row0;
  d.b_col0 = b_col0;
  d.b_tcol = b_tcol;
  d.c_row0 = c_row0;
  d.c_col0 = c_col0;
  d.lower = lower;
  d.ts = b->ts;
  d.nt = b->nt[p];
  d.np = b->nt[p] * b->ts;
  d.tile_base = b->tile_base[p];
  finish_desc(d);
  return d;
}

// Job tables of every tensor-core launch of an evaluation, built once.
int build_jobs(egs_batch* b) {
  const int ts = b->ts;
  std::vector<GemmDesc> jobs;
  std::vector<long long> begin;
  auto add_launch = [&](std::vector<egs_batch::Launch>& dst, const std::vector<GemmDesc>& js) {
    egs_batch::Launch L{(long long)jobs.size(), (long long)begin.size(), (int)js.size(), 0};
    long long acc = 0;
    for (const GemmDesc& d : js) {
      jobs.push_back(d);
      begin.push_back(acc);
      acc += d.total;
    }
    begin.push_back(acc);
    L.total = acc;
    dst.push_back(L);
  };
  const int nkb = ts / kBatchInner;
  for (int k = 0; k < b->nt_max; ++k) {
    const int A = b->active[k];
    const int A1 = (k + 1 < b->nt_max) ? b->active[k + 1] : 0;
    for (int kb = 0; kb < ts; kb += kBatchInner) {
      std::vector<GemmDesc> js;
      if (kb + kBatchInner < ts) {
        const int m = ts - kb - kBatchInner;
        const int r0 = k * ts + kb + kBatchInner;
        for (int p = 0; p < A; ++p) js.push_back(job_desc(b, p, m, m, kBatchInner, r0, kb, k, r0, kb, k, r0, r0, 1));
      }
      add_launch(b->diag_launch, js);
      js.clear();
      if (kb + kBatchInner < ts) {
        const int ncols = ts - kb - kBatchInner;
        const int brow = k * ts + kb + kBatchInner;
        for (int p = 0; p < A1; ++p)
          js.push_back(job_desc(b, p, (b->nt[p] - 1 - k) * ts, ncols, kBatchInner, (k + 1) * ts, kb, k, brow, kb, k,
                                (k + 1) * ts, brow, 0));
      }
      add_launch(b->panel_launch, js);
    }
    std::vector<GemmDesc> js;
    for (int p = 0; p < A1; ++p) {
      const int r0 = (k + 1) * ts;
      const int m = b->nt[p] * ts - r0;
      js.push_back(job_desc(b, p, m, m, ts, r0, 0, k, r0, 0, k, r0, r0, 1));
    }
    add_launch(b->trail_launch, js);
    (void)nkb;
  }
  int rc;
  if ((rc = balloc(b, &b->d_jobs, jobs.size())) || (rc = balloc(b, &b->d_begin, begin.size()))) return rc;
  if (!jobs.empty() && cudaMemcpy(b->d_jobs, jobs.data(), jobs.size() * sizeof(GemmDesc), cudaMemcpyHostToDevice))
    return check("build_jobs");
  if (!begin.empty() &&
      cudaMemcpy(b->d_begin, begin.data(), begin.size() * sizeof(long long), cudaMemcpyHostToDevice))
    return check("build_jobs");
  return EGS_OK;
}

int launch_jobs(egs_batch* b, const egs_batch::Launch& L) {
  if (L.njobs == 0 || L.total == 0) return EGS_OK;
  ++b->launches_per_eval;
  return launch_gemm_batched(b->tmap, b->tiles, b->d_jobs + L.job_off, b->d_begin + L.begin_off, L.njobs, L.total,
                             b->err, b->stream);
}

// All device work of one batched evaluation after the parameters are on the device.
int enqueue_batch_eval(egs_batch* b) {
  const int ts = b->ts;
  cudaStream_t st = b->stream;
  b->launches_per_eval = 0;
  if (cudaMemsetAsync(b->info, 0, b->B * sizeof(int), st) || cudaMemsetAsync(b->err, 0, sizeof(int), st) ||
      cudaMemcpyAsync(b->z, b->zcpy, b->total_loc * sizeof(double), cudaMemcpyDeviceToDevice, st))
    return check("enqueue_batch_eval");
  launch_matern_ktab(b->d_params, b->d_ktab, b->B, st);
  ++b->launches_per_eval;
  const unsigned gx = (unsigned)(((long long)ts * ts / 2 + kGenPairsPerBlock - 1) / kGenPairsPerBlock);
  for (long long t0 = 0; t0 < b->total_tiles; t0 += 65535) {
    const unsigned gy = (unsigned)std::min<long long>(65535, b->total_tiles - t0);
    matern_batch_kernel<<<dim3(gx, gy), kGenThreads, 0, st>>>(b->tiles, b->x, b->y, b->d_tinfo, t0, ts,
                                                              b->d_params, b->d_ktab, b->d_loc_base, b->d_n);
    ++b->launches_per_eval;
  }
  int li = 0;
  for (int k = 0; k < b->nt_max; ++k) {
    const int A = b->active[k];
    const int A1 = (k + 1 < b->nt_max) ? b->active[k + 1] : 0;
    for (int kb = 0; kb < ts; kb += kBatchInner, ++li) {
      potrf_batch_kernel<<<A, 256, 0, st>>>(b->tiles, ts, k, kb, b->d_tile_base, b->d_nt, b->info);
      ++b->launches_per_eval;
      if (kb + kBatchInner < ts) {
        const int rows = ts - kb - kBatchInner;
        trsm_batch_kernel<<<dim3((rows + 127) / 128, 1, A), 128, 0, st>>>(b->tiles, ts, k, kb + kBatchInner, kb, 0,
                                                                          b->d_tile_base, b->d_nt);
        ++b->launches_per_eval;
        int rc = launch_jobs(b, b->diag_launch[li]);
        if (rc != EGS_OK) return rc;
      }
    }
    li -= ts / kBatchInner;
    if (A1 > 0) {
      for (int kb = 0; kb < ts; kb += kBatchInner, ++li) {
        trsm_batch_kernel<<<dim3((ts + 127) / 128, b->nt_max - k - 1, A1), 128, 0, st>>>(b->tiles, ts, k, 0, kb, 1,
                                                                                           b->d_tile_base, b->d_nt);
        ++b->launches_per_eval;
        int rc = launch_jobs(b, b->panel_launch[li]);
        if (rc != EGS_OK) return rc;
      }
      int rc = launch_jobs(b, b->trail_launch[k]);
      if (rc != EGS_OK) return rc;
    } else {
      li += ts / kBatchInner;
    }
  }
  logdet_batch_kernel<<<dim3(b->nt_max, b->B), 256, 0, st>>>(b->tiles, ts, b->d_tile_base, b->d_nt, b->d_n,
                                                             b->partial, b->d_partial_base);
  ++b->launches_per_eval;
  for (int k = 0; k < b->nt_max; ++k) {
    const int A = b->active[k];
    const int A1 = (k + 1 < b->nt_max) ? b->active[k + 1] : 0;
    trsv_batch_kernel<<<A, 1024, ts * sizeof(double), st>>>(b->tiles, ts, k, b->d_tile_base, b->d_nt, b->z,
                                                            b->d_loc_base);
    ++b->launches_per_eval;
    if (A1 > 0) {
      gemv_batch_kernel<<<dim3(ts / kBatchInner, b->nt_max - k - 1, A1), 256, ts * sizeof(double), st>>>(
          b->tiles, ts, k, b->d_tile_base, b->d_nt, b->z, b->d_loc_base);
      ++b->launches_per_eval;
    }
  }
  finalize_batch_kernel<<<b->B, 256, 0, st>>>(b->partial, b->d_partial_base, b->d_nt, b->z, b->d_loc_base, b->d_n,
                                              b->result, b->info);
  ++b->launches_per_eval;
  if (cudaMemcpyAsync(b->h_result, b->result, 4 * b->B * sizeof(double), cudaMemcpyDeviceToHost, st) ||
      cudaMemcpyAsync(b->h_info, b->info, b->B * sizeof(int), cudaMemcpyDeviceToHost, st) ||
      cudaMemcpyAsync(b->h_err, b->err, sizeof(int), cudaMemcpyDeviceToHost, st))
    return check("enqueue_batch_eval/copy");
  return check("enqueue_batch_eval");
}

int round_batch_tile(int dts) {
  int ts = dts < kBatchInner ? kBatchInner : dts;
  return ((ts + kBatchInner - 1) / kBatchInner) * kBatchInner;
}

}  // namespace

extern "C" {

int egs_batch_create(egs_batch** out, int B, const int* n, int dts, const double* x, const double* y,
                     const double* z) {
  if (!out || B <= 0 || B > 65535 || !n || dts <= 0 || !x || !y || !z) return EGS_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set_last_error("no CUDA device visible", "egs_batch_create");
    return EGS_ERR_NO_DEVICE;
  }
  auto* b = new egs_batch();
  b->B = B;
  b->ts = round_batch_tile(dts);
  const int ts = b->ts;
  b->n.assign(n, n + B);
  b->nt.resize(B);
  std::vector<int> caller_nt(B);
  std::vector<long long> caller_off(B + 1, 0);
  for (int i = 0; i < B; ++i) {
    if (n[i] <= 0) {
      free_batch(b);
      return EGS_ERR_INVALID;
    }
    caller_nt[i] = (n[i] + ts - 1) / ts;
    caller_off[i + 1] = caller_off[i] + n[i];
  }
  b->order.resize(B);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) { return caller_nt[a] > caller_nt[c]; });
  for (int p = 0; p < B; ++p) {
    b->n[p] = n[b->order[p]];
    b->nt[p] = caller_nt[b->order[p]];
  }
  b->nt_max = b->nt[0];
  b->active.assign(b->nt_max, 0);
  for (int p = 0; p < B; ++p)
    for (int k = 0; k < b->nt[p]; ++k) b->active[k]++;
  b->tile_base.resize(B);
  b->loc_base.resize(B);
  b->partial_base.resize(B);
  std::vector<int4> tinfo;
  for (int p = 0; p < B; ++p) {
    b->tile_base[p] = b->total_tiles;
    b->loc_base[p] = b->total_loc;
    b->partial_base[p] = b->total_partial;
    const int nt = b->nt[p];
    for (int j = 0; j < nt; ++j)
      for (int i = j; i < nt; ++i) tinfo.push_back(make_int4(p, i, j, 0));
    b->total_tiles += lower_tiles(nt);
    b->total_loc += (long long)nt * ts;
    b->total_partial += nt;
  }
  // host staging of padded, sorted locations and observations
  std::vector<double> hx(b->total_loc, 0.0), hy(b->total_loc, 0.0), hz(b->total_loc, 0.0);
  for (int p = 0; p < B; ++p) {
    const long long src = caller_off[b->order[p]];
    std::copy(x + src, x + src + b->n[p], hx.begin() + b->loc_base[p]);
    std::copy(y + src, y + src + b->n[p], hy.begin() + b->loc_base[p]);
    std::copy(z + src, z + src + b->n[p], hz.begin() + b->loc_base[p]);
  }
  int rc = EGS_OK;
  if ((rc = balloc(b, &b->tiles, (size_t)b->total_tiles * ts * ts)) || (rc = balloc(b, &b->x, b->total_loc)) ||
      (rc = balloc(b, &b->y, b->total_loc)) || (rc = balloc(b, &b->z, b->total_loc)) ||
      (rc = balloc(b, &b->zcpy, b->total_loc)) || (rc = balloc(b, &b->partial, b->total_partial)) ||
      (rc = balloc(b, &b->result, 4 * (size_t)B)) || (rc = balloc(b, &b->info, B)) || (rc = balloc(b, &b->err, 1)) ||
      (rc = balloc(b, &b->d_n, B)) || (rc = balloc(b, &b->d_nt, B)) || (rc = balloc(b, &b->d_tile_base, B)) ||
      (rc = balloc(b, &b->d_loc_base, B)) || (rc = balloc(b, &b->d_partial_base, B)) ||
      (rc = balloc(b, &b->d_tinfo, tinfo.size())) || (rc = balloc(b, &b->d_params, B)) ||
      (rc = balloc(b, &b->d_ktab, (size_t)B * kKtabDoubles))) {
    free_batch(b);
    return rc;
  }
  if (cudaMallocHost(&b->h_params, B * sizeof(MaternParams)) || cudaMallocHost(&b->h_result, 4 * B * sizeof(double)) ||
      cudaMallocHost(&b->h_info, B * sizeof(int)) || cudaMallocHost(&b->h_err, sizeof(int)) ||
      cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) {
    cudaGetLastError();
    set_last_error("pinned host allocation or stream creation failed", "egs_batch_create");
    free_batch(b);
    return EGS_ERR_CUDA;
  }
  b->own_stream = true;
  if (cudaMemcpy(b->x, hx.data(), b->total_loc * sizeof(double), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->y, hy.data(), b->total_loc * sizeof(double), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->zcpy, hz.data(), b->total_loc * sizeof(double), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_n, b->n.data(), B * sizeof(int), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_nt, b->nt.data(), B * sizeof(int), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_tile_base, b->tile_base.data(), B * sizeof(long long), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_loc_base, b->loc_base.data(), B * sizeof(long long), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_partial_base, b->partial_base.data(), B * sizeof(long long), cudaMemcpyHostToDevice) ||
      cudaMemcpy(b->d_tinfo, tinfo.data(), tinfo.size() * sizeof(int4), cudaMemcpyHostToDevice)) {
    rc = check("egs_batch_create/upload");
    free_batch(b);
    return rc;
  }
  if ((rc = gemm_init_tensor_map(b->tmap, b->tiles, ts, b->total_tiles)) != EGS_OK || (rc = build_jobs(b)) != EGS_OK) {
    free_batch(b);
    return rc;
  }
  *out = b;
  return EGS_OK;
}

int egs_batch_destroy(egs_batch* b) {
  free_batch(b);
  return EGS_OK;
}

int egs_batch_info(const egs_batch* b, int* ts, int* nt_max, long long* bytes, long long* launches_per_eval) {
  if (!b) return EGS_ERR_INVALID;
  if (ts) *ts = b->ts;
  if (nt_max) *nt_max = b->nt_max;
  if (bytes) *bytes = b->bytes;
  if (launches_per_eval) *launches_per_eval = b->launches_per_eval;
  return EGS_OK;
}

}  // extern "C"

namespace {

// First half of an evaluation: parameters to the device and the whole batched
// evaluation enqueued on the batch's stream (captured as a graph from the
// second evaluation on).  Returns without waiting.
int batch_launch(egs_batch* b, const double* theta) {
  cudaStream_t st = b->stream;
  if (cudaStreamSynchronize(st) != cudaSuccess) return check("egs_batch_eval");
  for (int p = 0; p < b->B; ++p) {
    const int rc = make_matern_params(theta + 3 * b->order[p], &b->h_params[p]);
    if (rc != EGS_OK) {
      set_last_error("a theta is outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "egs_batch_eval");
      return rc;
    }
  }
  if (b->evals > 0 && !b->graph_exec) {
    // capture the whole evaluation once; replay it from now on
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      cudaMemcpyAsync(b->d_params, b->h_params, b->B * sizeof(MaternParams), cudaMemcpyHostToDevice, st);
      const long long lpe = b->launches_per_eval;
      const int rc = enqueue_batch_eval(b);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(st, &g);
      b->launches_per_eval = lpe;
      if (rc == EGS_OK && e == cudaSuccess && g && cudaGraphInstantiate(&b->graph_exec, g, 0) == cudaSuccess) {
        b->graph = g;
      } else {
        cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        b->graph_exec = nullptr;
      }
    } else {
      cudaGetLastError();
    }
  }
  if (b->graph_exec) {
    if (cudaGraphLaunch(b->graph_exec, st) != cudaSuccess) return check("egs_batch_eval/graph");
  } else {
    if (cudaMemcpyAsync(b->d_params, b->h_params, b->B * sizeof(MaternParams), cudaMemcpyHostToDevice, st))
      return check("egs_batch_eval/params");
    const int rc = enqueue_batch_eval(b);
    if (rc != EGS_OK) return rc;
  }
  ++b->evals;
  return EGS_OK;
}

// Second half: wait for the batch's stream and read every problem's result.
int batch_collect(egs_batch* b, double* loglik, int* status) {
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return check("egs_batch_eval/sync");
  if (*b->h_err != 0) {
    set_last_error("a device-side wait exceeded its limit", "egs_batch_eval");
    return EGS_ERR_TIMEOUT;
  }
  int failures = 0;
  for (int p = 0; p < b->B; ++p) {
    const int i = b->order[p];
    loglik[i] = b->h_result[4 * p];
    if (status) status[i] = b->h_info[p];
    if (b->h_info[p] > 0) ++failures;
  }
  return failures ? EGS_ERR_STATE : EGS_OK;
}

}  // namespace

extern "C" {

int egs_batch_eval(egs_batch* b, const double* theta, double* loglik, int* status) {
  if (!b || !theta || !loglik) return EGS_ERR_INVALID;
  const int rc = batch_launch(b, theta);
  if (rc != EGS_OK) return rc;
  return batch_collect(b, loglik, status);
}

int egs_batch_autotune(int B, const int* n, const double* x, const double* y, const double* z,
                       const double* theta, const int* candidates, int ncand, int* best_ts, double* best_ms) {
  if (!best_ts || !candidates || ncand <= 0) return EGS_ERR_INVALID;
  double best = 1e300;
  int arg = -1;
  std::vector<double> ll(B);
  for (int c = 0; c < ncand; ++c) {
    egs_batch* b = nullptr;
    if (egs_batch_create(&b, B, n, candidates[c], x, y, z) != EGS_OK) continue;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    egs_batch_eval(b, theta, ll.data(), nullptr);  // direct launches
    egs_batch_eval(b, theta, ll.data(), nullptr);  // captures the graph
    cudaEventRecord(e0, b->stream);
    egs_batch_eval(b, theta, ll.data(), nullptr);
    cudaEventRecord(e1, b->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    egs_batch_destroy(b);
    if (ms > 0 && ms < best) {
      best = ms;
      arg = candidates[c];
    }
  }
  if (arg < 0) return EGS_ERR_STATE;
  *best_ts = arg;
  if (best_ms) *best_ms = best;
  return EGS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Size classes: problems cut by N into classes, each an egs_batch with its own
// tile size; one evaluation launches every class on its own stream before it
// waits for any, so the classes' work overlaps on the device.
// ---------------------------------------------------------------------------

struct egs_batch_set {
  int B = 0;
  std::vector<egs_batch*> cls;
  std::vector<std::vector<int>> members;  // caller indices of each class
  std::vector<int> upper, ts;
  std::vector<double> th, ll;
  std::vector<int> st;
};

namespace {

void free_set(egs_batch_set* s) {
  if (!s) return;
  for (egs_batch* b : s->cls) free_batch(b);
  delete s;
}

// Class boundaries: the sorted sizes cut into ncl runs of about equal n^3 cost;
// upper[c] is the largest N of class c.
std::vector<int> cost_boundaries(std::vector<int> sizes, int ncl) {
  std::sort(sizes.begin(), sizes.end());
  double total = 0.0;
  for (int v : sizes) total += (double)v * v * v;
  std::vector<int> upper;
  double acc = 0.0;
  int c = 1;
  for (size_t i = 0; i < sizes.size(); ++i) {
    acc += (double)sizes[i] * sizes[i] * sizes[i];
    if (c < ncl && acc >= total * c / ncl && i + 1 < sizes.size() && sizes[i + 1] > sizes[i]) {
      upper.push_back(sizes[i]);
      ++c;
    }
  }
  upper.push_back(sizes.back());
  return upper;
}

}  // namespace

extern "C" {

int egs_batch_set_create(egs_batch_set** out, int B, const int* n, const double* x, const double* y,
                         const double* z, int nclass, const int* upper_n, const int* dts) {
  if (!out || B <= 0 || !n || !x || !y || !z || nclass <= 0 || nclass > 16 || !upper_n || !dts)
    return EGS_ERR_INVALID;
  *out = nullptr;
  for (int c = 0; c < nclass; ++c)
    if (dts[c] <= 0 || (c > 0 && upper_n[c] <= upper_n[c - 1])) return EGS_ERR_INVALID;
  std::vector<long long> off(B + 1, 0);
  for (int i = 0; i < B; ++i) {
    if (n[i] <= 0) return EGS_ERR_INVALID;
    if (n[i] > upper_n[nclass - 1]) {
      set_last_error("a problem is larger than the last class bound", "egs_batch_set_create");
      return EGS_ERR_INVALID;
    }
    off[i + 1] = off[i] + n[i];
  }
  auto* s = new egs_batch_set();
  s->B = B;
  for (int c = 0; c < nclass; ++c) {
    std::vector<int> mem, nn;
    std::vector<double> cx, cy, cz;
    for (int i = 0; i < B; ++i) {
      const int lo = c > 0 ? upper_n[c - 1] : 0;
      if (n[i] <= lo || n[i] > upper_n[c]) continue;
      mem.push_back(i);
      nn.push_back(n[i]);
      cx.insert(cx.end(), x + off[i], x + off[i + 1]);
      cy.insert(cy.end(), y + off[i], y + off[i + 1]);
      cz.insert(cz.end(), z + off[i], z + off[i + 1]);
    }
    if (mem.empty()) continue;
    egs_batch* b = nullptr;
    const int rc = egs_batch_create(&b, (int)mem.size(), nn.data(), dts[c], cx.data(), cy.data(), cz.data());
    if (rc != EGS_OK) {
      free_set(s);
      return rc;
    }
    s->cls.push_back(b);
    s->members.push_back(std::move(mem));
    s->upper.push_back(upper_n[c]);
    s->ts.push_back(b->ts);
  }
  *out = s;
  return EGS_OK;
}

int egs_batch_set_destroy(egs_batch_set* s) {
  free_set(s);
  return EGS_OK;
}

int egs_batch_set_eval(egs_batch_set* s, const double* theta, double* loglik, int* status) {
  if (!s || !theta || !loglik) return EGS_ERR_INVALID;
  int rc = EGS_OK;
  const size_t ncl = s->cls.size();
  size_t launched = 0;
  for (; launched < ncl; ++launched) {
    const auto& mem = s->members[launched];
    s->th.resize(3 * mem.size());
    for (size_t k = 0; k < mem.size(); ++k)
      for (int q = 0; q < 3; ++q) s->th[3 * k + q] = theta[3 * (size_t)mem[k] + q];
    if ((rc = batch_launch(s->cls[launched], s->th.data())) != EGS_OK) break;
  }
  bool failures = false;
  for (size_t c = 0; c < launched; ++c) {
    const auto& mem = s->members[c];
    s->ll.resize(mem.size());
    s->st.assign(mem.size(), 0);
    const int r = batch_collect(s->cls[c], s->ll.data(), s->st.data());
    if (r == EGS_ERR_STATE) failures = true;
    else if (r != EGS_OK && rc == EGS_OK) rc = r;
    for (size_t k = 0; k < mem.size(); ++k) {
      loglik[mem[k]] = s->ll[k];
      if (status) status[mem[k]] = s->st[k];
    }
  }
  if (rc != EGS_OK) return rc;
  return failures ? EGS_ERR_STATE : EGS_OK;
}

int egs_batch_set_info(const egs_batch_set* s, int* nclass, int* upper_n, int* ts, long long* bytes) {
  if (!s) return EGS_ERR_INVALID;
  if (nclass) *nclass = (int)s->cls.size();
  long long total = 0;
  for (size_t c = 0; c < s->cls.size(); ++c) {
    if (upper_n) upper_n[c] = s->upper[c];
    if (ts) ts[c] = s->ts[c];
    total += s->cls[c]->bytes;
  }
  if (bytes) *bytes = total;
  return EGS_OK;
}

int egs_batch_set_autotune(int B, const int* n, const double* x, const double* y, const double* z,
                           const double* theta, const int* candidates, int ncand, int max_classes, int* nclass,
                           int* upper_n, int* dts, double* best_ms) {
  if (B <= 0 || !n || !x || !y || !z || !theta || !candidates || ncand <= 0 || max_classes <= 0 ||
      max_classes > 16 || !nclass || !upper_n || !dts)
    return EGS_ERR_INVALID;
  std::vector<long long> off(B + 1, 0);
  for (int i = 0; i < B; ++i) off[i + 1] = off[i] + n[i];
  double best = 1e300;
  std::vector<double> ll(B);
  for (int ncl = 1; ncl <= max_classes; ++ncl) {
    const std::vector<int> upper = cost_boundaries(std::vector<int>(n, n + B), ncl);
    if ((int)upper.size() < ncl) break;  // fewer distinct sizes than classes
    // each class's tile size, timed on the class alone
    std::vector<int> ts(upper.size());
    bool ok = true;
    for (size_t c = 0; c < upper.size() && ok; ++c) {
      const int lo = c > 0 ? upper[c - 1] : 0;
      std::vector<int> nn;
      std::vector<double> cx, cy, cz, ct;
      for (int i = 0; i < B; ++i) {
        if (n[i] <= lo || n[i] > upper[c]) continue;
        nn.push_back(n[i]);
        cx.insert(cx.end(), x + off[i], x + off[i + 1]);
        cy.insert(cy.end(), y + off[i], y + off[i + 1]);
        cz.insert(cz.end(), z + off[i], z + off[i + 1]);
        ct.insert(ct.end(), theta + 3 * (size_t)i, theta + 3 * (size_t)i + 3);
      }
      ok = egs_batch_autotune((int)nn.size(), nn.data(), cx.data(), cy.data(), cz.data(), ct.data(), candidates,
                              ncand, &ts[c], nullptr) == EGS_OK;
    }
    if (!ok) continue;
    // the whole set, classes overlapping: one direct evaluation, one capture, one timed replay
    egs_batch_set* s = nullptr;
    if (egs_batch_set_create(&s, B, n, x, y, z, (int)upper.size(), upper.data(), ts.data()) != EGS_OK) continue;
    egs_batch_set_eval(s, theta, ll.data(), nullptr);
    egs_batch_set_eval(s, theta, ll.data(), nullptr);
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = egs_batch_set_eval(s, theta, ll.data(), nullptr);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    egs_batch_set_destroy(s);
    if ((rc == EGS_OK || rc == EGS_ERR_STATE) && ms < best) {
      best = ms;
      *nclass = (int)upper.size();
      for (size_t c = 0; c < upper.size(); ++c) {
        upper_n[c] = upper[c];
        dts[c] = ts[c];
      }
    }
  }
  if (best >= 1e300) return EGS_ERR_STATE;
  if (best_ms) *best_ms = best;
  return EGS_OK;
}

}  // extern "C"
