// extern "C" boundary of the B200 maximum-likelihood path and the host-side
// driver that sequences the device kernels of one evaluation.
//
// The evaluation follows ChameleonImplementation<T>::ExaGeoStatMLETile
// (src/linear-algebra-solvers/concrete/chameleon/ChameleonImplementation.cpp:35-327):
//   Z <- Zcpy (:113-125), C <- Matern(theta) lower tiles (:168-174),
//   C <- chol(C) (:180), logdet (:188-192), Z <- L^-1 Z (:216), dot (:224),
//   loglik (:257-265).
// All stages of one evaluation are enqueued on the problem's stream; the host
// blocks once per evaluation to read a 32-byte result record.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <cuda.h>
#include "common.cuh"
#include "kernels.cuh"

namespace egs {

static thread_local std::string g_last_error;

void set_last_error(const char* what, const char* where) {
  g_last_error = std::string(what ? what : "") + (where ? std::string(" [") + where + "]" : std::string());
}

}  // namespace egs

using namespace egs;

struct egs_problem {
  int n = 0, dts = 0, ts = 0, nt = 0, np = 0;
  long long ntiles = 0;
  long long bytes = 0;
  double* tiles = nullptr;
  double* x = nullptr;
  double* y = nullptr;
  double* z = nullptr;
  double* zcpy = nullptr;
  double* partial = nullptr;
  double* result = nullptr;
  int* flags = nullptr;  // [0] potrf info, [1] device wait error
  MaternParams* dparams = nullptr;
  double* ktab = nullptr;  // Chebyshev table of K_nu for the current theta (kKtabDoubles)
  // pinned host mirrors
  MaternParams* hparams = nullptr;
  double* hresult = nullptr;
  int* hflags = nullptr;
  alignas(64) unsigned char tmap[128];
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool have_locations = false;
  bool have_observations = false;
  // Mixed precision only: the order in which the device holds the points
  // (perm[d] = caller index of device point d), empty when it is the caller's.
  std::vector<int> perm;
  int band = 0;  // >= 1: diagonal super-tile approximation with this tile band
  // Replay of a whole evaluation: captured at the second evaluation, relaunched after.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_band = -1;
  long long graph_launches[EGS_NUM_STAGES] = {};
  long long evals = 0;
  bool graphs_enabled = true;
  // The same with the per-stage timing events captured as event-record nodes
  // (used while profiling); pgraphs_ok turns off only this variant.
  cudaGraph_t pgraph = nullptr;
  cudaGraphExec_t pgraph_exec = nullptr;
  int pgraph_band = -1;
  long long pgraph_launches[EGS_NUM_STAGES] = {};
  bool pgraphs_ok = true;
  // Per-stage accounting: launch counts always, CUDA-event times when profiling.
  bool profiling = false;
  struct Span {
    int stage;
    cudaEvent_t a, b;
    double flops;
  };
  std::vector<cudaEvent_t> events;
  size_t events_used = 0;
  std::vector<Span> spans;
  std::vector<Span> pgraph_spans;  // the spans of one replay of pgraph
  double stage_ms[EGS_NUM_STAGES] = {};
  double stage_flops[EGS_NUM_STAGES] = {};
  long long stage_launches[EGS_NUM_STAGES] = {};
  // Mixed precision (precision == EGS_PRECISION_MIXED): FP64 band of mband tile
  // rows below the diagonal, FP32 off-band tiles; see mixed.cu for the layout.
  int precision = EGS_PRECISION_DOUBLE;
  int mband = 0;
  double* band_pool = nullptr;
  float* off_pool = nullptr;
  double* W = nullptr;        // one FP64 tile column (panel workspace) + one identity tile
  double* inv_pool = nullptr; // L_kk^-T of every diagonal tile
  double* solve_tmp = nullptr;
  __half* ph = nullptr;       // FP16 split of the solved panel rows (hi, lo)
  __half* pl = nullptr;
  float* inv_scale = nullptr; // per panel row
  double* w = nullptr;        // refinement vector
  double* res_scratch = nullptr;
  int4* gen_tiles = nullptr;  // (i, j, pool, slot) of every generated tile
  long long ngen = 0;
  GemmDesc* band_jobs = nullptr;
  long long* band_begin = nullptr;
  struct JobLaunch {
    long long job_off, begin_off;
    int njobs;
    long long total;
  };
  std::vector<JobLaunch> band_launch;  // per step k
  // Ozaki-scheme band update: int8 slices of the panel rows, row scales, and
  // per-step target tables (offset into oz_targets, count, work items)
  int band_method = EGS_BAND_OZAKI_INT8;
  int8_t* oz_slices = nullptr;
  double* oz_scale = nullptr;
  int4* oz_targets = nullptr;
  struct OzLaunch {
    long long off;
    int count;
    long long items;
  };
  std::vector<OzLaunch> oz_launch;
  int4* oz_trsm_targets = nullptr;
  std::vector<OzLaunch> oz_trsm_launch;
  double* W2 = nullptr;  // short panel: diagonal tile, band tiles, identity
  // look-ahead: the short panel of step k+1 runs on `side` while the off-band
  // update of step k runs on the other SMs of the problem stream
  cudaStream_t side = nullptr;
  cudaEvent_t ev_band = nullptr, ev_panel = nullptr;
  int lookahead_sms = 0;  // SMs left to the look-ahead panel (0: no look-ahead)
  alignas(64) unsigned char tm_oz[128];
  alignas(64) unsigned char tmapW2[128];
  alignas(64) unsigned char tmapW[128];
  alignas(64) unsigned char tm_hi[128];
  alignas(64) unsigned char tm_lo[128];
  alignas(64) unsigned char tm_c[128];
};

namespace {

constexpr int kInnerBlock = 64;
constexpr int kOuterBlock = 256;
constexpr int kPrecisionBroken = -1;  // egs_problem_set_precision failed part-way

int round_tile(int dts) {
  int ts = dts < kInnerBlock ? kInnerBlock : dts;
  return ((ts + kInnerBlock - 1) / kInnerBlock) * kInnerBlock;
}

int check_cuda(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), where);
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

cudaEvent_t take_event(egs_problem* p) {
  if (p->events_used == p->events.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    p->events.push_back(e);
  }
  return p->events[p->events_used++];
}

// Opens a timed span of `stage` on the problem stream (no-op unless profiling).
int span_begin(egs_problem* p, int stage, cudaStream_t on = nullptr) {
  if (!p->profiling) return -1;
  egs_problem::Span s{stage, take_event(p), take_event(p), 0.0};
  // "external" records: inside a stream capture they become event-record
  // nodes of the graph (a plain record would only mark a dependency)
  cudaEventRecordWithFlags(s.a, on ? on : p->stream, cudaEventRecordExternal);
  p->spans.push_back(s);
  return (int)p->spans.size() - 1;
}

void span_end(egs_problem* p, int idx, double flops, cudaStream_t on = nullptr) {
  if (idx < 0) return;
  cudaEventRecordWithFlags(p->spans[idx].b, on ? on : p->stream, cudaEventRecordExternal);
  p->spans[idx].flops = flops;
}

void count_launches(egs_problem* p, int stage, long long n) { p->stage_launches[stage] += n; }

// After the stream has been synchronised: fold the recorded spans into the
// totals; returns how many spans had a valid time.
int collect_spans(egs_problem* p) {
  int timed = 0;
  for (auto& s : p->spans) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s.a, s.b) == cudaSuccess) {
      p->stage_ms[s.stage] += ms;
      p->stage_flops[s.stage] += s.flops;
      ++timed;
    }
  }
  cudaGetLastError();
  p->spans.clear();
  p->events_used = 0;
  return timed;
}

// Both captured evaluations (after a change of the problem's layout or method).
void drop_graphs(egs_problem* p) {
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->pgraph_exec) cudaGraphExecDestroy(p->pgraph_exec);
  if (p->pgraph) cudaGraphDestroy(p->pgraph);
  p->graph_exec = p->pgraph_exec = nullptr;
  p->graph = p->pgraph = nullptr;
  p->pgraph_spans.clear();
}

// Device buffers come from the stream-ordered allocator on the owning
// problem's stream: neither the allocation nor the release synchronises the
// device, so problems can be created and destroyed while other problems'
// work is running (the serving loop relies on this).
template <typename T>
int dev_alloc(T** p, size_t count, long long* bytes, cudaStream_t st) {
  const size_t b = count * sizeof(T);
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), b, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(cudaGetErrorString(e), "cudaMallocAsync");
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? EGS_ERR_OOM : EGS_ERR_CUDA;
  }
  *bytes += (long long)b;
  return EGS_OK;
}

void dev_free(void* ptr, cudaStream_t st) {
  if (ptr) cudaFreeAsync(ptr, st);
}

// Small pinned host records (parameter block, result record, status words) are
// 256-byte chunks of slabs that live until the process exits: cudaFreeHost
// would synchronise the device.
constexpr size_t kPinnedChunk = 256;
constexpr size_t kPinnedSlabChunks = 256;
std::mutex g_pinned_mutex;
std::vector<void*> g_pinned_free;

void* pinned_record() {
  std::lock_guard<std::mutex> lock(g_pinned_mutex);
  if (g_pinned_free.empty()) {
    void* slab = nullptr;
    if (cudaMallocHost(&slab, kPinnedChunk * kPinnedSlabChunks) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    for (size_t i = 0; i < kPinnedSlabChunks; ++i) g_pinned_free.push_back(static_cast<char*>(slab) + i * kPinnedChunk);
  }
  void* r = g_pinned_free.back();
  g_pinned_free.pop_back();
  return r;
}

void pinned_release(void* r) {
  if (!r) return;
  std::lock_guard<std::mutex> lock(g_pinned_mutex);
  g_pinned_free.push_back(r);
}

void free_mixed(egs_problem* p) {
  void* bufs[] = {p->band_pool, p->off_pool, p->W,         p->ph,      p->pl,          p->inv_scale,
                  p->w,         p->res_scratch, p->gen_tiles, p->band_jobs, p->band_begin, p->inv_pool,
                  p->solve_tmp, p->oz_slices, p->oz_scale, p->oz_targets, p->oz_trsm_targets, p->W2};
  for (void* b : bufs) dev_free(b, p->stream);
  p->band_pool = nullptr;
  p->off_pool = nullptr;
  p->W = nullptr;
  p->inv_pool = p->solve_tmp = nullptr;
  p->oz_slices = nullptr;
  p->oz_scale = nullptr;
  p->oz_targets = nullptr;
  p->oz_launch.clear();
  p->oz_trsm_targets = nullptr;
  p->oz_trsm_launch.clear();
  p->W2 = nullptr;
  if (p->side) {
    cudaStreamSynchronize(p->side);
    cudaStreamDestroy(p->side);
  }
  if (p->ev_band) cudaEventDestroy(p->ev_band);
  if (p->ev_panel) cudaEventDestroy(p->ev_panel);
  p->side = nullptr;
  p->ev_band = p->ev_panel = nullptr;
  p->ph = p->pl = nullptr;
  p->inv_scale = nullptr;
  p->w = p->res_scratch = nullptr;
  p->gen_tiles = nullptr;
  p->band_jobs = nullptr;
  p->band_begin = nullptr;
  p->band_launch.clear();
  p->ngen = 0;
}

void free_problem(egs_problem* p) {
  if (!p) return;
  if (p->stream) cudaStreamSynchronize(p->stream);
  void* bufs[] = {p->tiles, p->x, p->y, p->z, p->zcpy, p->partial, p->result, p->flags, p->dparams, p->ktab};
  for (void* b : bufs) dev_free(b, p->stream);
  free_mixed(p);
  pinned_release(p->hparams);
  pinned_release(p->hresult);
  pinned_release(p->hflags);
  drop_graphs(p);
  if (p->stream) cudaStreamSynchronize(p->stream);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  for (cudaEvent_t e : p->events) cudaEventDestroy(e);
  delete p;
}

// Panel of step k (tile column k of an nt-tile lower layout): factor diagonal
// tile (k, k) and solve tiles (k+1 .. nt-1, k) against it, as one right-looking
// blocked factorisation of the tall tile column.  Two-level blocking: the
// tile's columns go in outer blocks of kOuterBlock; inside an outer block each
// 64-column block is factored (64x64 potrf), every row below it -- the rest of
// the diagonal tile and all tiles below -- is solved in one row-solve launch,
// and one K = 64 update covers the remaining columns of the same outer block
// for all those rows; the columns right of the outer block then get one
// update with K = kOuterBlock.  The K = 64 updates thus touch at most 192
// columns, which cuts the read-modify-write traffic of the panel's C operand
// by ~2.5x against single-level 64-blocking.  Every element receives the same
// operations in the same order as with the diagonal tile factored first.
// col_base is the global column of the tile (for the LAPACK-style info of a
// failed pivot).  Returns the launch count in *nl.
int enqueue_panel(double* tiles, const void* tmap, int ts, int nt, int k, int col_base, int* info, int* err,
                  cudaStream_t st, long long* nl, int max_ctas = 0) {
  const long long skk = tile_slot(k, k, nt);
  const int ntp = nt - k;         // tiles of the column, the diagonal one first
  const int drow = k * ts;
  const int row_end = nt * ts;    // end of the column's global rows
  for (int KB = 0; KB < ts; KB += kOuterBlock) {
    const int KE = std::min(ts, KB + kOuterBlock);
    for (int kb = KB; kb < KE; kb += kInnerBlock) {
      launch_potrf_diag_block(tiles, ts, skk, kb, col_base, info, st);
      ++*nl;
      const int r0 = drow + kb + kInnerBlock;  // first row below the block
      if (r0 >= row_end) continue;
      launch_trsm_rows_panel(tiles, ts, skk, ntp, kb + kInnerBlock, 0, kb, skk, st);
      ++*nl;
      if (kb + kInnerBlock < KE) {
        int rc = launch_gemm_rows(tmap, tiles, ts, nt, row_end - r0, KE - kb - kInnerBlock, kInnerBlock, r0, kb, k,
                                  r0, kb, k, r0, r0, 1, err, st, max_ctas);
        if (rc != EGS_OK) return rc;
        ++*nl;
      }
    }
    if (KE < ts) {
      const int r0 = drow + KE;
      int rc = launch_gemm_rows(tmap, tiles, ts, nt, row_end - r0, ts - KE, KE - KB, r0, KB, k, r0, KB, k, r0, r0, 1,
                                err, st, max_ctas);
      if (rc != EGS_OK) return rc;
      ++*nl;
    }
  }
  return EGS_OK;
}

// Right-looking tiled Cholesky of the lower tiles (replaces CHAMELEON_dpotrf_Tile).
// Step k: factor diagonal tile k (64-wide blocked: potrf of the 64x64 block,
// row solve below it, tensor-core syrk of the rest of the tile), solve the tile
// column below it (64-wide blocked: row solve + tensor-core update), then the
// tensor-core trailing update of every tile (i, j), k < j <= i.
int enqueue_potrf(egs_problem* p, int steps = -1) {
  const int ts = p->ts, nt = p->nt, n = p->n;
  cudaStream_t st = p->stream;
  int* info = p->flags;
  int* err = p->flags + 1;
  const int kend = (steps >= 0 && steps < nt) ? steps : nt;
  for (int k = 0; k < kend; ++k) {
    const long long skk = tile_slot(k, k, nt);
    int sp = span_begin(p, EGS_STAGE_PANEL);
    long long nl = 0;
    int rc = enqueue_panel(p->tiles, p->tmap, ts, nt, k, k * ts, info, err, st, &nl);
    if (rc != EGS_OK) return rc;
    count_launches(p, EGS_STAGE_PANEL, nl);
    // Algorithmic flops of the panel step on the real (unpadded) rows: potrf of the
    // diagonal block plus the triangular solve of the rows below it.
    {
      const double w = (double)std::min(ts, n - k * ts);
      const double below = (double)std::max(0, n - (k + 1) * ts);
      span_end(p, sp, w * w * w / 3.0 + w * w / 2.0 + w / 6.0 + below * w * w);
    }
    if (k < nt - 1) {
      sp = span_begin(p, EGS_STAGE_UPDATE);
      int rc = launch_gemm_trailing(p->tmap, p->tiles, ts, nt, k, err, st);
      if (rc != EGS_OK) return rc;
      count_launches(p, EGS_STAGE_UPDATE, 1);
      const double m = (double)std::max(0, n - (k + 1) * ts);
      span_end(p, sp, m * (m + 1.0) * (double)ts);
    }
  }
  return check_cuda("enqueue_potrf");
}

// Diagonal super-tile (band) approximation of the factorisation, following
// ChameleonDST<T>::ExaGeoStatParallelPotrfDiagonal (src/linear-algebra-solvers/
// concrete/chameleon/dst/ChameleonDST.cpp:90-150): at step k only tiles (m, k)
// with m < k + band are solved, and only tiles (m, n) with k < n < k + band,
// n <= m < n + band are updated; the update reads tile (m, k) whether or not it
// was solved, and tiles outside the band keep their covariance values.
// Caller tiles that are not device tiles (dts not a multiple of 64) take the
// element-level form of the same loop on logical tiles of dts (dst.cu).
int enqueue_potrf_band(egs_problem* p) {
  const int ts = p->ts, nt = p->nt, n = p->n, band = p->band;
  cudaStream_t st = p->stream;
  int* info = p->flags;
  int* err = p->flags + 1;
  if (p->dts != ts) {
    const int sp = span_begin(p, EGS_STAGE_PANEL);
    const int rc = launch_dst_band(p->tiles, ts, nt, n, p->dts, band, info, st);
    const int ntl = (n + p->dts - 1) / p->dts;
    count_launches(p, EGS_STAGE_PANEL, 3LL * ntl);
    span_end(p, sp, 0.0);
    return rc;
  }
  for (int k = 0; k < nt; ++k) {
    const long long skk = tile_slot(k, k, nt);
    int sp = span_begin(p, EGS_STAGE_PANEL);
    for (int kb = 0; kb < ts; kb += kInnerBlock) {
      launch_potrf_diag_block(p->tiles, ts, skk, kb, k * ts, info, st);
      count_launches(p, EGS_STAGE_PANEL, 1);
      if (kb + kInnerBlock < ts) {
        launch_trsm_rows(p->tiles, ts, skk, 1, kb + kInnerBlock, kb, skk, st);
        const int r0 = k * ts + kb + kInnerBlock;
        const int m = ts - kb - kInnerBlock;
        int rc = launch_gemm_rows(p->tmap, p->tiles, ts, nt, m, m, kInnerBlock, r0, kb, k, r0, kb, k, r0, r0, 1,
                                  err, st);
        if (rc != EGS_OK) return rc;
        count_launches(p, EGS_STAGE_PANEL, 2);
      }
    }
    const int mend = std::min(nt, k + band);  // solved tiles: k < m < mend
    const int ntl = mend - k - 1;
    if (ntl > 0) {
      const long long s0 = tile_slot(k + 1, k, nt);
      for (int kb = 0; kb < ts; kb += kInnerBlock) {
        launch_trsm_rows(p->tiles, ts, s0, ntl, 0, kb, skk, st);
        count_launches(p, EGS_STAGE_PANEL, 1);
        if (kb + kInnerBlock < ts) {
          const int ncols = ts - kb - kInnerBlock;
          const int brow = k * ts + kb + kInnerBlock;
          int rc = launch_gemm_rows(p->tmap, p->tiles, ts, nt, ntl * ts, ncols, kInnerBlock, (k + 1) * ts, kb, k,
                                    brow, kb, k, (k + 1) * ts, brow, 0, err, st);
          if (rc != EGS_OK) return rc;
          count_launches(p, EGS_STAGE_PANEL, 1);
        }
      }
    }
    span_end(p, sp, 0.0);
    sp = span_begin(p, EGS_STAGE_UPDATE);
    double flops = 0.0;
    for (int c = k + 1; c < mend; ++c) {
      // tiles (m, c), c <= m < min(nt, c + band): one launch on the global rows of that range
      const int rows = (std::min(nt, c + band) - c) * ts;
      int rc = launch_gemm_rows(p->tmap, p->tiles, ts, nt, rows, ts, ts, c * ts, 0, k, c * ts, 0, k, c * ts, c * ts,
                                1, err, st);
      if (rc != EGS_OK) return rc;
      count_launches(p, EGS_STAGE_UPDATE, 1);
      const double rr = (double)std::max(0, std::min(n, std::min(nt, c + band) * ts) - c * ts);
      const double cc = (double)std::max(0, std::min(n, (c + 1) * ts) - c * ts);
      flops += 2.0 * rr * cc * ts - cc * (cc - 1.0) * ts;
    }
    span_end(p, sp, flops);
  }
  return check_cuda("enqueue_potrf_band");
}

// Z := L^-1 Z, tile by tile (forward substitution).
void enqueue_trsv(egs_problem* p) {
  const int sp = span_begin(p, EGS_STAGE_SOLVE);
  for (int k = 0; k < p->nt; ++k) {
    launch_trsv_diag(p->tiles, p->ts, tile_slot(k, k, p->nt), p->z + (long long)k * p->ts, p->stream);
    launch_gemv_panel(p->tiles, p->ts, p->nt, k, p->z, p->stream);
    count_launches(p, EGS_STAGE_SOLVE, k < p->nt - 1 ? 2 : 1);
  }
  span_end(p, sp, (double)p->n * (double)p->n);
}

// Z := L^-T Z (backward substitution), the second half of dposv.
void enqueue_trsv_t(egs_problem* p) {
  const int sp = span_begin(p, EGS_STAGE_SOLVE);
  for (int k = p->nt - 1; k >= 0; --k) {
    launch_trsv_t_diag(p->tiles, p->ts, tile_slot(k, k, p->nt), p->z + (long long)k * p->ts, p->stream);
    launch_gemv_t_panel(p->tiles, p->ts, p->nt, k, p->z, p->stream);
    count_launches(p, EGS_STAGE_SOLVE, k > 0 ? 2 : 1);
  }
  span_end(p, sp, (double)p->n * (double)p->n);
}

int set_params(egs_problem* p, const double* theta) {
  if (!theta) return EGS_ERR_INVALID;
  MaternParams mp;
  int rc = make_matern_params(theta, &mp);
  if (rc != EGS_OK) {
    set_last_error("theta outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "make_matern_params");
    return rc;
  }
  // The pinned mirror may still be read by an earlier in-flight copy.
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  *p->hparams = mp;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->dparams, p->hparams, sizeof(MaternParams), cudaMemcpyHostToDevice, p->stream));
  return EGS_OK;
}

int sync_flags(egs_problem* p, bool want_result) {
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hflags, p->flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  if (want_result)
    EGS_CUDA_TRY(cudaMemcpyAsync(p->hresult, p->result, 4 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  collect_spans(p);
  if (p->hflags[1] != 0) {
    set_last_error("a device-side wait exceeded its limit", "tensor-core update");
    return EGS_ERR_TIMEOUT;
  }
  if (p->hflags[0] > 0) {
    set_last_error("Matrix is not positive definite", "potrf");
    return p->hflags[0];
  }
  return EGS_OK;
}

// Device work of one evaluation after the parameter record is on the device:
// Z <- Zcpy, generation, factorisation, log-det, solve, assembly, and the copy
// of the result record and status words to the pinned host mirrors.
int enqueue_eval_mixed(egs_problem* p);

int enqueue_eval(egs_problem* p) {
  if (p->precision == EGS_PRECISION_MIXED) return enqueue_eval_mixed(p);
  cudaStream_t st = p->stream;
  EGS_CUDA_TRY(cudaMemsetAsync(p->flags, 0, 2 * sizeof(int), st));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, st));
  int sp = span_begin(p, EGS_STAGE_GENERATE);
  int rc = launch_matern_tiles(p->tiles, p->x, p->y, p->n, p->ts, p->nt, p->dparams, p->ktab, st);
  if (rc != EGS_OK) return rc;
  count_launches(p, EGS_STAGE_GENERATE, 1 + (lower_tiles(p->nt) + 65534) / 65535);
  span_end(p, sp, 0.0);
  rc = p->band > 0 ? enqueue_potrf_band(p) : enqueue_potrf(p);
  if (rc != EGS_OK) return rc;
  sp = span_begin(p, EGS_STAGE_REDUCE);
  launch_logdet_partials(p->tiles, p->ts, p->nt, p->n, p->partial, st);
  span_end(p, sp, 0.0);
  count_launches(p, EGS_STAGE_REDUCE, 1);
  enqueue_trsv(p);
  sp = span_begin(p, EGS_STAGE_REDUCE);
  launch_finalize(p->partial, p->nt, p->z, p->n, p->result, p->flags, st);
  span_end(p, sp, 0.0);
  count_launches(p, EGS_STAGE_REDUCE, 1);
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hflags, p->flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hresult, p->result, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  return check_cuda("egs_mle_eval");
}

// Off-band update (split-FP16 tensor cores) of step k on stream st.
static int enqueue_offband_update(egs_problem* p, int k, cudaStream_t st, int max_ctas) {
  const int ts = p->ts, nt = p->nt, b = p->mband;
  const long long off_targets = split_targets(nt, b, k);
  if (off_targets <= 0) return EGS_OK;
  int sp = span_begin(p, EGS_STAGE_UPDATE_LOW);
  int rc = launch_split_update(p->tm_hi, p->tm_lo, p->tm_c, ts, nt, b, k, p->off_pool, p->inv_scale,
                               p->flags + 1, st, max_ctas);
  if (rc != EGS_OK) return rc;
  count_launches(p, EGS_STAGE_UPDATE_LOW, 1);
  span_end(p, sp, 2.0 * (double)off_targets * (double)ts * ts * ts);
  return EGS_OK;
}

// Algorithmic flops of the band update of step k: syrk (ts^3 + ts^2) on the
// diagonal targets, gemm (2 ts^3) below them.
static double band_update_flops(int ts, int nt, int b, int k) {
  double f = 0.0;
  const double t = (double)ts;
  for (int j = k + 1; j < nt; ++j) f += t * t * (t + 1.0) + 2.0 * (double)(std::min(nt - 1, j + b) - j) * t * t * t;
  return f;
}

static double panel_flops(int ts, int n, int k) {
  const double wd = (double)std::min(ts, n - k * ts);
  const double below = (double)std::max(0, n - (k + 1) * ts);
  return wd * wd * wd / 3.0 + wd * wd / 2.0 + wd / 6.0 + below * wd * wd;
}

static int enqueue_mixed_head(egs_problem* p) {
  cudaStream_t st = p->stream;
  EGS_CUDA_TRY(cudaMemsetAsync(p->flags, 0, 2 * sizeof(int), st));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, st));
  int sp = span_begin(p, EGS_STAGE_GENERATE);
  launch_matern_mixed(p->band_pool, p->off_pool, p->x, p->y, p->n, p->ts, p->gen_tiles, p->ngen, p->dparams,
                      p->ktab, st);
  count_launches(p, EGS_STAGE_GENERATE, 1 + (p->ngen + 65534) / 65535);
  span_end(p, sp, 0.0);
  return EGS_OK;
}

// Log-det, the two solves with the refinement residual, the assembly and the
// copies of the result record: the tail of every mixed evaluation.
static int enqueue_mixed_tail(egs_problem* p) {
  cudaStream_t st = p->stream;
  const int ts = p->ts, nt = p->nt, n = p->n, b = p->mband;
  int sp = span_begin(p, EGS_STAGE_REDUCE);
  launch_logdet_band(p->band_pool, ts, nt, b, n, p->partial, st);
  count_launches(p, EGS_STAGE_REDUCE, 1);
  span_end(p, sp, 0.0);
  sp = span_begin(p, EGS_STAGE_SOLVE);
  long long ns = 0;
  launch_mixed_solve(p->band_pool, p->off_pool, p->inv_pool, ts, nt, b, p->z, p->solve_tmp, st, &ns);
  launch_matern_residual(p->x, p->y, p->zcpy, p->z, n, p->np, p->dparams, p->ktab, p->res_scratch, p->w, st);
  launch_mixed_solve(p->band_pool, p->off_pool, p->inv_pool, ts, nt, b, p->w, p->solve_tmp, st, &ns);
  count_launches(p, EGS_STAGE_SOLVE, ns + 2);
  span_end(p, sp, 6.0 * (double)n * (double)n);
  sp = span_begin(p, EGS_STAGE_REDUCE);
  launch_finalize_mixed(p->partial, nt, p->zcpy, p->z, p->w, n, p->result, p->flags, st);
  count_launches(p, EGS_STAGE_REDUCE, 1);
  span_end(p, sp, 0.0);
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hflags, p->flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hresult, p->result, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  return check_cuda("egs_mle_eval (mixed)");
}

// Short panel of step k on stream s: gather the diagonal tile, the band tiles
// and an identity tile into W2, factor and solve them with the FP64 panel
// kernels (the identity row becomes L_kk^-T), scatter back.  max_ctas bounds
// the persistent update kernels of the panel (look-ahead on spare SMs).
static int enqueue_short_panel(egs_problem* p, int k, cudaStream_t s, int max_ctas) {
  const int ts = p->ts, nt = p->nt, b = p->mband;
  const int nb = std::min(b, nt - k - 1);
  int sp = span_begin(p, EGS_STAGE_PANEL, s);
  long long nl = 0;
  launch_gather_panel(p->band_pool, p->W2, ts, b, nb, k, s);
  if (int rc = enqueue_panel(p->W2, p->tmapW2, ts, nb + 2, 0, k * ts, p->flags, p->flags + 1, s, &nl, max_ctas))
    return rc;
  launch_scatter_panel(p->W2, p->band_pool, p->inv_pool, p->W, ts, b, nb, k, s);
  count_launches(p, EGS_STAGE_PANEL, nl + 2);
  span_end(p, sp, panel_flops(ts, p->n, k), s);
  return EGS_OK;
}

// Mixed-precision evaluation, Ozaki form.  Step k on the problem stream: solve
// the off-band rows of tile column k as one product with L_kk^-1 on the int8
// tensor cores (read from the FP32 pool, written to W in FP64, rounded back),
// split the panel rows to FP16, update the FP64 band (Ozaki) and, on all but
// lookahead_sms SMs, the off-band targets (split-FP16).  The short FP64 panel
// of step k+1 (diagonal tile, band rows, L^-T) needs only the band update of
// step k, so it runs on the side stream during the off-band update of step k.
int enqueue_eval_mixed_ozaki(egs_problem* p) {
  cudaStream_t st = p->stream, side = p->side;
  const int ts = p->ts, nt = p->nt, b = p->mband;
  int* err = p->flags + 1;
  if (int rc = enqueue_mixed_head(p)) return rc;
  if (int rc = enqueue_short_panel(p, 0, st, 0)) return rc;
  for (int k = 0; k < nt; ++k) {
    const int ntp = nt - k;
    const int nb = std::min(b, ntp - 1);
    if (k > 0) EGS_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_panel, 0));
    int sp = span_begin(p, EGS_STAGE_PANEL);
    long long nl = 0;
    const egs_problem::OzLaunch& T = p->oz_trsm_launch[k];
    if (T.count > 0) {
      const long long srows = (long long)p->np + ts;
      launch_ozaki_slice_f32(offband_tile(p->off_pool, ts, nt, b, k + nb + 1, k), ts, T.count, k + nb + 1,
                             p->oz_scale, p->oz_slices, srows, st);
      launch_ozaki_slice_rows(p->W2 + (size_t)(nb + 1) * ts * ts, ts, p->np, p->oz_scale, p->oz_slices, srows, st);
      if (int rc = launch_ozaki_trsm(p->tm_oz, p->oz_trsm_targets + T.off, T.count, T.items, ts, k, p->np, p->W,
                                     p->oz_scale, err, st))
        return rc;
      launch_scatter_offband(p->W, p->off_pool, ts, nt, b, nb, k, st);
      nl += 5;
    }
    if (ntp > 1) {
      // one read of the solved rows: FP16 hi/lo for the off-band update, int8
      // slices for the band update
      launch_panel_prepare(p->W, ts, 1, ntp - 1, k, p->oz_scale, p->oz_slices, (long long)p->np + ts,
                           p->inv_scale, p->ph, p->pl, st);
      nl += 1;
    }
    count_launches(p, EGS_STAGE_PANEL, nl);
    span_end(p, sp, 0.0);
    if (ntp <= 1) continue;
    sp = span_begin(p, EGS_STAGE_UPDATE);
    const egs_problem::OzLaunch& O = p->oz_launch[k];
    if (O.count > 0) {
      if (int rc = launch_ozaki_band(p->tm_oz, p->oz_targets + O.off, O.count, O.items, ts, b, p->band_pool,
                                     p->oz_scale, err, st))
        return rc;
      count_launches(p, EGS_STAGE_UPDATE, 1);
    }
    span_end(p, sp, band_update_flops(ts, nt, b, k));
    const int la = p->lookahead_sms;
    if (la > 0) {
      // look-ahead: the next short panel beside the off-band update
      EGS_CUDA_TRY(cudaEventRecord(p->ev_band, st));
      EGS_CUDA_TRY(cudaStreamWaitEvent(side, p->ev_band, 0));
      if (int rc = enqueue_short_panel(p, k + 1, side, la)) return rc;
      EGS_CUDA_TRY(cudaEventRecord(p->ev_panel, side));
      if (int rc = enqueue_offband_update(p, k, st, gemm_num_sms() - la)) return rc;
    } else {
      if (int rc = enqueue_offband_update(p, k, st, 0)) return rc;
      if (int rc = enqueue_short_panel(p, k + 1, st, 0)) return rc;
      EGS_CUDA_TRY(cudaEventRecord(p->ev_panel, st));
    }
  }
  return enqueue_mixed_tail(p);
}

// Mixed-precision evaluation, FP64-DMMA form.  Step k: gather tile column k into
// the FP64 workspace W, factor and solve it there (the FP64 panel kernels with W
// as a one-column problem, plus an identity row that becomes L_kk^-T), scatter
// it back (off-band tiles rounded to FP32), split its rows for the FP16
// tensor-core update, then update the band targets with FP64 DMMA and the
// off-band targets with the split tcgen05 kernel.  After the factorisation:
// log-det from the FP64 diagonal tiles, v = (L L^T)^-1 z, one refinement step
// with the FP64 residual z - C v, and the assembly with z^T (v + w).
int enqueue_eval_mixed(egs_problem* p) {
  if (p->band_method == EGS_BAND_OZAKI_INT8) return enqueue_eval_mixed_ozaki(p);
  cudaStream_t st = p->stream;
  const int ts = p->ts, nt = p->nt, n = p->n, b = p->mband;
  int* info = p->flags;
  int* err = p->flags + 1;
  if (int rc = enqueue_mixed_head(p)) return rc;
  for (int k = 0; k < nt; ++k) {
    const int ntp = nt - k;
    int sp = span_begin(p, EGS_STAGE_PANEL);
    long long nl = 0;
    launch_gather_column(p->band_pool, p->off_pool, p->W, ts, nt, b, k, st);
    ++nl;
    // W holds tile column k and an identity tile as a one-column problem of
    // ntp + 1 tiles; the solve of the identity row gives L_kk^-T
    if (int rc = enqueue_panel(p->W, p->tmapW, ts, ntp + 1, 0, k * ts, info, err, st, &nl)) return rc;
    launch_scatter_column(p->W, p->band_pool, p->off_pool, p->inv_pool, ts, nt, b, k, st);
    ++nl;
    if (ntp > 1) {
      launch_panel_split(p->W, ts, 1, ntp - 1, k, p->inv_scale, p->ph, p->pl, st);
      nl += 2;
    }
    count_launches(p, EGS_STAGE_PANEL, nl);
    span_end(p, sp, panel_flops(ts, n, k));
    if (ntp <= 1) continue;
    sp = span_begin(p, EGS_STAGE_UPDATE);
    const egs_problem::JobLaunch& L = p->band_launch[k];
    if (L.njobs > 0 && L.total > 0) {
      int rc = launch_gemm_batched(p->tmapW, p->band_pool, p->band_jobs + L.job_off, p->band_begin + L.begin_off,
                                   L.njobs, L.total, err, st);
      if (rc != EGS_OK) return rc;
      count_launches(p, EGS_STAGE_UPDATE, 1);
    }
    span_end(p, sp, band_update_flops(ts, nt, b, k));
    if (int rc = enqueue_offband_update(p, k, st, 0)) return rc;
  }
  return enqueue_mixed_tail(p);
}

// Re-lays a problem out for mixed precision: device tile rounded up to a
// multiple of 256 (the FP16 update's tile), FP64 band of b tile rows, FP32
// off-band tiles, workspaces, the generator's tile table and the band update's
// job tables.
int setup_mixed(egs_problem* p, int b) {
  free_mixed(p);
  for (void* buf : {(void*)p->tiles, (void*)p->x, (void*)p->y, (void*)p->z, (void*)p->zcpy, (void*)p->partial})
    dev_free(buf, p->stream);
  p->tiles = p->x = p->y = p->z = p->zcpy = p->partial = nullptr;
  p->bytes = (long long)(sizeof(MaternParams) + kKtabDoubles * sizeof(double) + 2 * sizeof(int) + 4 * sizeof(double));
  const int ts = ((std::max(p->dts, 256) + 255) / 256) * 256;
  p->ts = ts;
  p->nt = (p->n + ts - 1) / ts;
  p->np = p->nt * ts;
  p->ntiles = 0;
  p->mband = b;
  const int nt = p->nt;
  const int m = std::max(0, nt - b - 1);
  const size_t ts2 = (size_t)ts * ts;
  int rc = EGS_OK;
  if ((rc = dev_alloc(&p->x, p->np, &p->bytes, p->stream)) || (rc = dev_alloc(&p->y, p->np, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->z, p->np, &p->bytes, p->stream)) || (rc = dev_alloc(&p->zcpy, p->np, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->partial, p->nt, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->band_pool, (size_t)nt * (b + 1) * ts2, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->off_pool, std::max<size_t>(1, (size_t)lower_tiles(m) * ts2), &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->W, (size_t)(nt + 1) * ts2, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->inv_pool, (size_t)nt * ts2, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->solve_tmp, ts, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->ph, (size_t)p->np * ts, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->pl, (size_t)p->np * ts, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->inv_scale, (size_t)p->np, &p->bytes, p->stream)) || (rc = dev_alloc(&p->w, p->np, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->res_scratch, (size_t)residual_scratch_doubles(p->n), &p->bytes, p->stream)))
    return rc;
  std::vector<int4> gen;
  for (int j = 0; j < nt; ++j)
    for (int i = j; i < nt; ++i)
      gen.push_back(i - j <= b ? make_int4(i, j, 0, (int)((long long)j * (b + 1) + (i - j)))
                               : make_int4(i, j, 1, (int)tile_slot(i - b - 1, j, m)));
  p->ngen = (long long)gen.size();
  if ((rc = dev_alloc(&p->gen_tiles, gen.size(), &p->bytes, p->stream))) return rc;
  EGS_CUDA_TRY(cudaMemcpy(p->gen_tiles, gen.data(), gen.size() * sizeof(int4), cudaMemcpyHostToDevice));
  // FP64 band update of step k: one job per target tile column j > k, rows of
  // tiles j .. min(nt-1, j+b), all operands W-relative (W[t] = tile (k+t, k)).
  std::vector<GemmDesc> jobs;
  std::vector<long long> begin;
  p->band_launch.clear();
  for (int k = 0; k < nt; ++k) {
    egs_problem::JobLaunch L{(long long)jobs.size(), (long long)begin.size(), 0, 0};
    long long acc = 0;
    for (int j = k + 1; j < nt; ++j) {
      const int t = j - k;
      GemmDesc d{};
      d.M = (std::min(nt - 1, j + b) - j + 1) * ts;
      d.N = ts;
      d.K = ts;
      d.a_row0 = d.b_row0 = d.c_row0 = d.c_col0 = t * ts;
      d.lower = 1;
      d.ts = ts;
      d.nt = nt - k;
      d.np = (nt - k) * ts;
      d.c_mode = 1;
      d.c_band = b;
      d.c_tile_off = k;
      finish_desc(d);
      jobs.push_back(d);
      begin.push_back(acc);
      acc += d.total;
      ++L.njobs;
    }
    begin.push_back(acc);
    L.total = acc;
    p->band_launch.push_back(L);
  }
  if ((rc = dev_alloc(&p->band_jobs, std::max<size_t>(1, jobs.size()), &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->band_begin, std::max<size_t>(1, begin.size()), &p->bytes, p->stream)))
    return rc;
  if (!jobs.empty())
    EGS_CUDA_TRY(cudaMemcpy(p->band_jobs, jobs.data(), jobs.size() * sizeof(GemmDesc), cudaMemcpyHostToDevice));
  EGS_CUDA_TRY(cudaMemcpy(p->band_begin, begin.data(), begin.size() * sizeof(long long), cudaMemcpyHostToDevice));
  // Ozaki band update: slices of every panel row, per-step target tables
  {
    std::vector<int4> targets;
    p->oz_launch.clear();
    for (int k = 0; k < nt; ++k) {
      const long long off = (long long)targets.size();
      const long long items = ozaki_targets(ts, nt, b, k, targets);
      p->oz_launch.push_back({off, (int)((long long)targets.size() - off), items});
    }
    // panel solve of the off-band rows through L_kk^-1: tiles k+b+1 .. nt-1
    std::vector<int4> tt;
    p->oz_trsm_launch.clear();
    for (int k = 0; k < nt; ++k) {
      const long long off = (long long)tt.size();
      const long long items = ozaki_trsm_targets(ts, nt, k + b + 1, tt);
      p->oz_trsm_launch.push_back({off, (int)((long long)tt.size() - off), items});
    }
    // slice rows: every panel row, then ts rows for L_kk^-1
    const long long srows = (long long)p->np + ts;
    if ((rc = dev_alloc(&p->oz_slices, (size_t)srows * ts * ozaki_slices(), &p->bytes, p->stream)) ||
        (rc = dev_alloc(&p->oz_scale, (size_t)srows, &p->bytes, p->stream)) ||
        (rc = dev_alloc(&p->oz_targets, std::max<size_t>(1, targets.size()), &p->bytes, p->stream)) ||
        (rc = dev_alloc(&p->oz_trsm_targets, std::max<size_t>(1, tt.size()), &p->bytes, p->stream)) ||
        (rc = dev_alloc(&p->W2, (size_t)(b + 2) * ts2, &p->bytes, p->stream)))
      return rc;
    if (!targets.empty())
      EGS_CUDA_TRY(cudaMemcpyAsync(p->oz_targets, targets.data(), targets.size() * sizeof(int4),
                                   cudaMemcpyHostToDevice, p->stream));
    if (!tt.empty())
      EGS_CUDA_TRY(cudaMemcpyAsync(p->oz_trsm_targets, tt.data(), tt.size() * sizeof(int4), cudaMemcpyHostToDevice,
                                   p->stream));
    EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
    if ((rc = ozaki_tensor_map(p->tm_oz, p->oz_slices, ts, srows)) != EGS_OK) return rc;
    if ((rc = gemm_init_tensor_map(p->tmapW2, p->W2, ts, b + 2)) != EGS_OK) return rc;
    EGS_CUDA_TRY(cudaMemsetAsync(p->oz_scale, 0, srows * sizeof(double), p->stream));
    if (cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_band, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_panel, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      set_last_error("stream or event creation failed", "egs_problem_set_precision");
      return EGS_ERR_CUDA;
    }
  }
  if ((rc = gemm_init_tensor_map(p->tmapW, p->W, ts, nt + 1)) != EGS_OK ||
      (rc = split_tensor_map(p->tm_hi, p->ph, ts, p->np)) != EGS_OK ||
      (rc = split_tensor_map(p->tm_lo, p->pl, ts, p->np)) != EGS_OK ||
      (rc = split_c_map(p->tm_c, p->off_pool, ts, lower_tiles(m))) != EGS_OK)
    return rc;
  EGS_CUDA_TRY(cudaMemset(p->x, 0, p->np * sizeof(double)));
  EGS_CUDA_TRY(cudaMemset(p->y, 0, p->np * sizeof(double)));
  EGS_CUDA_TRY(cudaMemset(p->z, 0, p->np * sizeof(double)));
  EGS_CUDA_TRY(cudaMemset(p->zcpy, 0, p->np * sizeof(double)));
  EGS_CUDA_TRY(cudaMemset(p->w, 0, p->np * sizeof(double)));
  EGS_CUDA_TRY(cudaMemset(p->inv_scale, 0, p->np * sizeof(float)));
  EGS_CUDA_TRY(cudaMemset(p->ph, 0, (size_t)p->np * ts * sizeof(__half)));
  EGS_CUDA_TRY(cudaMemset(p->pl, 0, (size_t)p->np * ts * sizeof(__half)));
  p->precision = EGS_PRECISION_MIXED;
  return EGS_OK;
}

int reject_mixed(const egs_problem* p, const char* where) {
  if (p->precision == EGS_PRECISION_DOUBLE) return EGS_OK;
  if (p->precision == kPrecisionBroken) {
    set_last_error("the problem's mixed-precision layout could not be built", where);
    return EGS_ERR_STATE;
  }
  set_last_error("not available for a mixed-precision problem (use egs_mle_eval)", where);
  return EGS_ERR_STATE;
}

// Capture the parameter upload and enqueue_eval into a graph: the plain one,
// or with prof the one that also records the per-stage timing events.  Capture
// problems (an unsupported call inside the stream) disable that kind of replay
// for this problem.
int capture_eval(egs_problem* p, bool prof) {
  cudaGraph_t& graph = prof ? p->pgraph : p->graph;
  cudaGraphExec_t& exec = prof ? p->pgraph_exec : p->graph_exec;
  long long* launches = prof ? p->pgraph_launches : p->graph_launches;
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
  auto disable = [&]() {
    if (prof) {
      p->pgraphs_ok = false;
    } else {
      p->graphs_enabled = false;
    }
  };
  long long before[EGS_NUM_STAGES];
  for (int i = 0; i < EGS_NUM_STAGES; ++i) before[i] = p->stage_launches[i];
  const size_t span0 = p->spans.size();
  cudaStream_t st = p->stream;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    disable();
    return EGS_OK;
  }
  cudaMemcpyAsync(p->dparams, p->hparams, sizeof(MaternParams), cudaMemcpyHostToDevice, st);
  const int rc = enqueue_eval(p);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  for (int i = 0; i < EGS_NUM_STAGES; ++i) {
    launches[i] = p->stage_launches[i] - before[i];
    p->stage_launches[i] = before[i];
  }
  // the captured spans ran nothing yet: keep them for the replays
  if (prof) p->pgraph_spans.assign(p->spans.begin() + span0, p->spans.end());
  p->spans.resize(span0);
  if (rc != EGS_OK || e != cudaSuccess || !g || cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    exec = nullptr;
    if (prof) p->pgraph_spans.clear();
    disable();
    return EGS_OK;
  }
  graph = g;
  (prof ? p->pgraph_band : p->graph_band) = p->band;
  return EGS_OK;
}

}  // namespace

extern "C" {

int egs_version(void) { return 100; }

const char* egs_status_string(int status) {
  switch (status) {
    case EGS_OK: return "ok";
    case EGS_ERR_INVALID: return "invalid argument";
    case EGS_ERR_CUDA: return "CUDA error";
    case EGS_ERR_NO_DEVICE: return "no CUDA device";
    case EGS_ERR_OOM: return "device allocation refused";
    case EGS_ERR_TIMEOUT: return "device wait timed out";
    case EGS_ERR_STATE: return "invalid call order";
    default: return status > 0 ? "matrix is not positive definite" : "unknown status";
  }
}

const char* egs_last_error(void) { return g_last_error.c_str(); }

int egs_hardware_init(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set_last_error("no CUDA device visible", "egs_hardware_init");
    return EGS_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return EGS_ERR_INVALID;
  EGS_CUDA_TRY(cudaSetDevice(device));
  EGS_CUDA_TRY(cudaFree(nullptr));
  return EGS_OK;
}

static int create_problem(egs_problem** out, int n, int dts, bool with_tiles) {
  if (!out || n <= 0 || dts <= 0) return EGS_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
    cudaGetLastError();
    set_last_error("no CUDA device visible", "egs_problem_create");
    return EGS_ERR_NO_DEVICE;
  }
  auto* p = new egs_problem();
  p->n = n;
  p->dts = dts;
  p->ts = round_tile(dts);
  p->nt = (n + p->ts - 1) / p->ts;
  p->np = p->nt * p->ts;
  p->ntiles = lower_tiles(p->nt);
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    set_last_error("stream creation failed", "egs_problem_create");
    delete p;
    return EGS_ERR_CUDA;
  }
  p->own_stream = true;
  int rc = EGS_OK;
  if ((with_tiles && (rc = dev_alloc(&p->tiles, (size_t)p->ntiles * p->ts * p->ts, &p->bytes, p->stream))) ||
      (rc = dev_alloc(&p->x, p->np, &p->bytes, p->stream)) || (rc = dev_alloc(&p->y, p->np, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->z, p->np, &p->bytes, p->stream)) || (rc = dev_alloc(&p->zcpy, p->np, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->partial, p->nt, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->result, 4, &p->bytes, p->stream)) || (rc = dev_alloc(&p->flags, 2, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->dparams, 1, &p->bytes, p->stream)) ||
      (rc = dev_alloc(&p->ktab, kKtabDoubles, &p->bytes, p->stream))) {
    free_problem(p);
    return rc;
  }
  p->hparams = static_cast<MaternParams*>(pinned_record());
  p->hresult = static_cast<double*>(pinned_record());
  p->hflags = static_cast<int*>(pinned_record());
  if (!p->hparams || !p->hresult || !p->hflags) {
    set_last_error("pinned host allocation failed", "egs_problem_create");
    free_problem(p);
    return EGS_ERR_CUDA;
  }
  if (with_tiles && (rc = gemm_init_tensor_map(p->tmap, p->tiles, p->ts, p->ntiles)) != EGS_OK) {
    free_problem(p);
    return rc;
  }
  // Padding rows: zero locations and observations (the generator writes the identity there).
  if (cudaMemsetAsync(p->x, 0, p->np * sizeof(double), p->stream) != cudaSuccess ||
      cudaMemsetAsync(p->y, 0, p->np * sizeof(double), p->stream) != cudaSuccess ||
      cudaMemsetAsync(p->zcpy, 0, p->np * sizeof(double), p->stream) != cudaSuccess ||
      cudaMemsetAsync(p->z, 0, p->np * sizeof(double), p->stream) != cudaSuccess ||
      cudaStreamSynchronize(p->stream) != cudaSuccess) {
    cudaGetLastError();
    free_problem(p);
    return EGS_ERR_CUDA;
  }
  *out = p;
  return EGS_OK;
}

int egs_problem_create(egs_problem** out, int n, int dts) { return create_problem(out, n, dts, true); }

int egs_problem_create_ex(egs_problem** out, int n, int dts, int precision, int band_tiles) {
  if (!out) return EGS_ERR_INVALID;
  *out = nullptr;
  if (precision == EGS_PRECISION_DOUBLE) return create_problem(out, n, dts, true);
  if (precision != EGS_PRECISION_MIXED || band_tiles < 0) return EGS_ERR_INVALID;
  egs_problem* p = nullptr;
  int rc = create_problem(&p, n, dts, false);  // the mixed layout replaces the FP64 tile storage
  if (rc != EGS_OK) return rc;
  if ((rc = egs_problem_set_precision(p, precision, band_tiles)) != EGS_OK) {
    free_problem(p);
    return rc;
  }
  *out = p;
  return EGS_OK;
}

int egs_problem_destroy(egs_problem* p) {
  free_problem(p);
  return EGS_OK;
}

int egs_problem_info(const egs_problem* p, int* n, int* ts, int* nt, long long* bytes) {
  if (!p) return EGS_ERR_INVALID;
  if (n) *n = p->n;
  if (ts) *ts = p->ts;
  if (nt) *nt = p->nt;
  if (bytes) *bytes = p->bytes;
  return EGS_OK;
}

int egs_problem_set_band(egs_problem* p, int band) {
  if (!p || band < 0) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_problem_set_band")) return rc;
  // Caller tiles that are not device tiles keep their own size in the band
  // factorisation (launch_dst_band), since merging them into a larger device
  // tile would change which elements the approximation keeps.
  p->band = band;
  return EGS_OK;
}

int egs_problem_set_precision(egs_problem* p, int precision, int band_tiles) {
  if (!p || band_tiles < 0) return EGS_ERR_INVALID;
  if (precision != EGS_PRECISION_DOUBLE && precision != EGS_PRECISION_MIXED) return EGS_ERR_INVALID;
  if (precision == p->precision && (precision == EGS_PRECISION_DOUBLE || band_tiles == p->mband)) return EGS_OK;
  if (p->have_locations || p->have_observations) {
    set_last_error("set the precision before locations and observations", "egs_problem_set_precision");
    return EGS_ERR_STATE;
  }
  if (precision == EGS_PRECISION_DOUBLE) {
    set_last_error("a mixed-precision problem cannot return to FP64; create a new problem",
                   "egs_problem_set_precision");
    return EGS_ERR_STATE;
  }
  if (p->band > 0) {
    set_last_error("the band approximation and mixed precision are exclusive", "egs_problem_set_precision");
    return EGS_ERR_STATE;
  }
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  drop_graphs(p);
  const int rc = setup_mixed(p, band_tiles);
  if (rc != EGS_OK) {
    // leave a problem that reports the failure instead of a half-built layout
    free_mixed(p);
    p->precision = kPrecisionBroken;
  }
  return rc;
}

int egs_problem_set_lookahead(egs_problem* p, int sms) {
  if (!p || sms < 0 || sms >= gemm_num_sms()) return EGS_ERR_INVALID;
  if (sms == p->lookahead_sms) return EGS_OK;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  drop_graphs(p);
  p->lookahead_sms = sms;
  return EGS_OK;
}

int egs_problem_set_band_method(egs_problem* p, int method) {
  if (!p || (method != EGS_BAND_OZAKI_INT8 && method != EGS_BAND_FP64_DMMA)) return EGS_ERR_INVALID;
  if (p->precision != EGS_PRECISION_MIXED) {
    set_last_error("only a mixed-precision problem has a band method", "egs_problem_set_band_method");
    return EGS_ERR_STATE;
  }
  if (method == p->band_method) return EGS_OK;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  drop_graphs(p);
  p->band_method = method;
  return EGS_OK;
}

int egs_problem_set_stream(egs_problem* p, void* cuda_stream) {
  if (!p) return EGS_ERR_INVALID;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (p->own_stream) cudaStreamDestroy(p->stream);
  if (cuda_stream) {
    p->stream = (cudaStream_t)cuda_stream;
    p->own_stream = false;
  } else {
    EGS_CUDA_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    p->own_stream = true;
  }
  return EGS_OK;
}

namespace {

uint64_t spread16(uint64_t v) {
  v &= 0xffffull;
  v = (v ^ (v << 24)) & 0x000000ff000000ffull;
  v = (v ^ (v << 12)) & 0x000f000f000f000full;
  v = (v ^ (v << 6)) & 0x0303030303030303ull;
  v = (v ^ (v << 3)) & 0x1111111111111111ull;
  return v;
}

// Locality order of n points for the mixed form: the FP64 band of the mixed
// factorisation holds the tiles next to the diagonal, which carry the large
// covariances only when nearby points are adjacent in the matrix.  Points are
// ordered by their Morton (Z-order) code at 16 bits per axis -- the key of the
// reference's SortLocations (LocationGenerator.cpp:91-123) -- on the unit
// square when every coordinate lies in [0, 1], else on the bounding box; ties
// keep the caller's order.  Returns an empty vector when the caller's order is
// already sorted (the reference generator's output is), so such problems run
// on exactly the caller's layout.
std::vector<int> locality_order(int n, const double* x, const double* y) {
  double x0 = x[0], x1 = x[0], y0 = y[0], y1 = y[0];
  for (int i = 1; i < n; ++i) {
    x0 = std::min(x0, x[i]);
    x1 = std::max(x1, x[i]);
    y0 = std::min(y0, y[i]);
    y1 = std::max(y1, y[i]);
  }
  const bool unit = x0 >= 0.0 && y0 >= 0.0 && x1 <= 1.0 && y1 <= 1.0;
  const double ox = unit ? 0.0 : x0, oy = unit ? 0.0 : y0;
  const double sx = unit ? 1.0 : (x1 > x0 ? x1 - x0 : 1.0), sy = unit ? 1.0 : (y1 > y0 ? y1 - y0 : 1.0);
  std::vector<uint64_t> key(n);
  bool sorted = true;
  for (int i = 0; i < n; ++i) {
    const uint16_t qx = (uint16_t)((x[i] - ox) / sx * 65535.0 + 0.5);
    const uint16_t qy = (uint16_t)((y[i] - oy) / sy * 65535.0 + 0.5);
    key[i] = (spread16(qy) << 1) + spread16(qx);
    if (i > 0 && key[i] < key[i - 1]) sorted = false;
  }
  if (sorted) return {};
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return key[a] < key[b]; });
  return perm;
}

// Caller-order host vector -> device order.
std::vector<double> to_device_order(const egs_problem* p, const double* v) {
  std::vector<double> out(p->n);
  for (int d = 0; d < p->n; ++d) out[d] = v[p->perm[d]];
  return out;
}

// A caller's vector of n doubles in host memory (copied from the device when
// kind says it lives there).
int host_copy(const egs_problem* p, const double* v, cudaMemcpyKind kind, std::vector<double>* out) {
  out->resize(p->n);
  if (kind == cudaMemcpyHostToDevice) {
    std::copy(v, v + p->n, out->begin());
    return EGS_OK;
  }
  EGS_CUDA_TRY(cudaMemcpyAsync(out->data(), v, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

}  // namespace

static int set_locs(egs_problem* p, const double* x, const double* y, cudaMemcpyKind kind) {
  if (!p || !x || !y) return EGS_ERR_INVALID;
  if (p->precision == kPrecisionBroken) return EGS_ERR_STATE;
  if (p->precision == EGS_PRECISION_MIXED) {
    std::vector<double> hx, hy, hz;
    const double *hxp = x, *hyp = y;
    if (kind != cudaMemcpyHostToDevice) {
      int rc;
      if ((rc = host_copy(p, x, kind, &hx)) != EGS_OK || (rc = host_copy(p, y, kind, &hy)) != EGS_OK) return rc;
      hxp = hx.data();
      hyp = hy.data();
    }
    if (p->have_observations) {
      // observations already uploaded in the previous order: back to the caller's
      std::vector<double> dz(p->n);
      EGS_CUDA_TRY(cudaMemcpyAsync(dz.data(), p->zcpy, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
      EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
      hz.resize(p->n);
      for (int d = 0; d < p->n; ++d) hz[p->perm.empty() ? d : p->perm[d]] = dz[d];
    }
    p->perm = locality_order(p->n, hxp, hyp);
    if (!p->perm.empty()) {
      hx = to_device_order(p, hxp);
      hy = to_device_order(p, hyp);
      hxp = hx.data();
      hyp = hy.data();
    }
    EGS_CUDA_TRY(cudaMemcpyAsync(p->x, hxp, p->n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    EGS_CUDA_TRY(cudaMemcpyAsync(p->y, hyp, p->n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    if (p->have_observations) {
      if (!p->perm.empty()) hz = to_device_order(p, hz.data());
      EGS_CUDA_TRY(cudaMemcpyAsync(p->zcpy, hz.data(), p->n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
      EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
    }
    EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
    p->have_locations = true;
    return EGS_OK;
  }
  EGS_CUDA_TRY(cudaMemcpyAsync(p->x, x, p->n * sizeof(double), kind, p->stream));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->y, y, p->n * sizeof(double), kind, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  p->have_locations = true;
  return EGS_OK;
}

int egs_problem_set_locations(egs_problem* p, const double* x, const double* y) {
  return set_locs(p, x, y, cudaMemcpyHostToDevice);
}
int egs_problem_set_locations_device(egs_problem* p, const double* x, const double* y) {
  return set_locs(p, x, y, cudaMemcpyDeviceToDevice);
}

static int set_obs(egs_problem* p, const double* z, cudaMemcpyKind kind) {
  if (!p || !z) return EGS_ERR_INVALID;
  if (p->precision == kPrecisionBroken) return EGS_ERR_STATE;
  if (!p->perm.empty()) {
    // a mixed problem holding its points in locality order
    std::vector<double> hz;
    int rc = host_copy(p, z, kind, &hz);
    if (rc != EGS_OK) return rc;
    hz = to_device_order(p, hz.data());
    EGS_CUDA_TRY(cudaMemcpyAsync(p->zcpy, hz.data(), p->n * sizeof(double), cudaMemcpyHostToDevice, p->stream));
    EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
    EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
    p->have_observations = true;
    return EGS_OK;
  }
  EGS_CUDA_TRY(cudaMemcpyAsync(p->zcpy, z, p->n * sizeof(double), kind, p->stream));
  EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  p->have_observations = true;
  return EGS_OK;
}

int egs_problem_set_observations(egs_problem* p, const double* z) { return set_obs(p, z, cudaMemcpyHostToDevice); }
int egs_problem_set_observations_device(egs_problem* p, const double* z) {
  return set_obs(p, z, cudaMemcpyDeviceToDevice);
}

int egs_covariance_generate(egs_problem* p, const double* theta) {
  if (!p) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_covariance_generate")) return rc;
  if (!p->have_locations) return EGS_ERR_STATE;
  int rc = set_params(p, theta);
  if (rc != EGS_OK) return rc;
  rc = launch_matern_tiles(p->tiles, p->x, p->y, p->n, p->ts, p->nt, p->dparams, p->ktab, p->stream);
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_potrf(egs_problem* p) {
  if (!p) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_potrf")) return rc;
  EGS_CUDA_TRY(cudaMemsetAsync(p->flags, 0, 2 * sizeof(int), p->stream));
  int rc = p->band > 0 ? enqueue_potrf_band(p) : enqueue_potrf(p);
  if (rc != EGS_OK) return rc;
  return sync_flags(p, false);
}

int egs_restore_observations(egs_problem* p) {
  if (!p) return EGS_ERR_INVALID;
  if (!p->have_observations) return EGS_ERR_STATE;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_trsv(egs_problem* p) {
  if (!p) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_trsv")) return rc;
  enqueue_trsv(p);
  int rc = check_cuda("egs_trsv");
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_loglik_parts(egs_problem* p, double* loglik, double* logdet, double* dot) {
  if (!p) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_loglik_parts")) return rc;
  launch_logdet_partials(p->tiles, p->ts, p->nt, p->n, p->partial, p->stream);
  launch_finalize(p->partial, p->nt, p->z, p->n, p->result, nullptr, p->stream);
  int rc = check_cuda("egs_loglik_parts");
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hresult, p->result, 4 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (loglik) *loglik = p->hresult[0];
  if (logdet) *logdet = p->hresult[1];
  if (dot) *dot = p->hresult[2];
  return EGS_OK;
}

int egs_get_tile(egs_problem* p, int i, int j, double* host_out) {
  if (!p || !host_out || i < j || i >= p->nt || j < 0) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_get_tile")) return rc;
  const size_t ts2 = (size_t)p->ts * p->ts;
  EGS_CUDA_TRY(cudaMemcpyAsync(host_out, p->tiles + tile_slot(i, j, p->nt) * ts2, ts2 * sizeof(double),
                               cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_get_observations(egs_problem* p, double* host_z) {
  if (!p || !host_z) return EGS_ERR_INVALID;
  if (!p->perm.empty()) {
    std::vector<double> dz(p->n);
    EGS_CUDA_TRY(cudaMemcpyAsync(dz.data(), p->z, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
    for (int d = 0; d < p->n; ++d) host_z[p->perm[d]] = dz[d];
    return EGS_OK;
  }
  EGS_CUDA_TRY(cudaMemcpyAsync(host_z, p->z, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_save_observations(egs_problem* p) {
  if (!p) return EGS_ERR_INVALID;
  if (!p->have_observations) return EGS_ERR_STATE;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->zcpy, p->z, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_trsv_transpose(egs_problem* p) {
  if (!p) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_trsv_transpose")) return rc;
  enqueue_trsv_t(p);
  int rc = check_cuda("egs_trsv_transpose");
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_set_tile(egs_problem* p, int i, int j, const double* host_in) {
  if (!p || !host_in || i < j || i >= p->nt || j < 0) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_set_tile")) return rc;
  const size_t ts2 = (size_t)p->ts * p->ts;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->tiles + tile_slot(i, j, p->nt) * ts2, host_in, ts2 * sizeof(double),
                               cudaMemcpyHostToDevice, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return EGS_OK;
}

int egs_sequence_create(void** sequence) {
  if (!sequence) return EGS_ERR_INVALID;
  cudaStream_t s = nullptr;
  EGS_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *sequence = s;
  return EGS_OK;
}

int egs_sequence_wait(void* sequence) {
  if (!sequence) return EGS_ERR_INVALID;
  EGS_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(sequence)));
  return EGS_OK;
}

int egs_sequence_destroy(void* sequence) {
  if (!sequence) return EGS_OK;
  EGS_CUDA_TRY(cudaStreamDestroy(static_cast<cudaStream_t>(sequence)));
  return EGS_OK;
}

int egs_mle_eval(egs_problem* p, const double* theta, double* loglik, double* logdet, double* dot) {
  if (!p || !loglik) return EGS_ERR_INVALID;
  if (!p->have_locations || !p->have_observations) return EGS_ERR_STATE;
  MaternParams mp;
  int rc = make_matern_params(theta, &mp);
  if (rc != EGS_OK) {
    set_last_error("theta outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "make_matern_params");
    return rc;
  }
  cudaStream_t st = p->stream;
  // The pinned mirrors may still be in use by the previous evaluation.
  EGS_CUDA_TRY(cudaStreamSynchronize(st));
  *p->hparams = mp;
  const bool prof = p->profiling;
  const bool replay = p->graphs_enabled && (!prof || p->pgraphs_ok) && p->evals > 0;
  cudaGraphExec_t& exec = prof ? p->pgraph_exec : p->graph_exec;
  if (replay && (!exec || (prof ? p->pgraph_band : p->graph_band) != p->band)) {
    if ((rc = capture_eval(p, prof)) != EGS_OK) return rc;
  }
  if (replay && exec) {
    EGS_CUDA_TRY(cudaGraphLaunch(exec, st));
    const long long* launches = prof ? p->pgraph_launches : p->graph_launches;
    for (int i = 0; i < EGS_NUM_STAGES; ++i) p->stage_launches[i] += launches[i];
    if (prof) p->spans.insert(p->spans.end(), p->pgraph_spans.begin(), p->pgraph_spans.end());
  } else {
    EGS_CUDA_TRY(cudaMemcpyAsync(p->dparams, p->hparams, sizeof(MaternParams), cudaMemcpyHostToDevice, st));
    if ((rc = enqueue_eval(p)) != EGS_OK) return rc;
  }
  ++p->evals;
  EGS_CUDA_TRY(cudaStreamSynchronize(st));
  const size_t nspans = p->spans.size();
  if (collect_spans(p) == 0 && nspans > 0 && prof && replay) {
    // the replayed timing events gave no times: time the next ones eagerly
    p->pgraphs_ok = false;
  }
  if (p->hflags[1] != 0) {
    set_last_error("a device-side wait exceeded its limit", "tensor-core update");
    return EGS_ERR_TIMEOUT;
  }
  if (p->hflags[0] > 0) {
    set_last_error("Matrix is not positive definite", "potrf");
    return p->hflags[0];
  }
  *loglik = p->hresult[0];
  if (logdet) *logdet = p->hresult[1];
  if (dot) *dot = p->hresult[2];
  return EGS_OK;
}

int egs_problem_set_graphs(egs_problem* p, int enable) {
  if (!p) return EGS_ERR_INVALID;
  p->graphs_enabled = enable != 0;
  return EGS_OK;
}

int egs_generate_observations(egs_problem* p, const double* theta, int seed, double* z_out) {
  if (!p || !theta || seed < 0 || seed > 4095) return EGS_ERR_INVALID;
  if (int rc = reject_mixed(p, "egs_generate_observations")) return rc;
  if (!p->have_locations) return EGS_ERR_STATE;
  if (lower_tiles(p->nt) > 65535) return EGS_ERR_INVALID;
  std::vector<double> e(p->np, 0.0);
  const int iseed[4] = {seed, seed, seed, 1};
  int rc = egs_dlarnv_normal(iseed, p->n, e.data());
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->z, e.data(), p->np * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  if ((rc = egs_covariance_generate(p, theta)) != EGS_OK) return rc;
  if ((rc = egs_potrf(p)) != EGS_OK) return rc;
  double* part = nullptr;
  long long dummy = 0;
  if ((rc = dev_alloc(&part, (size_t)p->ntiles * p->ts, &dummy, p->stream)) != EGS_OK) return rc;
  launch_trmv(p->tiles, p->ts, p->nt, p->z, part, p->zcpy, p->stream);
  cudaMemcpyAsync(p->z, p->zcpy, p->np * sizeof(double), cudaMemcpyDeviceToDevice, p->stream);
  if (z_out) cudaMemcpyAsync(z_out, p->zcpy, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->stream);
  rc = check_cuda("egs_generate_observations");
  dev_free(part, p->stream);
  cudaStreamSynchronize(p->stream);
  if (rc != EGS_OK) return rc;
  p->have_observations = true;
  return EGS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Evaluation without allocation.
//
// Some callers cannot call cudaMalloc: a host application whose device memory
// is owned by another allocator (a framework's caching allocator, or a pool
// sized once at start-up), where an extra cudaMalloc would go around that
// budget, and latency-bound loops such as an optimizer driving thousands of
// evaluations, where cudaMalloc / cudaFree would add device-wide
// synchronisation to every call.  egs_mle_eval_noalloc takes every large buffer
// from the caller and keeps the small per-call state (log-determinant partial
// sums, the result record, the status flags and the Matern parameters) in the
// file-scope device array below, which every GPU that loads this library holds
// until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxTileRows = 4096;  // n <= 4096 * device tile size
constexpr size_t kNoAllocPartialOff = 0;
constexpr size_t kNoAllocResultOff = kNoAllocPartialOff + kNoAllocMaxTileRows * sizeof(double);
constexpr size_t kNoAllocFlagsOff = kNoAllocResultOff + 4 * sizeof(double);
constexpr size_t kNoAllocParamsOff = kNoAllocFlagsOff + 256;
constexpr size_t kNoAllocKtabOff = kNoAllocParamsOff + 256;
constexpr size_t kNoAllocScratchBytes = kNoAllocKtabOff + kKtabDoubles * sizeof(double);
constexpr int kNoAllocMaxDevices = 64;
static_assert(sizeof(MaternParams) <= 256, "parameter slot of the static scratch");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once per
// device (the host-side symbol is only a stand-in and must not reach a kernel).
int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  EGS_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_last_error("device ordinal beyond the supported range", "egs_mle_eval_noalloc");
    return EGS_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      set_last_error(cudaGetErrorString(e), "cudaGetSymbolAddress(g_noalloc_scratch)");
      return EGS_ERR_CUDA;
    }
    g_noalloc_addr[dev] = static_cast<unsigned char*>(ptr);
  }
  *out = g_noalloc_addr[dev];
  return EGS_OK;
}

}  // namespace

extern "C" {

int egs_mle_noalloc_workspace(int n, int dts, long long* doubles) {
  if (n <= 0 || dts <= 0 || !doubles) return EGS_ERR_INVALID;
  const int ts = round_tile(dts);
  const int nt = (n + ts - 1) / ts;
  if (nt > kNoAllocMaxTileRows) {
    set_last_error("n exceeds 4096 device tiles, the limit of the allocation-free evaluation",
                   "egs_mle_noalloc_workspace");
    return EGS_ERR_INVALID;
  }
  const long long np = (long long)nt * ts;
  *doubles = lower_tiles(nt) * (long long)ts * ts + 3 * np;
  return EGS_OK;
}

int egs_mle_eval_noalloc(int n, int dts, const double* x, const double* y, const double* z, const double* theta,
                         double* work, long long work_doubles, double* loglik, void* cuda_stream) {
  if (n <= 0 || dts <= 0 || !x || !y || !z || !theta || !work || !loglik) return EGS_ERR_INVALID;
  long long need = 0;
  int rc = egs_mle_noalloc_workspace(n, dts, &need);
  if (rc != EGS_OK) return rc;
  if (work_doubles < need) {
    set_last_error("workspace smaller than egs_mle_noalloc_workspace requires", "egs_mle_eval_noalloc");
    return EGS_ERR_INVALID;
  }
  if (((uintptr_t)work & 15) != 0) {
    set_last_error("workspace must be 16-byte aligned", "egs_mle_eval_noalloc");
    return EGS_ERR_INVALID;
  }
  MaternParams mp;
  if ((rc = make_matern_params(theta, &mp)) != EGS_OK) {
    set_last_error("theta outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "egs_mle_eval_noalloc");
    return rc;
  }
  unsigned char* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch)) != EGS_OK) return rc;
  double* partial = reinterpret_cast<double*>(scratch + kNoAllocPartialOff);
  double* result = reinterpret_cast<double*>(scratch + kNoAllocResultOff);
  int* flags = reinterpret_cast<int*>(scratch + kNoAllocFlagsOff);
  MaternParams* dparams = reinterpret_cast<MaternParams*>(scratch + kNoAllocParamsOff);
  double* ktab = reinterpret_cast<double*>(scratch + kNoAllocKtabOff);

  // A problem record on the stack that points at the caller's workspace and the
  // static scratch; it owns nothing.
  egs_problem q;
  q.n = n;
  q.dts = dts;
  q.ts = round_tile(dts);
  q.nt = (n + q.ts - 1) / q.ts;
  q.np = q.nt * q.ts;
  q.ntiles = lower_tiles(q.nt);
  q.tiles = work;
  q.x = work + q.ntiles * (long long)q.ts * q.ts;
  q.y = q.x + q.np;
  q.z = q.y + q.np;
  q.partial = partial;
  q.result = result;
  q.flags = flags;
  q.dparams = dparams;
  q.ktab = ktab;
  q.stream = (cudaStream_t)cuda_stream;
  q.own_stream = false;
  if ((rc = gemm_init_tensor_map(q.tmap, q.tiles, q.ts, q.ntiles)) != EGS_OK) return rc;

  cudaStream_t st = q.stream;
  const size_t pad = (size_t)(q.np - n) * sizeof(double);
  EGS_CUDA_TRY(cudaMemcpyAsync(dparams, &mp, sizeof(MaternParams), cudaMemcpyHostToDevice, st));
  EGS_CUDA_TRY(cudaMemsetAsync(flags, 0, 2 * sizeof(int), st));
  EGS_CUDA_TRY(cudaMemcpyAsync(q.x, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  EGS_CUDA_TRY(cudaMemcpyAsync(q.y, y, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  EGS_CUDA_TRY(cudaMemcpyAsync(q.z, z, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (pad) {
    EGS_CUDA_TRY(cudaMemsetAsync(q.x + n, 0, pad, st));
    EGS_CUDA_TRY(cudaMemsetAsync(q.y + n, 0, pad, st));
    EGS_CUDA_TRY(cudaMemsetAsync(q.z + n, 0, pad, st));
  }
  if ((rc = launch_matern_tiles(q.tiles, q.x, q.y, n, q.ts, q.nt, dparams, ktab, st)) != EGS_OK) return rc;
  if ((rc = enqueue_potrf(&q)) != EGS_OK) return rc;
  launch_logdet_partials(q.tiles, q.ts, q.nt, n, partial, st);
  enqueue_trsv(&q);
  launch_finalize(partial, q.nt, q.z, n, result, flags, st);
  if ((rc = check_cuda("egs_mle_eval_noalloc")) != EGS_OK) return rc;
  double hres[4];
  int hflags[2];
  EGS_CUDA_TRY(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, st));
  EGS_CUDA_TRY(cudaMemcpyAsync(hres, result, sizeof(hres), cudaMemcpyDeviceToHost, st));
  EGS_CUDA_TRY(cudaStreamSynchronize(st));
  if (hflags[1] != 0) {
    set_last_error("a device-side wait exceeded its limit", "egs_mle_eval_noalloc");
    return EGS_ERR_TIMEOUT;
  }
  if (hflags[0] > 0) {
    set_last_error("Matrix is not positive definite", "egs_mle_eval_noalloc");
    return hflags[0];
  }
  *loglik = hres[0];
  return EGS_OK;
}

int egs_problem_set_profiling(egs_problem* p, int enable) {
  if (!p) return EGS_ERR_INVALID;
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  collect_spans(p);
  p->profiling = enable != 0;
  for (int i = 0; i < EGS_NUM_STAGES; ++i) {
    p->stage_ms[i] = 0.0;
    p->stage_flops[i] = 0.0;
    p->stage_launches[i] = 0;
  }
  return EGS_OK;
}

int egs_problem_stage_stats(egs_problem* p, double* ms, double* flops, long long* launches) {
  if (!p) return EGS_ERR_INVALID;
  for (int i = 0; i < EGS_NUM_STAGES; ++i) {
    if (ms) ms[i] = p->stage_ms[i];
    if (flops) flops[i] = p->stage_flops[i];
    if (launches) launches[i] = p->stage_launches[i];
  }
  return EGS_OK;
}

int egs_matern_block(double* a, int lda, int rows, int cols, const double* x1, const double* y1, const double* x2,
                     const double* y2, const double* theta, int distance_metric, void* cuda_stream) {
  if (!a || !x1 || !y1 || !x2 || !y2 || !theta || rows < 0 || cols < 0 || lda < rows) return EGS_ERR_INVALID;
  if (distance_metric != 0) {
    set_last_error("only the Euclidean distance (metric 0) is on the device path", "egs_matern_block");
    return EGS_ERR_INVALID;
  }
  MaternParams mp;
  int rc = make_matern_params(theta, &mp);
  if (rc != EGS_OK) return rc;
  return launch_matern_block(a, lda, rows, cols, x1, y1, x2, y2, mp, (cudaStream_t)cuda_stream);
}

namespace {
struct CachedProblem {
  std::unique_ptr<egs_problem, int (*)(egs_problem*)> p{nullptr, egs_problem_destroy};
  int n = 0, dts = 0;
};
thread_local CachedProblem g_cached;
}  // namespace

int egs_mle_loglik_host(int n, int dts, const double* x, const double* y, const double* z, const double* theta,
                        double* loglik) {
  if (n <= 0 || dts <= 0 || !x || !y || !z || !theta || !loglik) return EGS_ERR_INVALID;
  if (!g_cached.p || g_cached.n != n || g_cached.dts != dts) {
    g_cached.p.reset();
    egs_problem* p = nullptr;
    int rc = egs_problem_create(&p, n, dts);
    if (rc != EGS_OK) return rc;
    g_cached.p.reset(p);
    g_cached.n = n;
    g_cached.dts = dts;
  }
  egs_problem* p = g_cached.p.get();
  int rc = egs_problem_set_locations(p, x, y);
  if (rc != EGS_OK) return rc;
  rc = egs_problem_set_observations(p, z);
  if (rc != EGS_OK) return rc;
  return egs_mle_eval(p, theta, loglik, nullptr, nullptr);
}

int egs_predict_host(int n_obs, int n_miss, int dts, const double* x_obs, const double* y_obs, const double* z_obs,
                     const double* x_miss, const double* y_miss, const double* z_actual, const double* theta,
                     double* z_miss, double* mspe) {
  if (n_obs <= 0 || n_miss <= 0 || dts <= 0 || !x_obs || !y_obs || !z_obs || !x_miss || !y_miss || !theta ||
      !z_miss || !mspe)
    return EGS_ERR_INVALID;
  egs_problem* p = nullptr;
  int rc = egs_problem_create(&p, n_obs, dts);
  if (rc != EGS_OK) return rc;
  std::unique_ptr<egs_problem, int (*)(egs_problem*)> guard(p, egs_problem_destroy);
  if ((rc = egs_problem_set_locations(p, x_obs, y_obs)) != EGS_OK) return rc;
  if ((rc = egs_problem_set_observations(p, z_obs)) != EGS_OK) return rc;
  if ((rc = egs_covariance_generate(p, theta)) != EGS_OK) return rc;
  if ((rc = egs_potrf(p)) != EGS_OK) return rc;
  // dposv: w = C22^-1 Zobs (LinearAlgebraMethods.cpp:544)
  enqueue_trsv(p);
  enqueue_trsv_t(p);
  if ((rc = check_cuda("egs_predict_host/posv")) != EGS_OK) return rc;
  // C12^T (obs x miss) and Zmiss = C12 w (:535, :552)
  double *c12t = nullptr, *dxm = nullptr, *dym = nullptr, *dzm = nullptr, *dza = nullptr, *dsum = nullptr;
  long long dummy = 0;
  auto cleanup = [&]() {
    for (void* b : {(void*)c12t, (void*)dxm, (void*)dym, (void*)dzm, (void*)dza, (void*)dsum}) dev_free(b, p->stream);
    cudaStreamSynchronize(p->stream);
  };
  cudaStream_t ps = p->stream;
  if ((rc = dev_alloc(&c12t, (size_t)n_obs * n_miss, &dummy, ps)) || (rc = dev_alloc(&dxm, n_miss, &dummy, ps)) ||
      (rc = dev_alloc(&dym, n_miss, &dummy, ps)) || (rc = dev_alloc(&dzm, n_miss, &dummy, ps)) ||
      (rc = dev_alloc(&dza, n_miss, &dummy, ps)) || (rc = dev_alloc(&dsum, 1, &dummy, ps))) {
    cleanup();
    return rc;
  }
  cudaStream_t st = p->stream;
  if (cudaMemcpyAsync(dxm, x_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dym, y_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    cleanup();
    return EGS_ERR_CUDA;
  }
  MaternParams mp;
  make_matern_params(theta, &mp);
  if ((rc = launch_matern_block(c12t, n_obs, n_obs, n_miss, p->x, p->y, dxm, dym, mp, st)) != EGS_OK) {
    cleanup();
    return rc;
  }
  launch_gemv_t_block(c12t, n_obs, n_obs, n_miss, p->z, dzm, st);
  double sum = -1.0;
  if (z_actual) {
    cudaMemcpyAsync(dza, z_actual, n_miss * sizeof(double), cudaMemcpyHostToDevice, st);
    launch_sumsq_diff(dza, dzm, n_miss, dsum, st);
    cudaMemcpyAsync(&sum, dsum, sizeof(double), cudaMemcpyDeviceToHost, st);
  }
  cudaMemcpyAsync(z_miss, dzm, n_miss * sizeof(double), cudaMemcpyDeviceToHost, st);
  if ((rc = check_cuda("egs_predict_host")) != EGS_OK) {
    cleanup();
    return rc;
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    cleanup();
    return check_cuda("egs_predict_host/sync");
  }
  *mspe = z_actual ? sum / n_miss : -1.0;
  cleanup();
  return EGS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Footprint and prediction on a resident problem (used by the serving loop)
// ---------------------------------------------------------------------------

int egs_problem_footprint(int n, int dts, int precision, int band_tiles, long long* bytes) {
  if (n <= 0 || dts <= 0 || !bytes || band_tiles < 0) return EGS_ERR_INVALID;
  const long long small = (long long)(sizeof(MaternParams) + kKtabDoubles * sizeof(double) + 4 * sizeof(double) +
                                      2 * sizeof(int));
  long long b = 0;
  if (precision == EGS_PRECISION_DOUBLE) {
    const long long ts = round_tile(dts), nt = (n + ts - 1) / ts, np = nt * ts;
    b = lower_tiles((int)nt) * ts * ts * 8 + 4 * np * 8 + nt * 8 + small;
  } else if (precision == EGS_PRECISION_MIXED) {
    const long long ts = ((std::max(dts, 256) + 255) / 256) * 256, nt = (n + ts - 1) / ts, np = nt * ts;
    const long long m = std::max<long long>(0, nt - band_tiles - 1);
    b = 4 * np * 8 + nt * 8 + small;                                // x, y, z, zcpy, partial
    b += nt * (band_tiles + 1) * ts * ts * 8;                       // FP64 band
    b += std::max<long long>(1, lower_tiles((int)m)) * ts * ts * 4; // FP32 off-band
    b += (nt + 1) * ts * ts * 8 + nt * ts * ts * 8 + ts * 8;        // W, inverses, solve temp
    b += 2 * np * ts * 2 + np * 4 + np * 8;                         // FP16 split, row scales, w
    b += residual_scratch_doubles(n) * 8 + lower_tiles((int)nt) * (long long)sizeof(int4);
    b += (nt * nt / 2 + nt + 1) * ((long long)sizeof(GemmDesc) + 8);
  } else {
    return EGS_ERR_INVALID;
  }
  // allocator granularity: every buffer rounds up to 2 MiB in the worst case
  *bytes = b + 32ll * (2ll << 20);
  return EGS_OK;
}

int egs_problem_predict(egs_problem* p, const double* theta, int n_miss, const double* x_miss, const double* y_miss,
                        double* z_miss) {
  if (!p || !theta || n_miss <= 0 || !x_miss || !y_miss || !z_miss) return EGS_ERR_INVALID;
  if (p->precision == kPrecisionBroken) return EGS_ERR_STATE;
  if (!p->have_locations || !p->have_observations) {
    set_last_error("locations and observations must be set", "egs_problem_predict");
    return EGS_ERR_STATE;
  }
  int rc = EGS_OK;
  if (p->precision == EGS_PRECISION_MIXED) {
    // the mixed evaluation leaves (L L^T)^-1 z in z and the refinement
    // correction in w: the kriging weights are their sum
    double ll = 0.0;
    if ((rc = egs_mle_eval(p, theta, &ll, nullptr, nullptr)) != EGS_OK) return rc;
    launch_add_inplace(p->z, p->w, p->n, p->stream);
  } else {
    if ((rc = egs_covariance_generate(p, theta)) != EGS_OK) return rc;
    if ((rc = egs_potrf(p)) != EGS_OK) return rc;
    if ((rc = egs_restore_observations(p)) != EGS_OK) return rc;
    enqueue_trsv(p);
    enqueue_trsv_t(p);
  }
  cudaStream_t st = p->stream;
  double *c12t = nullptr, *dxm = nullptr, *dym = nullptr, *dzm = nullptr;
  long long dummy = 0;
  if ((rc = dev_alloc(&c12t, (size_t)p->n * n_miss, &dummy, st)) || (rc = dev_alloc(&dxm, n_miss, &dummy, st)) ||
      (rc = dev_alloc(&dym, n_miss, &dummy, st)) || (rc = dev_alloc(&dzm, n_miss, &dummy, st))) {
    for (void* b : {(void*)c12t, (void*)dxm, (void*)dym, (void*)dzm}) dev_free(b, st);
    return rc;
  }
  cudaMemcpyAsync(dxm, x_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dym, y_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st);
  MaternParams mp;
  make_matern_params(theta, &mp);
  rc = launch_matern_block(c12t, p->n, p->n, n_miss, p->x, p->y, dxm, dym, mp, st);
  launch_gemv_t_block(c12t, p->n, p->n, n_miss, p->z, dzm, st);
  cudaMemcpyAsync(z_miss, dzm, n_miss * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (rc == EGS_OK) rc = check_cuda("egs_problem_predict");
  for (void* b : {(void*)c12t, (void*)dxm, (void*)dym, (void*)dzm}) dev_free(b, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == EGS_OK) rc = check_cuda("egs_problem_predict/sync");
  return rc;
}

// ---------------------------------------------------------------------------
// MLOE / MMOM (LinearAlgebraMethods<T>::ExaGeoStatMLETileMLOEMMOM,
// src/linear-algebra-solvers/LinearAlgebraMethods.cpp:802-1131, and the
// dmloe-mmom codelet, src/runtime/starpu/concrete/dmloe-mmom-codelet.cpp:73-102)
// ---------------------------------------------------------------------------

int egs_mloe_mmom_host(int n_obs, int n_miss, int dts, const double* x_obs, const double* y_obs,
                       const double* x_miss, const double* y_miss, const double* theta_true,
                       const double* theta_est, double* mloe, double* mmom) {
  if (n_obs <= 0 || n_miss <= 0 || dts <= 0 || !x_obs || !y_obs || !x_miss || !y_miss || !theta_true ||
      !theta_est || !mloe || !mmom)
    return EGS_ERR_INVALID;
  MaternParams mt, ma;
  if (make_matern_params(theta_true, &mt) != EGS_OK || make_matern_params(theta_est, &ma) != EGS_OK) {
    set_last_error("theta outside the Matern domain (sigma2 > 0, beta > 0, nu > 0)", "egs_mloe_mmom_host");
    return EGS_ERR_INVALID;
  }
  // K_t, K_a: the observed covariance under the true / the estimated theta, factored
  // pa is created first so that pt, which borrows pa's stream below, is destroyed first
  egs_problem *pt = nullptr, *pa = nullptr;
  int rc = egs_problem_create(&pa, n_obs, dts);
  if (rc != EGS_OK) return rc;
  std::unique_ptr<egs_problem, int (*)(egs_problem*)> ga(pa, egs_problem_destroy);
  if ((rc = egs_problem_create(&pt, n_obs, dts)) != EGS_OK) return rc;
  std::unique_ptr<egs_problem, int (*)(egs_problem*)> gt(pt, egs_problem_destroy);
  for (egs_problem* p : {pt, pa}) {
    if ((rc = egs_problem_set_locations(p, x_obs, y_obs)) != EGS_OK) return rc;
    p->have_observations = true;  // the solves below set z themselves
  }
  if ((rc = egs_covariance_generate(pt, theta_true)) != EGS_OK || (rc = egs_potrf(pt)) != EGS_OK) return rc;
  if ((rc = egs_covariance_generate(pa, theta_est)) != EGS_OK || (rc = egs_potrf(pa)) != EGS_OK) return rc;
  // both problems run on pa's stream from here
  cudaStream_t st = pa->stream;
  const long long np = pa->np;
  double *kt = nullptr, *ka = nullptr, *dxm = nullptr, *dym = nullptr, *ya = nullptr, *u = nullptr, *dots = nullptr;
  long long dummy = 0;
  auto cleanup = [&]() {
    for (void* b : {(void*)kt, (void*)ka, (void*)dxm, (void*)dym, (void*)ya, (void*)u, (void*)dots}) dev_free(b, st);
    cudaStreamSynchronize(st);
  };
  if ((rc = dev_alloc(&kt, (size_t)np * n_miss, &dummy, st)) || (rc = dev_alloc(&ka, (size_t)np * n_miss, &dummy, st)) ||
      (rc = dev_alloc(&dxm, n_miss, &dummy, st)) || (rc = dev_alloc(&dym, n_miss, &dummy, st)) ||
      (rc = dev_alloc(&ya, np, &dummy, st)) || (rc = dev_alloc(&u, np, &dummy, st)) ||
      (rc = dev_alloc(&dots, (size_t)4 * n_miss, &dummy, st))) {
    cleanup();
    return rc;
  }
  cudaMemsetAsync(kt, 0, (size_t)np * n_miss * sizeof(double), st);
  cudaMemsetAsync(ka, 0, (size_t)np * n_miss * sizeof(double), st);
  cudaMemcpyAsync(dxm, x_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dym, y_miss, n_miss * sizeof(double), cudaMemcpyHostToDevice, st);
  // k_t, k_a for every target: columns of leading dimension np (padding rows stay 0)
  if ((rc = launch_matern_block(kt, (int)np, n_obs, n_miss, pa->x, pa->y, dxm, dym, mt, st)) != EGS_OK ||
      (rc = launch_matern_block(ka, (int)np, n_obs, n_miss, pa->x, pa->y, dxm, dym, ma, st)) != EGS_OK ||
      (rc = egs_problem_set_stream(pt, st)) != EGS_OK) {
    cleanup();
    return rc;
  }
  for (int q = 0; q < n_miss; ++q) {
    const double* ktq = kt + (long long)q * np;
    const double* kaq = ka + (long long)q * np;
    double* d = dots + 4ll * q;
    // y_a = L_a^-1 k_a
    cudaMemcpyAsync(pa->z, kaq, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    enqueue_trsv(pa);
    cudaMemcpyAsync(ya, pa->z, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    launch_dot(ya, ya, (int)np, d + 0, st);                       // k_a' K_a^-1 k_a
    // L_a^-1 k_t . y_a = k_t' K_a^-1 k_a
    cudaMemcpyAsync(pa->z, ktq, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    enqueue_trsv(pa);
    launch_dot(pa->z, ya, (int)np, d + 1, st);
    // k_t' K_t^-1 k_t
    cudaMemcpyAsync(pt->z, ktq, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    enqueue_trsv(pt);
    launch_dot(pt->z, pt->z, (int)np, d + 2, st);
    // w_a = L_a^-T y_a; w_a' K_t w_a = |L_t^T w_a|^2
    cudaMemcpyAsync(pa->z, ya, np * sizeof(double), cudaMemcpyDeviceToDevice, st);
    enqueue_trsv_t(pa);
    launch_trmv_t(pt->tiles, pt->ts, pt->nt, pa->z, u, st);
    launch_dot(u, u, (int)np, d + 3, st);
  }
  std::vector<double> h(4ll * n_miss);
  cudaMemcpyAsync(h.data(), dots, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  rc = check_cuda("egs_mloe_mmom_host");
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == EGS_OK) rc = check_cuda("egs_mloe_mmom_host/sync");
  cleanup();
  if (rc != EGS_OK) return rc;
  const double s2t = theta_true[0], s2a = theta_est[0];
  double loe = 0.0, mom = 0.0;
  for (int q = 0; q < n_miss; ++q) {
    const double aka = h[4 * q], tka = h[4 * q + 1], tkt = h[4 * q + 2], wkw = h[4 * q + 3];
    const double e2 = s2t - 2.0 * tka + wkw;  // MSE of the predictor built with theta_est
    const double e3 = s2t - tkt;              // MSE of the predictor built with theta_true
    const double e4 = s2a - aka;              // MSE the estimated model claims
    if (e3 == 0.0) {
      loe -= 1.0;
      mom -= 1.0;
    } else {
      loe += e2 / e3 - 1.0;
      mom += e4 / e2 - 1.0;
    }
  }
  *mloe = loe / n_miss;
  *mmom = mom / n_miss;
  return EGS_OK;
}

namespace egs {

// The first `steps` tile steps of the factorisation of p's tiles as they are
// (no generation): the panels of columns 0 .. steps-1 and their trailing
// updates of every later tile.  Used by the Fisher information
// (augmented matrices).  Returns the LAPACK-style info or an error.
int enqueue_potrf_steps(egs_problem* p, int steps) {
  EGS_CUDA_TRY(cudaMemsetAsync(p->flags, 0, 2 * sizeof(int), p->stream));
  int rc = enqueue_potrf(p, steps);
  if (rc != EGS_OK) return rc;
  EGS_CUDA_TRY(cudaMemcpyAsync(p->hflags, p->flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  EGS_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (p->hflags[1] != 0) {
    set_last_error("a device-side wait exceeded its limit", "enqueue_potrf_steps");
    return EGS_ERR_TIMEOUT;
  }
  if (p->hflags[0] > 0) {
    set_last_error("Matrix is not positive definite", "enqueue_potrf_steps");
    return p->hflags[0];
  }
  return check_cuda("enqueue_potrf_steps");
}

int problem_tiles(egs_problem* p, double** tiles, int* ts, int* nt, cudaStream_t* st) {
  *tiles = p->tiles;
  *ts = p->ts;
  *nt = p->nt;
  *st = p->stream;
  return EGS_OK;
}

}  // namespace egs
