// Launch helpers shared by the translation units of the B200 path.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include "common.cuh"
#include "bessel_k.cuh"

namespace egs {

int make_matern_params(const double* theta, MaternParams* out);
// Builds the Chebyshev table of K_nu for theta (ktab: kKtabDoubles device
// doubles), then generates every lower tile.
int launch_matern_tiles(double* tiles, const double* x, const double* y, int n, int ts, int nt,
                        const MaternParams* dparams, double* ktab, cudaStream_t st);
// Chebyshev tables of nproblems parameter sets (tab: nproblems * kKtabDoubles).
void launch_matern_ktab(const MaternParams* params, double* tab, int nproblems, cudaStream_t st);
int launch_matern_block(double* a, int lda, int rows, int cols, const double* x1, const double* y1,
                        const double* x2, const double* y2, const MaternParams& p, cudaStream_t st);

// Factorisation building blocks (potrf.cu).  All offsets are element offsets
// inside a tile; tiles are addressed by lower-tile slot.
void launch_potrf_diag_block(double* tiles, int ts, long long slot, int off, int col_base, int* info,
                             cudaStream_t st);
void launch_trsm_rows(double* tiles, int ts, long long slot0, int ntiles, int row0, int col0,
                      long long lslot, cudaStream_t st);
void launch_trsm_rows_panel(double* tiles, int ts, long long slot0, int ntiles, int row0_first, int row0, int col0,
                            long long lslot, cudaStream_t st);
void launch_trsv_diag(const double* tiles, int ts, long long slot, double* zk, cudaStream_t st);
void launch_gemv_panel(const double* tiles, int ts, int nt, int k, double* z, cudaStream_t st);
void launch_trsv_t_diag(const double* tiles, int ts, long long slot, double* zk, cudaStream_t st);
void launch_gemv_t_panel(const double* tiles, int ts, int nt, int k, double* z, cudaStream_t st);
void launch_logdet_partials(const double* tiles, int ts, int nt, int n, double* partial, cudaStream_t st);
void launch_finalize(const double* partial, int nt, const double* z, int n, double* result,
                     const int* info, cudaStream_t st);
void launch_sumsq_diff(const double* a, const double* b, int n, double* out, cudaStream_t st);
void launch_trmv(const double* tiles, int ts, int nt, const double* e, double* part, double* z, cudaStream_t st);
void launch_gemv_t_block(const double* a, long long lda, int rows, int cols, const double* w, double* out,
                         cudaStream_t st);

// Band (diagonal super-tile) factorisation on logical tiles of dts elements,
// element by element inside the lower-tile pool (dst.cu); for dts != ts.
int launch_dst_band(double* tiles, int ts, int nt, int n, int dts, int band, int* info, cudaStream_t st);

// FP64 tensor-core update C -= A * B^T over global row indices (dgemm_tma.cu).
// Every operand row is a global row of one problem (tile row g / ts); A and B take
// their K columns from one tile column starting at a local column offset; C is
// addressed by (global row, global column), upper tiles never written.
struct GemmDesc {
  int M, N, K;
  int a_row0, a_col0, a_tcol;
  int b_row0, b_col0, b_tcol;
  int c_row0, c_col0;
  int lower;
  int MB, NB;
  long long total;
  int ts, nt, np;
  long long tile_base;  // slot of this problem's tile (0, 0) in a pool of problems
  // C addressing: c_mode 0 = lower-tile pool (tile_base + tile_slot(ti, tj, nt));
  // c_mode 1 = FP64 band pool of a mixed-precision problem: only tiles with
  // ti - tj <= c_band are written, at slot (c_tile_off + tj) * (c_band + 1) + (ti - tj).
  int c_mode, c_band, c_tile_off;
};

// Batched launches: blocks [begin[j], begin[j+1]) belong to job j.
struct GemmJobs {
  const GemmDesc* jobs;
  const long long* begin;
  int njobs;
  long long total;
};

void finish_desc(GemmDesc& d);  // fills MB, NB, total
int launch_gemm_batched(const void* tmap, double* tiles, const GemmDesc* jobs, const long long* begin, int njobs,
                        long long total, int* err, cudaStream_t st);
int gemm_init_tensor_map(void* tmap_storage, double* tiles, int ts, long long ntiles);
// The driver's cuTensorMapEncodeTiled (looked up once).
int tensor_map_encoder(void** fn);
int launch_gemm_trailing(const void* tmap, double* tiles, int ts, int nt, int k, int* err, cudaStream_t st);
int launch_gemm_rows(const void* tmap, double* tiles, int ts, int nt, int M, int N, int K, int a_row0,
                     int a_col0, int a_tcol, int b_row0, int b_col0, int b_tcol, int c_row0, int c_col0,
                     int lower, int* err, cudaStream_t st, int max_ctas = 0);
int gemm_num_sms();

// Mixed-precision evaluation (mixed.cu, split_gemm.cu).
void launch_matern_mixed(double* band, float* off, const double* x, const double* y, int n, int ts,
                         const int4* tinfo, long long ntiles, const MaternParams* params, double* ktab,
                         cudaStream_t st);
void launch_gather_column(const double* band, const float* off, double* W, int ts, int nt, int b, int k,
                          cudaStream_t st);
void launch_scatter_column(const double* W, double* band, float* off, double* inv, int ts, int nt, int b, int k,
                           cudaStream_t st);
void launch_logdet_band(const double* band, int ts, int nt, int b, int n, double* partial, cudaStream_t st);
void launch_mixed_solve(const double* band, const float* off, const double* inv, int ts, int nt, int b, double* v,
                        double* tmp, cudaStream_t st, long long* launches);
void launch_gather_panel(const double* band, double* W2, int ts, int b, int nb, int k, cudaStream_t st);
void launch_scatter_panel(const double* W2, double* band, double* inv, double* W, int ts, int b, int nb, int k,
                          cudaStream_t st);
void launch_scatter_offband(const double* W, float* off, int ts, int nt, int b, int nb, int k, cudaStream_t st);
const float* offband_tile(const float* off, int ts, int nt, int b, int i, int k);
void launch_trmv_t(const double* tiles, int ts, int nt, const double* w, double* out, cudaStream_t st);
void launch_dot(const double* a, const double* b, int n, double* out, cudaStream_t st);
long long residual_scratch_doubles(int n);
void launch_add_inplace(double* a, const double* b, int n, cudaStream_t st);
void launch_matern_residual(const double* x, const double* y, const double* z, const double* v, int n, int np,
                            const MaternParams* params, const double* ktab, double* scratch, double* r,
                            cudaStream_t st);
void launch_finalize_mixed(const double* partial, int nt, const double* z, const double* v, const double* w, int n,
                           double* result, const int* info, cudaStream_t st);
int split_tensor_map(void* storage, const __half* base, int ts, long long rows);
int split_c_map(void* tm_c, const float* c_pool, int ts, long long nslots);
void launch_panel_split(const double* W, int ts, int t0, int ntiles, int row_tile0, float* inv_scale, __half* Ph,
                        __half* Pl, cudaStream_t st);
long long split_targets(int nt, int band, int k);
int ozaki_slices();
int ozaki_tensor_map(void* storage, const int8_t* slices, int ts, long long rows);
void launch_ozaki_slice(const double* W, int ts, int t0, int ntiles, int row_tile0, double* scale, int8_t* slices,
                        long long rows, cudaStream_t st);
}  // namespace egs
#include <vector>
namespace egs {
long long ozaki_targets(int ts, int nt, int band, int k, std::vector<int4>& out);
long long ozaki_trsm_targets(int ts, int nt, int first, std::vector<int4>& out);
void launch_panel_prepare(const double* W, int ts, int t0, int ntiles, int row_tile0, double* oz_scale,
                          int8_t* slices, long long rows, float* inv_scale, __half* Ph, __half* Pl, cudaStream_t st);
void launch_ozaki_slice_f32(const float* tiles0, int ts, int ntiles, int row_tile0, double* scale, int8_t* slices,
                            long long rows, cudaStream_t st);
void launch_ozaki_slice_rows(const double* src, int ts, long long row0, double* scale, int8_t* slices,
                             long long rows, cudaStream_t st);
int launch_ozaki_trsm(const void* tm_s, const int4* targets, int ntargets, long long total, int ts, int k,
                      long long b_row_base, double* w_out, const double* scale, int* err, cudaStream_t st);
int launch_ozaki_band(const void* tm_s, const int4* targets, int ntargets, long long total, int ts, int band,
                      double* band_pool, const double* scale, int* err, cudaStream_t st);
int launch_split_update(const void* tm_hi, const void* tm_lo, const void* tm_c, int ts, int nt,
                        int band, int k, float* c_pool,
                        const float* inv_scale, int* err, cudaStream_t st, int max_ctas = 0);

}  // namespace egs
