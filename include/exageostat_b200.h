/*
 * exageostat_b200.h -- C ABI of the B200 (sm_100a) maximum-likelihood path.
 *
 * Plain C: pointers, sizes and int status codes; nothing here throws, traps or
 * needs a C++ or torch type.  Every function returns EGS_OK (0) on success, a
 * positive value for a Cholesky failure (1-based global column of the first
 * non-positive pivot, the LAPACK "info"), or a negative EGS_ERR_* code.
 *
 * Each entry point names the ExaGeoStatCPP interface it replaces (paths are
 * relative to the ExaGeoStatCPP source tree).
 */
#ifndef EXAGEOSTAT_B200_H
#define EXAGEOSTAT_B200_H

#if defined(__GNUC__)
#define EGS_API __attribute__((visibility("default")))
#else
#define EGS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define EGS_OK 0
#define EGS_ERR_INVALID (-1)     /* bad argument: sizes, null pointers, theta outside its domain */
#define EGS_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define EGS_ERR_NO_DEVICE (-3)   /* no usable CUDA device */
#define EGS_ERR_OOM (-4)         /* device allocation refused */
#define EGS_ERR_TIMEOUT (-5)     /* a bounded device-side wait gave up */
#define EGS_ERR_STATE (-6)       /* call order: e.g. evaluation before locations were set */

/* Opaque device-resident problem: locations, observations, the tile-major lower
 * covariance storage and the reduction buffers of one N.  Replaces the
 * DescriptorData<T> set of Chameleon descriptors (C, Z, Zcpy, det, product)
 * created by LinearAlgebraMethods<T>::InitiateDescriptors
 * (src/linear-algebra-solvers/LinearAlgebraMethods.cpp:36-118). */
typedef struct egs_problem egs_problem;

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
EGS_API int egs_version(void);
/* Human-readable name of a status code (static storage). */
EGS_API const char* egs_status_string(int status);
/* Message of the last error raised on the calling host thread ("" if none). */
EGS_API const char* egs_last_error(void);

/* Select and initialise the CUDA device.  Replaces
 * ExaGeoStatHardware::InitHardware (src/hardware/ExaGeoStatHardware.cpp:126-172). */
EGS_API int egs_hardware_init(int device);

/* ---- descriptors ------------------------------------------------------- */

/* Allocate a problem of n locations with dense tile size dts (the reference's
 * --dts; the device tile is dts rounded up to a multiple of 64).
 * Replaces LinearAlgebraMethods<T>::InitiateDescriptors
 * (LinearAlgebraMethods.cpp:36-118) + DescriptorData<T>::SetDescriptor
 * (src/data-units/DescriptorData.cpp:148-191). */
EGS_API int egs_problem_create(egs_problem** out, int n, int dts);
/* Free everything; replaces DescriptorData<T>::~DescriptorData (DescriptorData.cpp:21-62). */
EGS_API int egs_problem_destroy(egs_problem* p);
/* n, device tile size, number of tile rows, device bytes held. */
EGS_API int egs_problem_info(const egs_problem* p, int* n, int* ts, int* nt, long long* bytes);
/* Run all later work of this problem on the given cudaStream_t (NULL: the problem's own stream). */
EGS_API int egs_problem_set_stream(egs_problem* p, void* cuda_stream);

/* Select the factorisation of this problem: band = 0 (default) is the exact dense
 * Cholesky; band >= 1 is the diagonal super-tile approximation with that many
 * tiles in the band, replacing ChameleonDST<T>::ExaGeoStatPotrfTile
 * (src/linear-algebra-solvers/concrete/chameleon/dst/ChameleonDST.cpp:23-150,
 * --computation=diag_approx --band=b).  The approximation is defined on the
 * caller's tiles of dts elements: when dts is a multiple of 64 they are the
 * device tiles (tensor-core updates); otherwise the same loop runs on logical
 * tiles of dts inside the device tiles, element by element (a slower form for
 * small or odd tiles such as the reference's dts = 8 tests). */
EGS_API int egs_problem_set_band(egs_problem* p, int band);

/* Precision of the factorisation, the reference's Precision enum
 * (inst/include/common/Definitions.hpp:258-262, Configurations --precision). */
#define EGS_PRECISION_DOUBLE 1
#define EGS_PRECISION_MIXED 2

/* Select the precision before locations and observations are set.
 * EGS_PRECISION_DOUBLE (default) is the exact FP64 path.  EGS_PRECISION_MIXED
 * keeps the diagonal tiles and band_tiles tile rows below them in FP64 and
 * stores every other tile in FP32: the diagonal potrf, the panel solves, the
 * band updates, the log-determinant and the dot product run in FP64; off-band
 * updates run on FP16 tensor cores from a per-row scaled two-part split of the
 * panel (FP32-level accuracy), and the quadratic form gets one iterative
 * refinement step against the FP64 covariance.  The device tile becomes dts
 * rounded up to a multiple of 256.  Only egs_mle_eval (and the info, stream,
 * profiling and observation calls) is available on a mixed problem; a mixed
 * problem cannot return to FP64.  The reference declares the option but its
 * dense path has no mixed implementation. */
EGS_API int egs_problem_set_precision(egs_problem* p, int precision, int band_tiles);

/* Arithmetic of the FP64 band updates of a mixed problem:
 * EGS_BAND_OZAKI_INT8 (default) splits the panel into seven signed 7-bit
 * slices per row and forms the products exactly on the int8 tensor cores
 * (FP64-class accuracy, 2^-49 of the row maxima per operand);
 * EGS_BAND_FP64_DMMA uses the FP64 tensor path. */
#define EGS_BAND_OZAKI_INT8 0
#define EGS_BAND_FP64_DMMA 1
EGS_API int egs_problem_set_band_method(egs_problem* p, int method);

/* Look-ahead of a mixed problem (Ozaki band method): the FP64 panel of step
 * k+1 (diagonal tile, band rows, L^-1) runs on `sms` SMs beside the off-band
 * update of step k, which keeps the other SMs; 0 runs them one after the
 * other (the default: at N = 102,400 the off-band update loses as much time
 * to the reserved SMs as the overlap hides).  A scheduling choice only:
 * results are bit-identical either way. */
EGS_API int egs_problem_set_lookahead(egs_problem* p, int sms);

/* Create a problem directly in the given precision (EGS_PRECISION_DOUBLE or
 * EGS_PRECISION_MIXED with band_tiles FP64 tile rows): the same as
 * egs_problem_create followed by egs_problem_set_precision, without ever
 * holding the FP64 tile storage of a mixed problem.  Replaces the descriptor
 * set-up of LinearAlgebraMethods<T>::InitiateDescriptors for the precision the
 * Configurations select (LinearAlgebraMethods.cpp:36-118, Definitions.hpp:258-262). */
EGS_API int egs_problem_create_ex(egs_problem** out, int n, int dts, int precision, int band_tiles);

/* Device bytes a problem of this shape holds (an upper bound of what
 * egs_problem_info reports after creation), for admission by HBM footprint.
 * Pure arithmetic: needs no device. */
EGS_API int egs_problem_footprint(int n, int dts, int precision, int band_tiles, long long* bytes);

/* Copy n locations from host memory (Locations<T> SoA x[], y[],
 * src/data-units/Locations.cpp:94-118).  A mixed-precision problem keeps its
 * points in locality (Morton) order: it sorts them here -- keeping the
 * caller's order when it is already sorted -- and permutes the observations
 * given to it the same way, so that its FP64 band holds the large covariances;
 * results do not depend on the caller's order, and egs_get_observations
 * returns vectors in the caller's order. */
EGS_API int egs_problem_set_locations(egs_problem* p, const double* x, const double* y);
/* Same from device memory. */
EGS_API int egs_problem_set_locations_device(egs_problem* p, const double* x, const double* y);
/* Copy the n observations Z into the saved copy Zcpy (the iteration-0 dlacpy
 * Z -> Zcpy of ChameleonImplementation.cpp:113-119). */
EGS_API int egs_problem_set_observations(egs_problem* p, const double* z);
EGS_API int egs_problem_set_observations_device(egs_problem* p, const double* z);

/* ---- stages of one evaluation (device resident) ------------------------ */

/* Lower tiles of C(theta), theta = (sigma^2, beta, nu).  Replaces
 * RuntimeFunctions<T>::CovarianceMatrix (src/runtime/starpu/StarPuFunctions.cpp:24-45)
 * with UnivariateMaternStationary<T>::GenerateCovarianceMatrix
 * (src/kernels/concrete/UnivariateMaternStationary.cpp:39-67). */
EGS_API int egs_covariance_generate(egs_problem* p, const double* theta);
/* In-place lower Cholesky of the tiles.  Replaces ChameleonDense<T>::ExaGeoStatPotrfTile
 * (src/linear-algebra-solvers/concrete/chameleon/dense/ChameleonDense.cpp:25-37).
 * Returns > 0 (info) when the matrix is not positive definite. */
EGS_API int egs_potrf(egs_problem* p);
/* Z := Zcpy (ChameleonImplementation.cpp:120-124). */
EGS_API int egs_restore_observations(egs_problem* p);
/* Z := L^-1 Z.  Replaces ChameleonImplementation<T>::ExaGeoStatTrsmTile
 * (ChameleonImplementation.cpp:337-347, called at :216-217). */
EGS_API int egs_trsv(egs_problem* p);
/* log|C| = 2 sum log L_kk (RuntimeFunctions<T>::ExaGeoStatMeasureDetTileAsync,
 * StarPuFunctions.cpp:119-135; dmdet-codelet.cpp:73-80), Z^T Z
 * (RuntimeFunctions<T>::ExaGeoStatDoubleDotProduct, StarPuFunctions.cpp:189-204)
 * and the log-likelihood (ChameleonImplementation.cpp:257-265). */
EGS_API int egs_loglik_parts(egs_problem* p, double* loglik, double* logdet, double* dot);
/* Copy tile (i, j), i >= j, to host (ts*ts doubles, column-major). */
EGS_API int egs_get_tile(egs_problem* p, int i, int j, double* host_out);
/* Copy the current Z (n doubles) to host. */
EGS_API int egs_get_observations(egs_problem* p, double* host_z);
/* Zcpy := Z, the iteration-0 copy of ChameleonImplementation.cpp:113-119
 * (ExaGeoStatLapackCopyTile, ChameleonImplementation.cpp:329-335, from Z to Zcpy). */
EGS_API int egs_save_observations(egs_problem* p);
/* Z := L^-T Z with the factor in the tiles: the transposed solve of
 * ExaGeoStatTrsmTile (ChameleonImplementation.cpp:337-347 with Trans) and the
 * second half of ExaGeoStatPosvTile (LinearAlgebraMethods.hpp:216, dposv). */
EGS_API int egs_trsv_transpose(egs_problem* p);
/* Copy a host tile (ts*ts doubles, column-major) into tile (i, j), i >= j: the
 * tile-wise form of ExaGeoStatLap2Desc (LinearAlgebraMethods.hpp:275).  The
 * caller keeps the identity padding of the last diagonal tile. */
EGS_API int egs_set_tile(egs_problem* p, int i, int j, const double* host_in);
/* A sequence is a CUDA stream owned by the library: egs_sequence_create replaces
 * ExaGeoStatCreateSequence (CHAMELEON_Sequence_Create, LinearAlgebraMethods.hpp:169),
 * egs_sequence_wait replaces ExaGeoStatSequenceWait (CHAMELEON_Sequence_Wait,
 * LinearAlgebraMethods.hpp:161): it returns when all work on the stream is done.
 * A problem runs its work on a sequence after egs_problem_set_stream(p, sequence). */
EGS_API int egs_sequence_create(void** sequence);
EGS_API int egs_sequence_wait(void* sequence);
EGS_API int egs_sequence_destroy(void* sequence);

/* One full log-likelihood evaluation at theta on the resident data: restore Z,
 * generate, factor, log-det, solve, dot, assemble.  Replaces
 * ChameleonImplementation<T>::ExaGeoStatMLETile (ChameleonImplementation.cpp:35-327).
 * logdet and dot may be NULL. */
EGS_API int egs_mle_eval(egs_problem* p, const double* theta, double* loglik, double* logdet, double* dot);

/* ---- synthetic data (the reference's generator semantics) ---------------- */

/* n jittered-grid locations in [0,1]^2, Morton sorted and 16-bit quantised, drawn
 * from the C library's rand(); srand(seed) first when reseed != 0.  Replaces
 * LocationGenerator<T>::GenerateLocations (src/data-generators/LocationGenerator.cpp:25-123). */
EGS_API int egs_generate_locations(int n, int seed, int reseed, double* x, double* y);
/* Random hold-out split of n values with their locations (host arrays): a
 * Fisher-Yates shuffle drawing j = i + rand() / (RAND_MAX / (n - i) + 1) from the
 * C library's rand() state as it stands (no reseeding), then the first n_miss
 * entries go to *_miss and the other n - n_miss, in order, to *_obs.  The inputs
 * are not modified.  Replaces PredictionHelpers<T>::PickRandomPoints / Shuffle
 * (src/prediction/PredictionHelpers.cpp:23-168, draw at :146) for one variable. */
EGS_API int egs_shuffle_split(int n, int n_miss, const double* z, const double* x, const double* y,
                              double* z_obs, double* x_obs, double* y_obs, double* z_miss, double* x_miss,
                              double* y_miss);
/* n N(0,1) samples of LAPACK DLARNV(IDIST=3, ISEED) (ISEED entries in [0, 4095],
 * ISEED[3] odd), as drawn at LinearAlgebraMethods.cpp:347-364. */
EGS_API int egs_dlarnv_normal(const int* iseed, int n, double* out);
/* Z = L e at theta with e = DLARNV(3, {seed, seed, seed, 1}) and L = chol(C(theta))
 * on the resident locations; Z becomes the problem's observations (and is copied
 * to z_out when it is not NULL).  Replaces
 * LinearAlgebraMethods<T>::GenerateObservationsVector (LinearAlgebraMethods.cpp:333-449). */
EGS_API int egs_generate_observations(egs_problem* p, const double* theta, int seed, double* z_out);

/* ---- optimiser ----------------------------------------------------------- */

/* Objective for egs_bobyqa_maximize: value at x (n parameters). */
typedef double (*egs_objective_fn)(int n, const double* x, void* ctx);
/* Maximise f over the box [lb, ub] without derivatives, starting from x (in/out:
 * the best point on return), with initial trust radius rhobeg (<= 0: a quarter
 * of the narrowest box width), stopping after maxeval evaluations or when an
 * improvement of the best value is below ftol_abs.  *fbest receives the best
 * value, *nevals the number of evaluations.  Replaces the NLopt LN_BOBYQA run of
 * StarpuRuntimeSolver<T>::ModelingOperations (src/runtime-solver/concrete/
 * StarpuRuntimeSolver.cpp:28-66): same first evaluations (x0, then x0 + rhobeg
 * e_i ...), same maxeval / ftol_abs stopping, best value returned. */
EGS_API int egs_bobyqa_maximize(int n, double* x, const double* lb, const double* ub, double rhobeg,
                                double ftol_abs, int maxeval, egs_objective_fn f, void* ctx, double* fbest,
                                int* nevals);

/* ---- instrumentation ----------------------------------------------------- */

/* Stages of an evaluation, for the per-stage counters below (the reference's
 * START_TIMING/STOP_TIMING around matrix generation, factorisation and solve,
 * ChameleonImplementation.cpp:127-220). */
#define EGS_STAGE_GENERATE 0   /* Matern tiles */
#define EGS_STAGE_PANEL 1      /* diagonal-tile factorisation + panel triangular solve */
#define EGS_STAGE_UPDATE 2     /* trailing syrk/gemm on the FP64 tensor path */
#define EGS_STAGE_SOLVE 3      /* Z := L^-1 Z (and L^-T for kriging) */
#define EGS_STAGE_REDUCE 4     /* log-det, dot, log-likelihood assembly */
#define EGS_STAGE_UPDATE_LOW 5 /* mixed precision: off-band update on FP16 tensor cores (FP32-accurate) */
#define EGS_NUM_STAGES 6

/* Enable (1) or disable (0) CUDA-event timing of every stage on the problem's
 * stream; either call resets the counters.  Kernel launches are always counted. */
EGS_API int egs_problem_set_profiling(egs_problem* p, int enable);
/* Accumulated device milliseconds, algorithmic flops (real rows only) and kernel
 * launches per stage since the last egs_problem_set_profiling; each pointer may be
 * NULL or point to EGS_NUM_STAGES elements. */
EGS_API int egs_problem_stage_stats(egs_problem* p, double* ms, double* flops, long long* launches);

/* ---- evaluation without allocation ---------------------------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc --
 * an application whose device memory belongs to another allocator (a
 * framework's caching allocator, or a pool sized once at start-up) and loops
 * that must not pay the device-wide synchronisation of cudaMalloc/cudaFree on
 * every evaluation -- this pair evaluates one log-likelihood without allocating
 * anything.  egs_mle_noalloc_workspace reports how many doubles of device
 * workspace an evaluation of n points with tile dts needs (lower tiles plus
 * three padded vectors); it rejects n above 4096 device tiles (4096 *
 * round-up(dts, 64) points).
 *
 * egs_mle_eval_noalloc then runs the whole evaluation of egs_mle_eval on the
 * caller's stream: x, y, z are n device doubles (read only), theta is host
 * memory, work is the 16-byte aligned device workspace (overwritten), and the
 * log-likelihood is written to the host double *loglik.  It calls no
 * cudaMalloc, cudaFree or other allocating routine: its small per-call state
 * lives in one static device array of about 41 KB that every GPU which loads
 * the library keeps until the process exits.  The first call on a device looks
 * up that array's device address, so make this first call before any stream
 * capture.  All calls share the array: calls whose work overlaps on the GPU
 * (other streams, other host threads) race on it and must be serialised by the
 * caller. */
EGS_API int egs_mle_noalloc_workspace(int n, int dts, long long* doubles);
EGS_API int egs_mle_eval_noalloc(int n, int dts, const double* x, const double* y, const double* z,
                                 const double* theta, double* work, long long work_doubles, double* loglik,
                                 void* cuda_stream);

/* From its second evaluation on, egs_mle_eval replays the whole evaluation of a
 * problem as one CUDA graph (captured once).  While profiling is on, a second
 * graph that also records the stage-timing events is captured and replayed
 * (at the first profiled evaluation after the first one); if its events give no
 * times, profiled evaluations of this problem fall back to direct launches.
 * enable = 0 turns replay off for this problem, 1 (the default) on. */
EGS_API int egs_problem_set_graphs(egs_problem* p, int enable);

/* ---- batched evaluation of many independent problems -------------------- */

/* No counterpart in the reference, which evaluates one problem per call of
 * ExaGeoStatMLETile (ChameleonImplementation.cpp:35-327).  A batch holds B
 * independent problems (problem i: n[i] points, caller arrays concatenated in
 * order in x, y, z, host memory) factored with one common tile size
 * (round-up(dts, 64)).  Every stage runs once per batch: one tile pool and one
 * TMA descriptor for all problems, the 64x64 potrf, row solves and
 * tensor-core updates of all problems still active at step k in one launch
 * each.  From the second egs_batch_eval on, the whole batched evaluation is one
 * CUDA graph replay.  Results are the same formulas as egs_mle_eval per
 * problem; the tile size can differ from a single-problem call with another dts,
 * so results agree to rounding, not bit for bit. */
typedef struct egs_batch egs_batch;
EGS_API int egs_batch_create(egs_batch** out, int B, const int* n, int dts, const double* x, const double* y,
                             const double* z);
EGS_API int egs_batch_destroy(egs_batch* b);
/* Common tile size, tile rows of the largest problem, device bytes held, and
 * kernel launches of one evaluation (0 before the first). */
EGS_API int egs_batch_info(const egs_batch* b, int* ts, int* nt_max, long long* bytes,
                           long long* launches_per_eval);
/* theta: 3*B host doubles (sigma^2, beta, nu of problem i at 3i); loglik: B
 * host doubles; status (may be NULL): B ints, 0 or the potrf info of problem i
 * (1-based column of the first non-positive pivot).  Returns EGS_OK, or
 * EGS_ERR_STATE when at least one problem was not positive definite (the other
 * problems' results are still valid). */
EGS_API int egs_batch_eval(egs_batch* b, const double* theta, double* loglik, int* status);
/* Times one graph-replayed evaluation for each candidate tile size and returns
 * the fastest in *best_ts (device milliseconds of that evaluation in *best_ms,
 * may be NULL). */
EGS_API int egs_batch_autotune(int B, const int* n, const double* x, const double* y, const double* z,
                               const double* theta, const int* candidates, int ncand, int* best_ts,
                               double* best_ms);

/* Size classes of a batch (no counterpart in the reference, which evaluates
 * one problem per process).  The problems are cut by N into nclass classes --
 * class c holds upper_n[c-1] < n <= upper_n[c] (upper_n ascending, the last at
 * least the largest n) -- each an egs_batch with its own tile size dts[c];
 * egs_batch_set_eval launches every class on its own stream before waiting for
 * any, so the classes' work overlaps on the device.  Arguments and results are
 * in the caller's problem order, as for egs_batch_eval. */
typedef struct egs_batch_set egs_batch_set;
EGS_API int egs_batch_set_create(egs_batch_set** out, int B, const int* n, const double* x, const double* y,
                                 const double* z, int nclass, const int* upper_n, const int* dts);
EGS_API int egs_batch_set_destroy(egs_batch_set* s);
EGS_API int egs_batch_set_eval(egs_batch_set* s, const double* theta, double* loglik, int* status);
/* Classes actually formed (empty ones are dropped), their bounds and tile sizes
 * (arrays of at least nclass entries), device bytes held. */
EGS_API int egs_batch_set_info(const egs_batch_set* s, int* nclass, int* upper_n, int* ts, long long* bytes);
/* The schedule for a batch: for 1 .. max_classes classes (bounds at equal shares
 * of the n^3 cost), each class's tile size from the candidates by timing the
 * class alone, then one timed replay of the whole set with the classes
 * overlapping; returns the fastest (nclass, upper_n[], dts[]) and its host-timed
 * milliseconds per evaluation. */
EGS_API int egs_batch_set_autotune(int B, const int* n, const double* x, const double* y, const double* z,
                                   const double* theta, const int* candidates, int ncand, int max_classes,
                                   int* nclass, int* upper_n, int* dts, double* best_ms);

/* ---- mixed-precision building block --------------------------------------- */

/* No counterpart in the reference.  One step k of the off-band trailing update
 * of the mixed-precision factorisation, on caller device memory: panel holds nt
 * column-major ts x ts FP64 tiles (tile t = rows t*ts.. of the solved panel
 * column; tiles <= k are not read), offband the FP32 off-band tiles
 * (i, j), i - j > band, in lower-tile order over nt - band - 1 tile rows.  Every
 * target (i, j) with k < j, j + band < i < nt gets C -= P_i P_j^T computed from
 * a per-row scaled two-part FP16 split of the panel on the tcgen05 tensor cores
 * (FP32 accumulation; about 2^-22 relative).  ts must be a multiple of 256;
 * k = -1 updates every off-band tile.  *ms (may be NULL) receives the device
 * time of the update kernel.  Allocates and frees its scratch per call. */
EGS_API int egs_split_update(int ts, int nt, int band, int k, const double* panel, float* offband, double* ms);

/* Test entry of the FP64-class band update of the mixed-precision form (Ozaki
 * scheme on the int8 tensor cores): for step k, C_ij -= L_ik L_jk^T for every
 * band target k < j <= i <= min(nt-1, j+band), with panel tiles
 * W[t] = L_{k+t,k} (t = 0 .. nt-k-1, FP64 column-major ts x ts, device; W[0]
 * is not read) and the FP64 band pool (nt*(band+1) tiles, slot
 * j*(band+1) + i-j, device).  ts must be a multiple of 128.  *ms receives the
 * update kernel's time.  Allocates its own scratch. */
EGS_API int egs_ozaki_band_update(int ts, int nt, int band, int k, const double* W, double* band_pool, double* ms);

/* ---- kernel plugin ------------------------------------------------------ */

/* rows x cols column-major block (leading dimension lda) on caller device
 * memory: A[i + j*lda] = Matern(|loc1[i] - loc2[j]|; theta); the device form of
 * Kernel<T>::GenerateCovarianceMatrix (inst/include/kernels/Kernel.hpp:93-97)
 * for "UnivariateMaternStationary".  The location pointers are already offset
 * to the block's first row / column.  distance_metric must be 0 (Euclidean),
 * which is what the MLE passes (ChameleonImplementation.cpp:172). */
EGS_API int egs_matern_block(double* a, int lda, int rows, int cols, const double* x1, const double* y1,
                     const double* x2, const double* y2, const double* theta, int distance_metric,
                     void* cuda_stream);

/* ---- host-buffer entry points ------------------------------------------- */

/* Log-likelihood of host data: copies locations and Z to the device, evaluates,
 * returns the scalar.  Reuses one cached problem per (n, dts) on the calling
 * thread, the way ExaGeoStatData keeps its descriptors across NLopt iterations. */
EGS_API int egs_mle_loglik_host(int n, int dts, const double* x, const double* y, const double* z,
                        const double* theta, double* loglik);

/* Kriging on a resident problem of either precision: z_miss = C(miss, obs)
 * C(obs, obs)^-1 z_obs at theta, for n_miss host target locations; the result
 * goes to host memory.  The mixed form uses its refined solve.  The same
 * computation as LinearAlgebraMethods<T>::ExaGeoStatMLEPredictTile
 * (LinearAlgebraMethods.cpp:527-552) with the observed locations, observations
 * and factor storage kept on the device between calls. */
EGS_API int egs_problem_predict(egs_problem* p, const double* theta, int n_miss, const double* x_miss,
                                const double* y_miss, double* z_miss);

/* Kriging.  Replaces LinearAlgebraMethods<T>::ExaGeoStatMLEPredictTile
 * (src/linear-algebra-solvers/LinearAlgebraMethods.cpp:451-605):
 * C22 = C(obs, obs), w = C22^-1 z_obs (dposv), z_miss = C12 w, and
 * mspe = sum (z_actual - z_miss)^2 / n_miss, or -1 when z_actual is NULL
 * (:579-581).  All arrays are host memory. */
EGS_API int egs_predict_host(int n_obs, int n_miss, int dts, const double* x_obs, const double* y_obs,
                     const double* z_obs, const double* x_miss, const double* y_miss,
                     const double* z_actual, const double* theta, double* z_miss, double* mspe);

/* Mean loss of efficiency (MLOE) and mean misspecification of the mean square
 * error (MMOM) of kriging with theta_est when theta_true holds, over n_miss
 * target locations (host arrays).  Replaces
 * LinearAlgebraMethods<T>::ExaGeoStatMLETileMLOEMMOM
 * (src/linear-algebra-solvers/LinearAlgebraMethods.cpp:802-1131) with the
 * dmloe-mmom codelet (src/runtime/starpu/concrete/dmloe-mmom-codelet.cpp:73-102);
 * univariate: the sill is sigma^2.  Both observed covariances are factored
 * once; each target costs four triangular solves and one L^T product. */
EGS_API int egs_mloe_mmom_host(int n_obs, int n_miss, int dts, const double* x_obs, const double* y_obs,
                               const double* x_miss, const double* y_miss, const double* theta_true,
                               const double* theta_est, double* mloe, double* mmom);

/* Inverse of the Fisher information of (sigma^2, beta, nu) at theta for n
 * host locations: A_jk = 1/2 tr(C^-1 dC/dtheta_j C^-1 dC/dtheta_k), written
 * column-major (3 x 3).  Replaces LinearAlgebraMethods<T>::ExaGeoStatFisherTile
 * (src/linear-algebra-solvers/LinearAlgebraMethods.cpp:1133-1306) with the
 * derivative kernels UnivariateMaternDdsigmaSquare / Dbeta / Dnu
 * (src/kernels/concrete/); d K_nu / d nu by Richardson-extrapolated central
 * differences (steps 1e-3, 5e-4) where the reference takes a forward one
 * (step 1e-9, BasselFunction.cpp:23-33).
 * Works in dense n x n buffers (about 8 n^2 doubles). */
EGS_API int egs_fisher_host(int n, int dts, const double* x, const double* y, const double* theta,
                            double* fisher_inverse);

/* ---- serving ------------------------------------------------------------ */

/* A request loop on one GPU: likelihood, fit and predict requests of any N are
 * queued, admitted while the sum of the admitted requests' HBM footprints
 * (egs_problem_footprint) stays within a budget and fewer than max_active run,
 * and executed concurrently, each on its own stream with its problem
 * (locations, observations, factor storage) resident for the whole request --
 * across every optimizer iteration of a fit.  Requests that arrive while others
 * run are admitted as slots and memory free up; the oldest waiting request
 * that fits goes first, and one that has waited longer than a few seconds
 * blocks younger ones until it fits.  Results of a request do not depend on
 * what else runs (all reductions have a fixed order).
 * The reference runs one request per process (ExaGeoStat<T>::ExaGeoStatDataModeling
 * / ExaGeoStatPrediction, src/api/ExaGeoStat.cpp:46-120); the request kinds map
 * to those calls. */
typedef struct egs_server egs_server;

#define EGS_REQ_LOGLIK 1   /* log-likelihood at theta (one ExaGeoStatMLETile evaluation) */
#define EGS_REQ_FIT 2      /* maximum-likelihood fit (ExaGeoStatDataModeling): BOBYQA from lb */
#define EGS_REQ_PREDICT 3  /* kriging at n_miss targets with theta (ExaGeoStatPrediction) */

typedef struct egs_request {
  int kind;            /* EGS_REQ_* */
  int n;               /* observed locations */
  int dts;             /* tile size (the reference's --dts) */
  int precision;       /* EGS_PRECISION_DOUBLE or EGS_PRECISION_MIXED */
  int band_tiles;      /* FP64 band of a mixed request */
  const double* x;     /* n locations and observations, copied at submission */
  const double* y;
  const double* z;
  double theta[3];     /* LOGLIK, PREDICT: (sigma^2, beta, nu) */
  double lb[3];        /* FIT: box bounds; the search starts at lb (Configurations.cpp:200) */
  double ub[3];
  double ftol_abs;     /* FIT: stop when an improvement is below this (10^-tol) */
  int max_evals;       /* FIT: evaluation limit (--max_mle_iterations) */
  int n_miss;          /* PREDICT: targets, copied at submission */
  const double* x_miss;
  const double* y_miss;
} egs_request;

typedef struct egs_result {
  int status;          /* EGS_OK, a potrf info (> 0) or an EGS_ERR_* code of this request */
  int kind;
  double loglik;       /* LOGLIK: value at theta; FIT: best value; PREDICT: unused */
  double theta[3];     /* FIT: fitted parameters; otherwise the request's theta */
  int evals;           /* device log-likelihood evaluations made for the request */
  double queue_ms;     /* submission -> admission */
  double latency_ms;   /* submission -> completion */
  long long footprint; /* HBM bytes reserved at admission */
  int precision_used;  /* the precision that produced the result: a mixed request whose
                          factorisation is not positive definite (FP32 off-band storage
                          of a very smooth kernel) is answered by the FP64 path */
  int fp64_reason;     /* why a mixed request was answered in FP64: EGS_FP64_REASON_* */
} egs_result;

#define EGS_FP64_REASON_NONE 0           /* answered in the requested precision */
#define EGS_FP64_REASON_PREDICTED 1      /* estimated too ill-conditioned for FP32 tiles: FP64 from the start */
#define EGS_FP64_REASON_AFTER_FAILURE 2  /* the mixed factorisation failed; re-run in FP64 */

/* Condition estimate of the Matern covariance of n locations at theta that the
 * serving loop uses to send a mixed-precision request to the FP64 path up front
 * (no counterpart in the reference, which has no mixed form): with h the mean
 * spacing sqrt(bounding-box area / n), *kappa = (1 + (pi beta / h)^2)^(nu + 1),
 * the ratio of the Matern spectral density at frequency 0 and at the grid's
 * Nyquist frequency pi / h.  Host arithmetic only. */
EGS_API int egs_mixed_conditioning_estimate(int n, const double* x, const double* y, const double* theta,
                                            double* kappa);

/* Start a server on `device` with hbm_budget bytes of admission budget and at
 * most max_active concurrently running requests (one host worker thread and
 * one stream each). */
EGS_API int egs_server_create(egs_server** out, int device, long long hbm_budget, int max_active);
/* Queue a request (its arrays are copied); *ticket identifies it.  A request
 * whose footprint alone exceeds the budget is refused with EGS_ERR_OOM. */
EGS_API int egs_server_submit(egs_server* s, const egs_request* r, long long* ticket);
/* Block until the request is done; copy its result (and, for PREDICT, n_miss
 * predictions into z_miss when it is not NULL) and release the ticket. */
EGS_API int egs_server_wait(egs_server* s, long long ticket, egs_result* out, double* z_miss);
/* Snapshot: queued and running requests, reserved bytes, the peak of running
 * requests and of reserved bytes so far, completed requests, and device
 * evaluations made. */
EGS_API int egs_server_stats(egs_server* s, int* queued, int* active, long long* reserved, int* peak_active,
                             long long* peak_reserved, long long* completed, long long* evals);
/* Finish every queued and running request, then stop the workers and free the server. */
EGS_API int egs_server_destroy(egs_server* s);

#ifdef __cplusplus
}
#endif
#endif /* EXAGEOSTAT_B200_H */
