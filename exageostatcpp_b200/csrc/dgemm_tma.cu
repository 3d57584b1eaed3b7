// FP64 tensor-core update  C := C - A * B^T  on the tile-major lower storage,
// fed by TMA, for sm_100a.
//
// This is the trailing syrk/gemm of the tiled Cholesky (the N^3/3 part of
// CHAMELEON_dpotrf_Tile, ChameleonDense.cpp:25-37) and, with K = 64, the
// updates inside the panel factorisation and the panel triangular solve.
//
// Geometry.  Every operand row is a *global* matrix row g in [0, Np); its data
// lives in tile row g / ts at local row g % ts.  A and B take their K columns
// from one tile column (a_tcol / b_tcol) starting at a local column offset; C is
// addressed element by element through (global row, global column) and
// elements of upper tiles are never written.  Because ts is a multiple of 64,
// a 16-row TMA box never straddles two tiles, so a 128 x 128 CTA tile may span
// tile boundaries and no MMA work is wasted when 128 does not divide ts.
//
// Pipeline.  Thread 0 issues 3-D TMA loads (rows x cols x tile-slot), running up to
// two stages ahead, into a 3-stage ring of 32-column 128B-swizzled shared-memory
// stages guarded by mbarriers; eight warps each own a 64 x 32 sub-tile and run
// mma.sync m16n8k16 .f64 (the FP64 tensor path of sm_100a).  The 16 rows of an
// MMA fragment are mapped to tile rows through fixed permutations chosen so
// that every fragment load is free of shared-memory bank conflicts under the
// 128-byte swizzle (A: 16-byte loads of row pairs; B: 8-byte loads).
//
// Every wait is bounded: a thread that polls longer than the limit records an
// error in *err and leaves; the host turns that into EGS_ERR_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cstdint>
#include "common.cuh"
#include "kernels.cuh"
#include "mbarrier.cuh"

namespace egs {

namespace gemm {
#ifndef EGS_GEMM_BK
#define EGS_GEMM_BK 32
#endif
#ifndef EGS_GEMM_STAGES
#define EGS_GEMM_STAGES 3
#endif
constexpr int BM = 128, BN = 128, BK = EGS_GEMM_BK, STAGES = EGS_GEMM_STAGES;
constexpr int CONSUMER_WARPS = 8;
constexpr int THREADS = CONSUMER_WARPS * 32;   // thread 0 also issues the TMA loads
constexpr int BOX_ROWS = 16;                          // 16 doubles = one 128-byte swizzle row
constexpr int BOX_BYTES = BOX_ROWS * BK * 8;          // 16 rows x BK columns
constexpr int A_STAGE_BYTES = (BM / BOX_ROWS) * BOX_BYTES;
constexpr int B_STAGE_BYTES = (BN / BOX_ROWS) * BOX_BYTES;
constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 2 * STAGES * 8 + 1024;
constexpr int GROUP = 8;                              // block-columns per raster group
}  // namespace gemm

__device__ __forceinline__ double lds_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ void lds_v2f64(uint32_t addr, double& a, double& b) {
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "r"(addr));
}
__device__ __forceinline__ void ldg_v2f64(const double* p, double& a, double& b) {
  asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "l"(p));
}
__device__ __forceinline__ void stg_v2f64(double* p, double a, double b) {
  asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(a), "d"(b) : "memory");
}
__device__ __forceinline__ void dmma_16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// MMA row g (0..7) of an A fragment -> tile row 2*perm[g] within a 16-row box;
// row g+8 -> the next row, so (a_2j, a_2j+1) is one 16-byte load.
__device__ __forceinline__ int perm_a(int g) { return ((g & 1) << 2) | (g >> 1); }
// MMA row r (0..15) of a B fragment (the n index) -> tile row within a 16-row box.
__device__ __forceinline__ int perm_b(int r) {
  return (r & 1) | (((r >> 2) & 1) << 1) | (((r >> 1) & 1) << 3) | (((r >> 3) & 1) << 2);
}

template <bool kBatched>
__device__ __forceinline__ const GemmDesc* locate_job(long long L, const GemmDesc& single, const GemmJobs& J,
                                                      long long& local) {
  if constexpr (!kBatched) {
    local = L;
    return &single;
  } else {
    int lo = 0, hi = J.njobs - 1;
    while (lo < hi) {  // last job with begin <= L
      const int mid = (lo + hi + 1) >> 1;
      if (J.begin[mid] <= L) lo = mid; else hi = mid - 1;
    }
    local = L - J.begin[lo];
    return J.jobs + lo;
  }
}

// Raster: groups of GROUP block-columns; inside a group, block-rows outer,
// block-columns inner, so a group's B panel stays in L2 while A streams once.
__device__ __forceinline__ bool decode_block(long long L, const GemmDesc& d, int& mb, int& nb) {
  for (int nb0 = 0; nb0 < d.NB; nb0 += gemm::GROUP) {
    const int ge = min(gemm::GROUP, d.NB - nb0);
    const int mstart = d.lower ? nb0 : 0;
    const long long cnt = (long long)ge * (d.MB - mstart);
    if (L < cnt) {
      mb = mstart + (int)(L / ge);
      nb = nb0 + (int)(L % ge);
      return true;
    }
    L -= cnt;
  }
  return false;
}

// Producer cursor: walks the same (block, k-step) sequence as the consumers,
// running up to STAGES-1 stages ahead of them.  The TMA (x, z) coordinates of
// the 2 x 8 boxes of a block depend only on the block, so they are computed
// once per block into shared memory; a stage then only adds its k offset.
struct Cursor {
  long long L;
  int kt;
  bool valid;
  const GemmDesc* d;
};

__device__ __forceinline__ void box_coords(int g0, int tcol, const GemmDesc& d, int2* out) {
#pragma unroll
  for (int b = 0; b < gemm::BM / gemm::BOX_ROWS; ++b) {
    const int g = g0 + b * gemm::BOX_ROWS;
    int x = d.ts, z = 0;  // fully out of bounds -> zero fill
    if (g < d.np) {
      const int ti = g / d.ts;
      x = g - ti * d.ts;
      z = (int)(d.tile_base + tile_slot(ti, tcol, d.nt));
    }
    out[b] = make_int2(x, z);
  }
}

template <bool kBatched>
__device__ __forceinline__ void cursor_seek(Cursor& c, const GemmDesc& single, const GemmJobs& J, long long total,
                                            int2* coords) {
  while (c.L < total) {
    long long local;
    const GemmDesc& d = *locate_job<kBatched>(c.L, single, J, local);
    int mb, nb;
    decode_block(local, d, mb, nb);
    if (!(d.lower && mb < nb)) {
      box_coords(d.a_row0 + mb * gemm::BM, d.a_tcol, d, coords);
      box_coords(d.b_row0 + nb * gemm::BN, d.b_tcol, d, coords + gemm::BM / gemm::BOX_ROWS);
      c.d = &d;
      c.valid = true;
      return;
    }
    c.L += gridDim.x;
  }
  c.valid = false;
}

__device__ __forceinline__ void issue_stage(const CUtensorMap* tmap, uint8_t* smem, uint64_t* full, uint32_t s,
                                            const Cursor& c, const int2* coords) {
  using namespace gemm;
  const GemmDesc& d = *c.d;
  mbar_expect_tx(&full[s], STAGE_BYTES);
  uint8_t* sa = smem + s * STAGE_BYTES;
  uint8_t* sb = sa + A_STAGE_BYTES;
  const int ya = d.a_col0 + c.kt * BK, yb = d.b_col0 + c.kt * BK;
#pragma unroll
  for (int b = 0; b < BM / BOX_ROWS; ++b) {
    const int2 xz = coords[b];
    tma_load_3d(sa + b * BOX_BYTES, tmap, &full[s], xz.x, ya, xz.y);
  }
#pragma unroll
  for (int b = 0; b < BN / BOX_ROWS; ++b) {
    const int2 xz = coords[BM / BOX_ROWS + b];
    tma_load_3d(sb + b * BOX_BYTES, tmap, &full[s], xz.x, yb, xz.y);
  }
}

template <bool kBatched>
__global__ void __launch_bounds__(gemm::THREADS, 1)
dgemm_update_kernel(const __grid_constant__ CUtensorMap tmap, double* __restrict__ tiles, const __grid_constant__ GemmDesc single,
                    GemmJobs J, int* __restrict__ err) {
  using namespace gemm;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned stage base (128B-swizzle atoms), kept as an offset into the
  // shared array so every access stays a shared-memory access.
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const uint32_t smem_s = smem_u32(smem);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool producer = threadIdx.x == 0;
  const long long total = kBatched ? J.total : single.total;
  if (producer) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmap) : "memory");
  }
  __syncthreads();

  // Producer state (meaningful in thread 0 only).
  __shared__ int2 coords[(BM + BN) / BOX_ROWS];
  Cursor cur;
  cur.L = blockIdx.x;
  cur.kt = 0;
  cur.valid = false;
  uint32_t issued = 0;
  bool alive = true;
  cur.d = &single;
  if (producer) cursor_seek<kBatched>(cur, single, J, total, coords);
  auto top_up = [&](uint32_t consumed) {
    // Keep up to STAGES-1 stages in flight ahead of the consumers.
    while (alive && cur.valid && issued < consumed + STAGES - 1) {
      const uint32_t s = issued % STAGES, ph = (issued / STAGES) & 1;
      if (!mbar_wait(&empty[s], ph ^ 1, err)) {
        alive = false;
        break;
      }
      issue_stage(&tmap, smem, full, s, cur, coords);
      ++issued;
      if (++cur.kt == cur.d->K / BK) {
        cur.kt = 0;
        cur.L += gridDim.x;
        cursor_seek<kBatched>(cur, single, J, total, coords);
      }
    }
  };

  const int g = lane >> 2, t = lane & 3;
  const int wm = warp & 1, wn = warp >> 1;  // warp sub-tile: rows wm*64.., cols wn*32..
  const int pa = perm_a(g);
  const int row_in_box = 2 * pa;  // accumulator rows row_in_box, row_in_box + 1
  // Byte offsets (inside one 16-row box) of this thread's fragment elements.
  uint32_t aoff[4], boff[2][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int k = t + 4 * j;
    aoff[j] = k * 128 + ((pa ^ (k & 7)) << 4);
  }
#pragma unroll
  for (int sN = 0; sN < 2; ++sN) {
    const int fb = perm_b(g + 8 * sN);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = t + 4 * i;
      boff[sN][i] = k * 128 + (((fb >> 1) ^ (k & 7)) << 4) + ((fb & 1) << 3);
    }
  }

  uint32_t it = 0;
  bool ok = true;
  for (long long L = blockIdx.x; L < total && ok; L += gridDim.x) {
    long long local;
    const GemmDesc& d = *locate_job<kBatched>(L, single, J, local);
    int mb, nb;
    decode_block(local, d, mb, nb);
    if (d.lower && mb < nb) continue;
    const int ksteps = d.K / BK;
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[mi][ni][q] = 0.0;

    for (int kt = 0; kt < ksteps; ++kt, ++it) {
      if (producer) top_up(it);
      __syncwarp();
      const uint32_t s = it % STAGES, ph = (it / STAGES) & 1;
      if (!mbar_wait(&full[s], ph, err)) {
        ok = false;
        break;
      }
      __syncwarp();
      const uint32_t sa = smem_s + s * STAGE_BYTES;
      const uint32_t sb = sa + A_STAGE_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint32_t koff = kk * 16 * 128;  // 16 k-rows of 128 bytes per MMA k-step
        double bf[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          const uint32_t box = sb + (wn * 2 + (ni >> 1)) * BOX_BYTES + koff;
#pragma unroll
          for (int i = 0; i < 4; ++i) bf[ni][i] = lds_f64(box + boff[ni & 1][i]);
        }
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          const uint32_t box = sa + (wm * 4 + mi) * BOX_BYTES + koff;
          double af[8];
#pragma unroll
          for (int j = 0; j < 4; ++j) lds_v2f64(box + aoff[j], af[2 * j], af[2 * j + 1]);
#pragma unroll
          for (int ni = 0; ni < 4; ++ni) dmma_16816(acc[mi][ni], af, bf[ni]);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (!ok) break;

    // Epilogue: C -= acc; element pairs (row, row+1) are contiguous in a column.
    // Per n8 block the eight 16-byte loads are issued before any store, so a
    // thread pays one memory round trip per block instead of one per pair.
    const int ts = d.ts;
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      double* ptr[2][4];
      double cv[2][4][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nl = nb * BN + wn * 32 + (ni >> 1) * 16 + perm_b(2 * t + 8 * (ni & 1)) + h;
        const int gj = d.c_col0 + nl;
        const int tj = gj / ts, lc = gj - tj * ts;
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) {
          const int ml = mb * BM + wm * 64 + mi * 16 + row_in_box;
          const int gi = d.c_row0 + ml;
          const int ti = gi / ts, lr = gi - ti * ts;
          const bool ok_el = nl < d.N && ml < d.M && ti >= tj && (d.c_mode == 0 || ti - tj <= d.c_band);
          const long long cslot = d.c_mode == 0 ? d.tile_base + tile_slot(ti, tj, d.nt)
                                                : (long long)(d.c_tile_off + tj) * (d.c_band + 1) + (ti - tj);
          ptr[h][mi] = ok_el ? tiles + cslot * (long long)ts * ts + (long long)lc * ts + lr : nullptr;
          if (ok_el) ldg_v2f64(ptr[h][mi], cv[h][mi][0], cv[h][mi][1]);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
          if (ptr[h][mi])
            stg_v2f64(ptr[h][mi], cv[h][mi][0] - acc[mi][ni][h], cv[h][mi][1] - acc[mi][ni][2 + h]);
    }
  }
  // Drain: every stage this CTA issued must have landed before it exits.
  if (producer) {
    for (uint32_t j = (issued > (uint32_t)STAGES ? issued - STAGES : 0); j < issued; ++j)
      mbar_wait(&full[j % STAGES], (j / STAGES) & 1, err);
  }
}

// One-time lookups below use function-local statics, whose initialisation is
// thread-safe: problems may be created from several host threads at once.
int tensor_map_encoder(void** fn_out) {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  if (!fn) {
    set_last_error("cuTensorMapEncodeTiled unavailable", "tensor_map_encoder");
    return EGS_ERR_CUDA;
  }
  *fn_out = reinterpret_cast<void*>(fn);
  return EGS_OK;
}

int gemm_init_tensor_map(void* tmap_storage, double* tiles, int ts, long long ntiles) {
  void* fn = nullptr;
  if (tensor_map_encoder(&fn) != EGS_OK) return EGS_ERR_CUDA;
  if (ts % 64 != 0 || ((uintptr_t)tiles & 15) != 0) return EGS_ERR_INVALID;
  cuuint64_t dims[3] = {(cuuint64_t)ts, (cuuint64_t)ts, (cuuint64_t)ntiles};
  cuuint64_t strides[2] = {(cuuint64_t)ts * 8, (cuuint64_t)ts * ts * 8};
  cuuint32_t box[3] = {gemm::BOX_ROWS, gemm::BK, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  CUresult r = encode(reinterpret_cast<CUtensorMap*>(tmap_storage), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, tiles,
                        dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed", "gemm_init_tensor_map");
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

int gemm_num_sms() {
  static const int sms = []() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  return sms;
}

static void set_gemm_smem_attributes() {
  static std::once_flag done[64];
  once_per_device(done, []() {
    cudaFuncSetAttribute(dgemm_update_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm::SMEM_BYTES);
    cudaFuncSetAttribute(dgemm_update_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm::SMEM_BYTES);
  });
}

void finish_desc(GemmDesc& d) {
  using namespace gemm;
  d.MB = (d.M + BM - 1) / BM;
  d.NB = (d.N + BN - 1) / BN;
  long long total = 0;
  for (int nb0 = 0; nb0 < d.NB; nb0 += GROUP) {
    const int ge = (d.NB - nb0) < GROUP ? (d.NB - nb0) : GROUP;
    total += (long long)ge * (d.MB - (d.lower ? nb0 : 0));
  }
  d.total = total;
}

static int launch_desc(const void* tmap, double* tiles, GemmDesc& d, int* err, cudaStream_t st, int max_ctas = 0) {
  using namespace gemm;
  if (d.M <= 0 || d.N <= 0 || d.K <= 0) return EGS_OK;
  if (d.K % BK != 0) return EGS_ERR_INVALID;
  finish_desc(d);
  const long long total = d.total;
  set_gemm_smem_attributes();
  const long long cap = (max_ctas > 0 && max_ctas < gemm_num_sms()) ? max_ctas : gemm_num_sms();
  const long long grid = total < cap ? total : cap;
  GemmJobs none{nullptr, nullptr, 0, 0};
  dgemm_update_kernel<false><<<(unsigned)grid, THREADS, SMEM_BYTES, st>>>(
      *reinterpret_cast<const CUtensorMap*>(tmap), tiles, d, none, err);
  return launch_status("dgemm_update_kernel");
}

// Trailing update of step k: C(i, j) -= L(i, k) L(j, k)^T for all k < j <= i.
int launch_gemm_trailing(const void* tmap, double* tiles, int ts, int nt, int k, int* err, cudaStream_t st) {
  GemmDesc d{};
  d.ts = ts;
  d.nt = nt;
  d.np = nt * ts;
  const int r0 = (k + 1) * ts;
  d.M = d.N = d.np - r0;
  d.K = ts;
  d.a_row0 = d.b_row0 = d.c_row0 = d.c_col0 = r0;
  d.a_col0 = d.b_col0 = 0;
  d.a_tcol = d.b_tcol = k;
  d.lower = 1;
  return launch_desc(tmap, tiles, d, err, st);
}

// General form used by the panel factorisation (see kernels.cuh).
int launch_gemm_rows(const void* tmap, double* tiles, int ts, int nt, int M, int N, int K, int a_row0,
                     int a_col0, int a_tcol, int b_row0, int b_col0, int b_tcol, int c_row0, int c_col0,
                     int lower, int* err, cudaStream_t st, int max_ctas) {
  GemmDesc d{};
  d.ts = ts;
  d.nt = nt;
  d.np = nt * ts;
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
  return launch_desc(tmap, tiles, d, err, st, max_ctas);
}

}  // namespace egs

namespace egs {

// One launch over many jobs (one per problem of a batch); jobs and begin live in
// device memory, begin[j] = number of blocks of jobs 0..j-1 (finish_desc totals).
int launch_gemm_batched(const void* tmap, double* tiles, const GemmDesc* jobs, const long long* begin, int njobs,
                        long long total, int* err, cudaStream_t st) {
  using namespace gemm;
  if (njobs <= 0 || total <= 0) return EGS_OK;
  set_gemm_smem_attributes();
  const long long grid = total < gemm_num_sms() ? total : gemm_num_sms();
  GemmDesc none{};
  GemmJobs J{jobs, begin, njobs, total};
  dgemm_update_kernel<true><<<(unsigned)grid, THREADS, SMEM_BYTES, st>>>(
      *reinterpret_cast<const CUtensorMap*>(tmap), tiles, none, J, err);
  return launch_status("dgemm_update_kernel (jobs)");
}

}  // namespace egs
