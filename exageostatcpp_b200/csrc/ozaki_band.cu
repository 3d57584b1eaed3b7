// FP64-class band update of the mixed-precision factorisation on the integer
// tensor cores (tcgen05 kind::i8, sm_100a): the Ozaki splitting scheme.
//
// At step k every band target tile (i, j), k < j <= i <= j + band, receives
// C_ij -= L_ik L_jk^T in FP64 storage.  The FP64 panel rows are split, after a
// power-of-two row scaling 2^-e_r (|L_r.| < 2^e_r), into S signed 7-bit
// slices:
//     L_rc = 2^e_r * sum_{p=1..S} a_p(r, c) 2^(-7p),   a_p in [-127, 127],
// exact up to 2^(-7S) of the row maximum (S = 7: 2^-49).  Then
//     (L_i L_j^T)(r, c) = 2^(e_r + e_c) * sum_{d=2..S+1} 2^(-7d) G_d(r, c),
//     G_d = sum_{p+q=d} A_p B_q^T,
// where every G_d is an exact integer dot product: the int8 MMAs accumulate
// in 32-bit integers without rounding (|G_d| <= S * K * 127^2 < 2^31 for
// K <= 16384), so the only roundings are the final FP64 combination and the
// dropped terms p + q > S + 1 (each below 2^(-7(S+1)) of the row maxima).
// This follows Ozaki, Ogita, Oishi and Rump, "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and
// its applications", Numer. Algorithms 59 (2012), with the integer-slice
// variant of Ootomo, Ozaki and Yokota (2024).
//
// The band update uses all S = 7 slices; the off-band panel solve (FP32-stored
// rows times rows of L_kk^-1, written back in FP32) uses the first six, 2^-42
// of the row maxima, which is 21 slice products instead of 28.
//
// Kernel (one CTA per SM, persistent over 128 x 64 output tiles; 320 threads;
// NS = slices used):
//   warp 0    TMA producer: per 64-wide K stage the NS slices of the tile's 128
//             A rows and 64 B rows (64-byte swizzle), a ring of 2 (NS = 7) or
//             3 (NS = 6) stages;
//   warp 1    allocates 512 TMEM columns -- NS groups of 64 int32 columns, one
//             per d, in order of d -- and issues the NS(NS+1)/2 slice products
//             of a 32-wide K step from one thread as ten (NS = 7) or nine
//             (NS = 6) MMAs (the products of one A slice with up to four
//             consecutive B slices form one MMA of N <= 256 over consecutive
//             groups), the first K step with accumulate = 0;
//   warps 2-9 epilogue: warp w reads TMEM lane quarter w % 4 and 32 of the 64
//             columns, combines the groups exactly in 64-bit integers and then
//             in FP64 (two roundings), scales by 2^(e_r + e_c) and subtracts
//             from the FP64 band tile.
// The accumulator is single-buffered (NS groups fill TMEM); the epilogue
// releases it as soon as its last TMEM load is done, before the C update.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cstdint>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "kernels.cuh"
#include "mbarrier.cuh"
#include "panel_scales.cuh"

namespace egs {

namespace oz {
constexpr int S = kOzSlices;               // slices per operand stored (and used by the band update)
constexpr int BM = 128, BN = 64, BK = 64;  // BK int8 = one 64-byte swizzle row
constexpr int BOX_ROWS = 64;
constexpr int A_SLICE = BM * BK;           // 8 KB
constexpr int B_SLICE = BN * BK;           // 4 KB
constexpr int EPI_WARPS = 8;
constexpr int THREADS = 64 + 32 * EPI_WARPS;
constexpr uint32_t TMEM_COLS = 512;
constexpr int kMaxSmem = 232448;
// A kernel that uses the first NS slices of each operand: ring stages of NS
// (A, B) slice pairs, as many as fit up to three, and NS int32 groups of BN
// columns in tensor memory (groups d = 2 .. NS + 1).
template <int NS>
struct Cfg {
  static constexpr int STAGE_BYTES = NS * (A_SLICE + B_SLICE);
  static constexpr int STAGES = 1024 + 3 * STAGE_BYTES + 256 <= kMaxSmem ? 3 : 2;
  static constexpr int SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + 256;
  static_assert(NS >= 1 && NS <= S, "slices stored per operand");
  static_assert(NS * BN <= (int)TMEM_COLS, "groups fit in tensor memory");
  static_assert(SMEM_BYTES <= kMaxSmem, "shared memory per CTA");
};
// Instruction descriptor of kind::i8: D S32 (bits 4-5 = 2), A and B signed 8-bit
// (bits 7-9 = 1, bits 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
}  // namespace oz

// ---------------------------------------------------------------------------
// Slicing of the solved panel
// ---------------------------------------------------------------------------

// Row scales and int8 slices -- and, with kSplit, the FP16 split scales and
// hi/lo parts -- of ntiles column-major tiles (tiles0 + t ts^2, global tile row
// row_tile0 + t), in one kernel: one CTA per 64-row strip of a tile reads the
// strip once for its row maxima, then again in 64 x 64 blocks, transposed
// through shared memory into the row-major (K contiguous) outputs
// slices[p][row][c] and Ph / Pl[row][c].
template <typename T, bool kSplit, int NP>
__global__ void __launch_bounds__(256, 2)
panel_prepare_kernel(const T* __restrict__ tiles0, int ts, int row_tile0, double* __restrict__ oz_scale,
                     int8_t* __restrict__ slices, long long slice_stride, float* __restrict__ inv_scale,
                     __half* __restrict__ Ph, __half* __restrict__ Pl) {
  __shared__ double Sm[64][65];
  __shared__ double red[4][64];
  __shared__ double s_oz[64], s_f16[64];
  const int t = blockIdx.y;
  const int r0 = blockIdx.x * 64;
  const T* src = tiles0 + (long long)t * ts * ts;
  const long long grow0 = (long long)(row_tile0 + t) * ts + r0;
  {
    const int rl = threadIdx.x & 63, g = threadIdx.x >> 6;
    const T* col = src + r0 + rl;
    double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;  // ts is a multiple of 64
#pragma unroll 4
    for (int c = g; c < ts; c += 16) {
      m0 = fmax(m0, fabs((double)col[(long long)c * ts]));
      m1 = fmax(m1, fabs((double)col[(long long)(c + 4) * ts]));
      m2 = fmax(m2, fabs((double)col[(long long)(c + 8) * ts]));
      m3 = fmax(m3, fabs((double)col[(long long)(c + 12) * ts]));
    }
    red[g][rl] = fmax(fmax(m0, m1), fmax(m2, m3));
    __syncthreads();
    if (g == 0) {
      const double m = fmax(fmax(red[0][rl], red[1][rl]), fmax(red[2][rl], red[3][rl]));
      const double so = oz_row_scale(m);
      oz_scale[grow0 + rl] = so;
      s_oz[rl] = (so > 0.0) ? 1.0 / so : 0.0;  // exact: a power of two
      if constexpr (kSplit) {
        const float inv = f16_row_inv_scale(m);
        inv_scale[grow0 + rl] = inv;
        s_f16[rl] = (inv > 0.0f) ? 1.0 / (double)inv : 0.0;  // exact: a power of two
      }
    }
  }
  // Pass 2, 64 x 64 blocks; the next block's loads are issued before the
  // current block is split.  Without kSplit every thread slices 16 columns of
  // one row; with kSplit warps 0-3 slice and warps 4-7 split to FP16, 2 x 16
  // columns of one row per thread, so neither needs both sets of registers.
  T w[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int e = q * 256 + threadIdx.x;
    w[q] = src[(long long)(e >> 6) * ts + r0 + (e & 63)];
  }
  for (int c0 = 0; c0 < ts; c0 += 64) {
    __syncthreads();  // Sm free; the scales are visible
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = q * 256 + threadIdx.x;
      Sm[e & 63][e >> 6] = (double)w[q];
    }
    if (c0 + 64 < ts) {
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int e = q * 256 + threadIdx.x;
        w[q] = src[(long long)(c0 + 64 + (e >> 6)) * ts + r0 + (e & 63)];
      }
    }
    __syncthreads();
    if constexpr (!kSplit) {
      const int r = threadIdx.x >> 2, cq = (threadIdx.x & 3) * 16;
      const double io = s_oz[r];
      double v[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] = Sm[r][cq + c] * io;  // |v| < 1
      oz_emit_slices<NP>(v, slices + (grow0 + r) * ts + c0 + cq, slice_stride);
    } else {
      const int tt = threadIdx.x & 127, r = tt >> 1;
      const bool to_f16 = threadIdx.x >= 128;  // warp-uniform
      const double sc = to_f16 ? s_f16[r] : s_oz[r];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cq = (tt & 1) * 32 + h * 16;
        const long long off = (grow0 + r) * ts + c0 + cq;
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = Sm[r][cq + c] * sc;
        if (to_f16)
          f16_emit_split(v, Ph + off, Pl + off);
        else
          oz_emit_slices<NP>(v, slices + off, slice_stride);  // |v| < 1
      }
    }
  }
}

// Row scale of ts rows stored row by row (row r at src + r ts), written to
// scale[row0 + r]: one warp per row.
__global__ void __launch_bounds__(256)
ozaki_rowscale_rm_kernel(const double* __restrict__ src, int ts, long long row0, double* __restrict__ scale) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * 8 + warp;
  if (r >= ts) return;
  const double* row = src + (long long)r * ts;
  double m = 0.0;
  for (int c = lane; c < ts; c += 32) m = fmax(m, fabs(row[c]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) scale[row0 + r] = oz_row_scale(m);
}

// The first NP slices of rows stored row by row (row r at src + r ts) into
// slice rows row0 + r.
template <int NP>
__global__ void __launch_bounds__(256)
ozaki_slice_rm_kernel(const double* __restrict__ src, int ts, long long row0, const double* __restrict__ scale,
                      int8_t* __restrict__ slices, long long slice_stride) {
  const long long idx = (long long)blockIdx.x * 256 + threadIdx.x;  // one 16-column chunk
  const int chunks = ts / 16;
  const int r = (int)(idx / chunks), cq = (int)(idx % chunks) * 16;
  if (r >= ts) return;
  const double sc = scale[row0 + r];
  const double inv = (sc > 0.0) ? 1.0 / sc : 0.0;  // exact: a power of two
  const double* row = src + (long long)r * ts + cq;
  double v[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) v[c] = row[c] * inv;
  oz_emit_slices<NP>(v, slices + (row0 + r) * ts + cq, slice_stride);
}

// ---------------------------------------------------------------------------
// tcgen05 helpers (kind::i8, 64-byte swizzle)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;   // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;            // descriptor version
  d |= (uint64_t)4 << 61;            // SWIZZLE_64B
  return d;
}
// One int8 MMA.  COLLECT selects the use of the tensor core's A collector
// buffer: 0 reads A from shared memory only, 1 reads it and keeps it in the
// collector (fill), 2 takes A from the collector and keeps it (use), 3 takes
// it from the collector and releases it (lastuse).  Consecutive MMAs with the
// same A slice read it from shared memory once.
template <int COLLECT>
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  if constexpr (COLLECT == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (COLLECT == 1) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::fill [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else if constexpr (COLLECT == 2) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::use [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8.collector::a::lastuse [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}
__device__ __forceinline__ void oz_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void oz_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void oz_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void oz_tma_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
// 32 consecutive int32 columns of this warp's TMEM lane quarter, one load and
// one wait.
__device__ __forceinline__ void tmem_ld32_i32(uint32_t taddr, int (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = (int)r[i];
}

// Targets of one step: target t = (i, j, first work item, diagonal flag);
// items of an off-diagonal target: MB x NB tiles (row block fastest); of a
// diagonal target: the tiles touching the lower triangle, nb <= 2 mb + 1,
// enumerated row block by row block.
// mode 0 (band update): targets (i, j): C_ij -= A_i A_j^T into the band pool.
// mode 1 (panel solve through the inverse): targets (i, -): W[i - k] =
// A_i B^T, B = rows b_row_base .. + ts of the slice storage (rows of L_kk^-1).
struct OzStep {
  const int4* targets;
  int ntargets;
  long long total;
  int ts, band;
  int mode, k;
  long long b_row_base;
  double* band_pool;
  double* w_out;
  const double* scale;   // per slice row
  int* err;
};

__device__ __forceinline__ void oz_decode(const OzStep& P, long long L, int& i, int& j, int& mb, int& nb) {
  int lo = 0, hi = P.ntargets - 1;
  while (lo < hi) {  // last target whose first item <= L
    const int mid = (lo + hi + 1) >> 1;
    if ((long long)P.targets[mid].z <= L) lo = mid; else hi = mid - 1;
  }
  const int4 t = P.targets[lo];
  i = t.x;
  j = t.y;
  const int l = (int)(L - t.z);
  const int MB = P.ts / oz::BM;
  if (t.w == 0) {
    mb = l % MB;
    nb = l / MB;
  } else {
    int m = 0;
    while ((m + 1) * (m + 1) + (m + 1) <= l) ++m;  // items before row block m: m^2 + m
    mb = m;
    nb = l - (m * m + m);
  }
}

template <int NS>
__global__ void __launch_bounds__(oz::THREADS, 1)
ozaki_band_kernel(const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ OzStep P) {
  using namespace oz;
  constexpr int STAGES = Cfg<NS>::STAGES, STAGE_BYTES = Cfg<NS>::STAGE_BYTES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 1);
  __shared__ int bail_flag;
  volatile int& bail = bail_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, EPI_WARPS);
    bail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  oz_fence_before();
  __syncthreads();
  oz_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int ksteps = P.ts / BK;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (long long L = blockIdx.x; L < P.total && !bail; L += gridDim.x) {
        int i, j, mb, nb;
        oz_decode(P, L, i, j, mb, nb);
        const int arow = i * P.ts + mb * BM;
        const int brow = P.mode == 0 ? j * P.ts + nb * BN : (int)(P.b_row_base + nb * BN);
        for (int kt = 0; kt < ksteps; ++kt, ++it) {
          const uint32_t s = it % STAGES;
          if (it >= (uint32_t)STAGES && !mbar_wait(&empty[s], ((it / STAGES) & 1) ^ 1, P.err)) {
            bail = 1;
            break;
          }
          uint8_t* st = smem + s * STAGE_BYTES;
          mbar_expect_tx(&full[s], STAGE_BYTES);
          const int x = kt * BK;
#pragma unroll 1
          for (int p = 0; p < NS; ++p) {
            oz_tma_3d(st + p * A_SLICE, &tm_s, &full[s], x, arow, p);
            oz_tma_3d(st + p * A_SLICE + BOX_ROWS * BK, &tm_s, &full[s], x, arow + BOX_ROWS, p);
            oz_tma_3d(st + NS * A_SLICE + p * B_SLICE, &tm_s, &full[s], x, brow, p);
          }
        }
      }
      const uint32_t first = it > (uint32_t)STAGES ? it - STAGES : 0;
      for (uint32_t q = first; q < it; ++q) mbar_wait(&full[q % STAGES], (q / STAGES) & 1, P.err);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      uint32_t it = 0, tcount = 0;
      bool ok = true;
      for (long long L = blockIdx.x; L < P.total && ok && !bail; L += gridDim.x, ++tcount) {
        if (tcount >= 1 && !mbar_wait(acc_empty, (tcount - 1) & 1, P.err)) {
          ok = false;
          break;
        }
        oz_fence_after();
        for (int kt = 0; kt < ksteps; ++kt, ++it) {
          const uint32_t s = it % STAGES;
          if (!mbar_wait(&full[s], (it / STAGES) & 1, P.err)) {
            ok = false;
            break;
          }
          oz_fence_after();
          const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t sb = sa + NS * A_SLICE;
          // A slice p against B slices q = 1 .. NS+1-p: group d = p + q sits at
          // TMEM columns (d - 2) BN and the B slices are stacked in shared
          // memory, so the products of A_p with B_q .. B_q+m-1 are one MMA of
          // N = m BN into the columns of groups p+q .. p+q+m-1 (N <= 256: at
          // most four slices a time).  Ten MMAs per 32-wide K step for seven
          // slices, nine for six; an A slice used by two of them is read once
          // through the collector buffer.
#pragma unroll
          for (int kk = 0; kk < BK / 32; ++kk) {
#pragma unroll
            for (int p = 1; p <= NS; ++p) {
              const uint64_t ad = sdesc_sw64(sa + (p - 1) * A_SLICE + kk * 32);
              const uint32_t acc = (kt > 0 || kk > 0 || p > 1) ? 1u : 0u;  // p = 1 opens every group
              constexpr int kMaxSlices = 256 / BN;
              const int qmax = NS + 1 - p;
              const int nmma = (qmax + kMaxSlices - 1) / kMaxSlices;
#pragma unroll
              for (int q0 = 1; q0 <= qmax; q0 += kMaxSlices) {
                const int m = (qmax - q0 + 1) < kMaxSlices ? (qmax - q0 + 1) : kMaxSlices;
                const uint32_t dcol = tmem_base + (uint32_t)((p + q0 - 2) * BN);
                const uint64_t bd = sdesc_sw64(sb + (q0 - 1) * B_SLICE + kk * 32);
                const uint32_t id = idesc_i8(m * BN);
                if (nmma == 1) umma_i8<0>(dcol, ad, bd, id, acc);
                else if (q0 == 1) umma_i8<1>(dcol, ad, bd, id, acc);
                else umma_i8<3>(dcol, ad, bd, id, acc);
              }
            }
          }
          oz_commit(&empty[s]);
        }
        if (!ok) break;
        oz_commit(acc_full);
      }
      if (!ok) bail = 1;
    }
  } else {
    // epilogue warps 2..9: lane quarter warp % 4, columns [half * 32, half * 32 + 32)
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    const uint32_t tl = tmem_base + ((uint32_t)(quarter * 32) << 16) + half * 32;
    uint32_t tcount = 0;
    bool ok = true;
    for (long long L = blockIdx.x; L < P.total && ok; L += gridDim.x, ++tcount) {
      int i, j, mb, nb;
      oz_decode(P, L, i, j, mb, nb);
      const int r = mb * BM + quarter * 32 + lane;
      const int c0 = nb * BN + half * 32;
      double* cp = nullptr;  // this thread's row of the C block, column c0
      if (P.mode == 0) {
        cp = P.band_pool + ((long long)j * (P.band + 1) + (i - j)) * P.ts * P.ts + (long long)c0 * P.ts + r;
        // the warp's 32 x 32 block of C into L2 while the tile's MMAs run: lane l
        // fetches the two 128-byte lines of column c0 + l
        const double* col = cp - lane + (long long)lane * P.ts;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(col));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(col + 16));
      }
      int w = 1;
      if (lane == 0) w = mbar_wait(acc_full, tcount & 1, P.err) ? 1 : 0;
      w = __shfl_sync(0xffffffffu, w, 0);
      if (!w) {
        ok = false;
        break;
      }
      oz_fence_after();
      // sum_d 2^(-7d) G_d with the groups combined exactly in 64-bit integers
      // first (group g holds d = g + 2):
      //   H = G_2 2^21 + G_3 2^14 + G_4 2^7 + G_5,   t = G_6 2^7 + G_7,
      //   value = H 2^-35 + t 2^-49 (+ G_8 2^-56 with seven slices),
      // |H| < 2^50 for K <= 16384, so H and t convert to FP64 exactly and the
      // value takes at most two roundings; the tensor memory goes back to the
      // MMAs right after the last group's load.
      static_assert(NS == 6 || NS == 7, "the exact grouping below is written for six or seven slices");
      double acc[32];
      {
        long long h[32];
        int v[32];
        tmem_ld32_i32(tl, v);
#pragma unroll
        for (int c = 0; c < 32; ++c) h[c] = v[c];
#pragma unroll 1
        for (int g = 1; g < 4; ++g) {
          tmem_ld32_i32(tl + (uint32_t)(g * BN), v);
#pragma unroll
          for (int c = 0; c < 32; ++c) h[c] = h[c] * 128 + v[c];
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = (double)h[c] * 0x1p-35;
      }
      {
        int v4[32], v5[32];
        tmem_ld32_i32(tl + (uint32_t)(4 * BN), v4);
        tmem_ld32_i32(tl + (uint32_t)(5 * BN), v5);
        if constexpr (NS == 6) {
          oz_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(acc_empty);
        }
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = fma((double)((long long)v4[c] * 128 + v5[c]), 0x1p-49, acc[c]);
      }
      if constexpr (NS == 7) {
        int v[32];
        tmem_ld32_i32(tl + (uint32_t)(6 * BN), v);
        oz_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acc_empty);
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = fma((double)v[c], 0x1p-56, acc[c]);
      }
      const double sr = P.scale[(long long)i * P.ts + r];
      if (P.mode == 0) {
        // all 32 loads of C first: a store may alias a later element as far as
        // the compiler knows, so interleaved read-modify-writes would serialise
        // 32 memory round trips per tile
        const double* sc = P.scale + (long long)j * P.ts + c0;
        const bool diag = (i == j);
        double cv[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) cv[c] = (!diag || r >= c0 + c) ? cp[(long long)c * P.ts] : 0.0;
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (!diag || r >= c0 + c) cp[(long long)c * P.ts] = cv[c] - acc[c] * (sr * __ldg(sc + c));
      } else {
        const double* sc = P.scale + P.b_row_base + c0;
        double* cp = P.w_out + (long long)(i - P.k) * P.ts * P.ts + (long long)c0 * P.ts + r;
#pragma unroll
        for (int c = 0; c < 32; ++c) cp[(long long)c * P.ts] = acc[c] * (sr * __ldg(sc + c));
      }
    }
    if (!ok) bail = 1;
  }
  oz_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    oz_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int ozaki_slices() { return oz::S; }

// Slice storage: S planes of rows x ts int8 (rows = every global panel row).
int ozaki_tensor_map(void* storage, const int8_t* slices, int ts, long long rows) {
  void* fn = nullptr;
  if (tensor_map_encoder(&fn) != EGS_OK) return EGS_ERR_CUDA;
  if (ts % oz::BK != 0 || ((uintptr_t)slices & 15) != 0) return EGS_ERR_INVALID;
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  cuuint64_t dims[3] = {(cuuint64_t)ts, (cuuint64_t)rows, (cuuint64_t)oz::S};
  cuuint64_t strides[2] = {(cuuint64_t)ts, (cuuint64_t)ts * (cuuint64_t)rows};
  cuuint32_t box[3] = {oz::BK, oz::BOX_ROWS, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(reinterpret_cast<CUtensorMap*>(storage), CU_TENSOR_MAP_DATA_TYPE_UINT8, 3,
                      const_cast<int8_t*>(slices), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed", "ozaki_tensor_map");
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

// Panel tiles W[t0 .. t0+ntiles) = global tile rows row_tile0 + t0 .. (column-major FP64).
void launch_ozaki_slice(const double* W, int ts, int t0, int ntiles, int row_tile0, double* scale, int8_t* slices,
                        long long rows, cudaStream_t st) {
  if (ntiles <= 0) return;
  panel_prepare_kernel<double, false, kOzSlices><<<dim3(ts / 64, ntiles), 256, 0, st>>>(
      W + (long long)t0 * ts * ts, ts, row_tile0 + t0, scale, slices, rows * (long long)ts, nullptr, nullptr, nullptr);
}

// As launch_ozaki_slice, plus the FP16 split (inv_scale, Ph, Pl) of the same
// rows for the split-FP16 update, from one read of the panel.
void launch_panel_prepare(const double* W, int ts, int t0, int ntiles, int row_tile0, double* oz_scale,
                          int8_t* slices, long long rows, float* inv_scale, __half* Ph, __half* Pl, cudaStream_t st) {
  if (ntiles <= 0) return;
  panel_prepare_kernel<double, true, kOzSlices><<<dim3(ts / 64, ntiles), 256, 0, st>>>(
      W + (long long)t0 * ts * ts, ts, row_tile0 + t0, oz_scale, slices, rows * (long long)ts, inv_scale, Ph, Pl);
}

// Contiguous FP32 column-major tiles (global tile rows row_tile0 ..).
void launch_ozaki_slice_f32(const float* tiles0, int ts, int ntiles, int row_tile0, double* scale, int8_t* slices,
                            long long rows, cudaStream_t st) {
  if (ntiles <= 0) return;
  panel_prepare_kernel<float, false, kOzPanelSlices><<<dim3(ts / 64, ntiles), 256, 0, st>>>(
      tiles0, ts, row_tile0, scale, slices, rows * (long long)ts, nullptr, nullptr, nullptr);
}

// ts rows stored row by row at src into slice rows row0 .. row0 + ts.
void launch_ozaki_slice_rows(const double* src, int ts, long long row0, double* scale, int8_t* slices,
                             long long rows, cudaStream_t st) {
  ozaki_rowscale_rm_kernel<<<(ts + 7) / 8, 256, 0, st>>>(src, ts, row0, scale);
  const long long chunks = (long long)ts * (ts / 16);
  ozaki_slice_rm_kernel<kOzPanelSlices><<<(unsigned)((chunks + 255) / 256), 256, 0, st>>>(src, ts, row0, scale, slices,
                                                                          rows * (long long)ts);
}

// Target table of step k: band targets (i, j), k < j <= i <= min(nt-1, j+band),
// column by column; returns the total work items.
long long ozaki_targets(int ts, int nt, int band, int k, std::vector<int4>& out) {
  const int MB = ts / oz::BM, NB = ts / oz::BN;
  long long items = 0;
  for (int j = k + 1; j < nt; ++j) {
    for (int i = j; i <= j + band && i < nt; ++i) {
      out.push_back(make_int4(i, j, (int)items, i == j ? 1 : 0));
      if (i == j) {
        for (int m = 0; m < MB; ++m) items += std::min(NB, 2 * m + 2);
      } else {
        items += (long long)MB * NB;
      }
    }
  }
  return items;
}

template <int NS>
static int launch_ozaki(const void* tm_s, const OzStep& P, cudaStream_t st) {
  using namespace oz;
  constexpr int SMEM_BYTES = Cfg<NS>::SMEM_BYTES;
  static std::once_flag attr_done[64];
  once_per_device(attr_done, []() {
    cudaFuncSetAttribute(ozaki_band_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  });
  const long long grid = P.total < gemm_num_sms() ? P.total : gemm_num_sms();
  ozaki_band_kernel<NS><<<(unsigned)grid, THREADS, SMEM_BYTES, st>>>(*reinterpret_cast<const CUtensorMap*>(tm_s), P);
  return launch_status("ozaki_band_kernel");
}

// Targets of the panel solve at step k: off-band tiles i = first .. nt-1, all
// MB x NB items each.
long long ozaki_trsm_targets(int ts, int nt, int first, std::vector<int4>& out) {
  const int MB = ts / oz::BM, NB = ts / oz::BN;
  long long items = 0;
  for (int i = first; i < nt; ++i) {
    out.push_back(make_int4(i, 0, (int)items, 0));
    items += (long long)MB * NB;
  }
  return items;
}

int launch_ozaki_trsm(const void* tm_s, const int4* targets, int ntargets, long long total, int ts, int k,
                      long long b_row_base, double* w_out, const double* scale, int* err, cudaStream_t st) {
  if (ts % oz::BM != 0) return EGS_ERR_INVALID;
  if (total <= 0 || ntargets <= 0) return EGS_OK;
  OzStep P{};
  P.targets = targets;
  P.ntargets = ntargets;
  P.total = total;
  P.ts = ts;
  P.mode = 1;
  P.k = k;
  P.b_row_base = b_row_base;
  P.w_out = w_out;
  P.scale = scale;
  P.err = err;
  return launch_ozaki<kOzPanelSlices>(tm_s, P, st);
}

int launch_ozaki_band(const void* tm_s, const int4* targets, int ntargets, long long total, int ts, int band,
                      double* band_pool, const double* scale, int* err, cudaStream_t st) {
  using namespace oz;
  if (ts % BM != 0 || ts / BN > 2 * (ts / BM)) return EGS_ERR_INVALID;
  if (total <= 0 || ntargets <= 0) return EGS_OK;
  OzStep P{};
  P.targets = targets;
  P.ntargets = ntargets;
  P.total = total;
  P.ts = ts;
  P.band = band;
  P.mode = 0;
  P.band_pool = band_pool;
  P.scale = scale;
  P.err = err;
  return launch_ozaki<kOzSlices>(tm_s, P, st);
}

}  // namespace egs

using namespace egs;

// Test entry: one band update of step k from panel tiles W[t] = L_{k+t,k}
// (t = 0 .. nt-k-1, FP64 column-major ts x ts; W[0] is not read) into the FP64
// band pool (nt * (band + 1) tiles, slot j * (band + 1) + (i - j)).
extern "C" int egs_ozaki_band_update(int ts, int nt, int band, int k, const double* W, double* band_pool,
                                     double* ms) {
  if (ts <= 0 || ts % oz::BM != 0 || nt <= 0 || band < 0 || k < 0 || k >= nt || !W || !band_pool)
    return EGS_ERR_INVALID;
  const int ntp = nt - k;
  const long long rows = (long long)nt * ts;
  int8_t* sl = nullptr;
  double* scale = nullptr;
  int* err = nullptr;
  int4* dt = nullptr;
  alignas(64) unsigned char tm[128];
  std::vector<int4> targets;
  const long long total = ozaki_targets(ts, nt, band, k, targets);
  int rc = EGS_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&sl, (size_t)rows * ts * oz::S) || cudaMalloc(&scale, rows * sizeof(double)) ||
      cudaMalloc(&err, sizeof(int)) || cudaMalloc(&dt, std::max<size_t>(1, targets.size()) * sizeof(int4))) {
    cudaGetLastError();
    rc = EGS_ERR_OOM;
    goto done;
  }
  cudaMemset(err, 0, sizeof(int));
  cudaMemset(scale, 0, rows * sizeof(double));
  cudaMemset(sl, 0, (size_t)rows * ts * oz::S);
  if (!targets.empty()) cudaMemcpy(dt, targets.data(), targets.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if ((rc = ozaki_tensor_map(tm, sl, ts, rows)) != EGS_OK) goto done;
  launch_ozaki_slice(W, ts, 1, ntp - 1, k, scale, sl, rows, 0);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  if ((rc = launch_ozaki_band(tm, dt, (int)targets.size(), total, ts, band, band_pool, scale, err, 0)) != EGS_OK)
    goto done;
  cudaEventRecord(e1, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    rc = EGS_ERR_CUDA;
    set_last_error(cudaGetErrorString(cudaGetLastError()), "egs_ozaki_band_update");
    goto done;
  }
  {
    int h = 0;
    cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (h) {
      set_last_error("a device-side wait exceeded its limit", "egs_ozaki_band_update");
      rc = EGS_ERR_TIMEOUT;
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(sl);
  cudaFree(scale);
  cudaFree(err);
  cudaFree(dt);
  return rc;
}
