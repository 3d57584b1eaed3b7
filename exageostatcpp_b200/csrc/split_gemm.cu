// Off-band trailing update of the mixed-precision factorisation on the
// 5th-generation tensor cores (tcgen05, sm_100a), with FP32 accuracy from
// FP16 operands.
//
// At step k every off-band target tile (i, j), k < j, j + band < i, is updated
// C_ij -= L_ik L_jk^T with C stored in FP32.  The solved panel column
// (FP64) is first split per row into two FP16 parts after a power-of-two row
// scaling s_r (max |s_r L_r.| in [2^13, 2^14)):
//     hi = fp16(s L),  lo = fp16(s L - hi),   s L = hi + lo + O(2^-22 |s L|),
// and the product is assembled from three FP16 tensor-core products with FP32
// accumulation in tensor memory,
//     (s_a a)(s_b b) ~ hi_a hi_b + hi_a lo_b + lo_a hi_b,
// then unscaled exactly (powers of two) in the epilogue.  The dropped lo*lo
// term is O(2^-22) relative, so the update has FP32-level accuracy while it
// runs on the FP16 tensor path (kind::f16).  Per-row scaling keeps the FP16
// parts in range whatever the magnitude of the factor's rows.
//
// Promotion.  The tensor core's FP32 accumulation does not round to nearest:
// sums of same-sign products come out systematically short (about 8e-6
// relative after K = 1024, i.e. ~1 ulp per instruction).  The Cholesky
// updates of a positively correlated covariance are such sums, and the bias
// reaches the log-determinant at first order.  So each 64-wide K stage is
// accumulated from zero in tensor memory -- the two small correction products
// first, the main hi*hi product last, so at most four instructions add into a
// full-size accumulator -- and the epilogue adds the stage's partial sum into
// FP32 registers with round-to-nearest.  The bias drops to that of four
// instructions (~2e-7 relative), the same order as plain FP32 rounding.
//
// Kernel structure: persistent clusters of two CTAs on the two SMs of a TPC,
// one 256 x 256 output tile per pair at a time, issued as tcgen05.mma of
// cta_group::2 (M = 256, N = 256): each CTA holds its 128 rows of A and 128
// of the 256 rows of B in its own shared memory, the tensor cores of both SMs
// read both B halves, and each CTA's tensor memory receives its 128 rows x 256
// columns of the product.  Against one CTA per 128 x 256 tile this halves the
// B operand every SM stages (64 KB per 64-wide K stage instead of 96 KB), so
// the ring holds three stages instead of two and the L2 -> SM operand traffic
// per flop drops by a third.
//   warp 0    TMA producer of each CTA: per K stage its A rows (hi, lo) and its
//             B half (hi, lo), 128B-swizzled, into a 3-stage ring; the copies of
//             both CTAs complete on the leader CTA's full barrier; a few stages
//             before a tile ends it prefetches its C block to L2;
//   warp 1    allocates 512 TMEM columns in both CTAs (two 128 x 256 FP32 stage
//             accumulators per CTA); in the leader CTA (rank 0) one thread
//             issues the MMAs, and its commits arrive on the ring and the
//             accumulator barriers of both CTAs;
//   warps 2-9 epilogue of each CTA: warp w reads TMEM lanes 32 (w % 4) .. +32
//             (thread = tile row) and one half of the columns, adds every stage
//             into 128 FP32 registers, releases the stage accumulator to the
//             leader, and after the last stage applies C -= acc * inv_s_row *
//             inv_s_col with reductions into L2 (red.global.add), issued
//             straight from the registers without waiting.
// The two stage accumulators let the MMAs of stage s+1 overlap the draining of
// stage s.  Every mbarrier wait is bounded; a timed-out CTA records the error,
// stops, and still meets its peer at the final cluster barrier and frees its
// tensor memory.  No copy is multicast: each CTA loads only what it holds.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstring>
#include "common.cuh"
#include "kernels.cuh"
#include "mbarrier.cuh"
#include "panel_scales.cuh"

namespace egs {

namespace sg {
// BM: rows of the output tile each CTA holds; the pair covers PM = 2 BM rows.
constexpr int BM = 128, PM = 256, BN = 256, BK = 64, STAGES = 3;
constexpr int BOX_ROWS = 128;                      // TMA box: 64 fp16 (128 B) x 128 rows
constexpr int A_BYTES = BM * BK * 2;               // 16 KB: this CTA's A rows
constexpr int B_BYTES = (BN / 2) * BK * 2;         // 16 KB: this CTA's half of B
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int EPI_WARPS = 8;                       // two per TMEM lane quarter
constexpr int THREADS = 64 + 32 * EPI_WARPS;       // producer, MMA issuer, epilogue
constexpr int HALF_COLS = BN / 2;                  // accumulator columns per epilogue thread
constexpr int PF_AHEAD = 6;                        // stages before a tile's end at which C is prefetched
constexpr int SMEM_BYTES = 1024 + STAGES * STAGE_BYTES + 256;
static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");
constexpr uint32_t TMEM_COLS = 512;
// Instruction descriptor of kind::f16: D F32 (bits 4-5 = 1), A and B F16 (0),
// both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28 (M of the pair).
constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(PM >> 4) << 24);
}  // namespace sg

// ---------------------------------------------------------------------------
// Row scaling and FP16 split of a solved panel
// ---------------------------------------------------------------------------

// Power-of-two scale of row r of panel tile t: inv_scale = 2^(e - 13) with
// 2^e <= max_c |W(r, c)| < 2^(e+1); rows whose maximum is 0 (or below 2^-120)
// get inv_scale 0 and split to zeros.  W: column-major ts x ts tiles.
__global__ void __launch_bounds__(256)
panel_rowscale_kernel(const double* __restrict__ W, int ts, int t0, int row_tile0, float* __restrict__ inv_scale) {
  __shared__ double red[4][64];
  const int t = t0 + blockIdx.y;
  const int rl = threadIdx.x & 63, g = threadIdx.x >> 6;
  const int r = blockIdx.x * 64 + rl;
  const double* col = W + (long long)t * ts * ts + r;
  double m = 0.0;
  for (int c = g; c < ts; c += 4) m = fmax(m, fabs(col[(long long)c * ts]));
  red[g][rl] = m;
  __syncthreads();
  if (g == 0) {
    m = fmax(fmax(red[0][rl], red[1][rl]), fmax(red[2][rl], red[3][rl]));
    inv_scale[(long long)(row_tile0 + t) * ts + r] = f16_row_inv_scale(m);
  }
}

// hi/lo FP16 parts of 64 x 64 blocks of panel tiles, transposed to row-major
// (K contiguous) rows of Ph / Pl (row stride ts).
__global__ void __launch_bounds__(256)
panel_split_kernel(const double* __restrict__ W, int ts, int t0, int row_tile0, const float* __restrict__ inv_scale,
                   __half* __restrict__ Ph, __half* __restrict__ Pl) {
  __shared__ double S[64][65];
  const int t = t0 + blockIdx.z;
  const int r0 = blockIdx.x * 64, c0 = blockIdx.y * 64;
  const double* src = W + (long long)t * ts * ts;
  for (int e = threadIdx.x; e < 64 * 64; e += 256) {
    const int r = e & 63, c = e >> 6;
    S[r][c] = src[(long long)(c0 + c) * ts + r0 + r];
  }
  __syncthreads();
  const long long grow0 = (long long)(row_tile0 + t) * ts + r0;
  for (int e = threadIdx.x; e < 64 * 32; e += 256) {
    const int r = e >> 5, c = (e & 31) * 2;
    const float inv = inv_scale[grow0 + r];
    const double s = (inv > 0.0f) ? 1.0 / (double)inv : 0.0;  // exact: inv is a power of two
    const double v0 = S[r][c] * s, v1 = S[r][c + 1] * s;
    const __half h0 = __double2half(v0), h1 = __double2half(v1);
    const __half l0 = __double2half(v0 - (double)__half2float(h0));
    const __half l1 = __double2half(v1 - (double)__half2float(h1));
    const long long off = (grow0 + r) * ts + c0 + c;
    *reinterpret_cast<__half2*>(Ph + off) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2*>(Pl + off) = __halves2half2(l0, l1);
  }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms of
// 1024 bytes stacked contiguously (stride byte offset 1024), sm_100 version 1.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFF) >> 4);
  d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
  d |= (uint64_t)1 << 46;             // descriptor version
  d |= (uint64_t)2 << 61;             // SWIZZLE_128B
  return d;
}
// D (both CTAs' tensor memory) += A B^T over the CTA pair; issued by one thread
// of the leader CTA, the operands at the same shared-memory offsets in both CTAs.
__device__ __forceinline__ void umma_f16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(sg::IDESC), "r"(accumulate)
      : "memory");
}
// Arrives on the barrier at this offset in both CTAs of the pair once the MMAs
// issued so far have completed.
__device__ __forceinline__ void umma_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)0x3)
      : "memory");
}
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Address of this CTA's shared variable p in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
// Arrive on a barrier of the peer CTA.  The default (CTA-scope release)
// semantics suffice: what the arrive publishes is the completion of this
// warp's tensor-memory loads, ordered by tcgen05.fence::before_thread_sync;
// a cluster-scope release would add a memory barrier to every stage.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar_cluster_addr) {
  asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster_addr) : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Box (x, y) into this CTA's shared memory; the bytes complete on the barrier at
// bar_cluster_addr, which may lie in the peer CTA of the pair (no multicast).
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, uint32_t bar_cluster_addr, int x,
                                                 int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar_cluster_addr)
      : "memory");
}
// L2 prefetch of one box of a tiled tensor (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch_l2_2d(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"((uint64_t)map), "r"(x),
               "r"(y)
               : "memory");
}
// 32 consecutive FP32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
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
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive FP32 columns of this warp's 32 TMEM lanes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void red_add_f32(float* addr, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(addr), "f"(v) : "memory");
}

// Target tile of work item L at step k: targets are enumerated column by column
// (j = k+1, ...; i = j+band+1 .. nt-1), each split into (ts/PM) x (ts/BN) pair
// tiles with the row block fastest.
struct SplitStep {
  int ts, nt, band, k;
  int mblocks, nblocks;
  long long total;
  float* c_pool;            // off-band FP32 tiles: slot(i, j) = tile_slot(i - band - 1, j, nt - band - 1)
  const float* inv_scale;   // per global row
  int* err;
};

__device__ __forceinline__ void decode_item(const SplitStep& P, long long L, int& i, int& j, int& mb, int& nb) {
  const long long per = (long long)P.mblocks * P.nblocks;
  long long q = L / per;
  const int w = (int)(L - q * per);
  nb = w / P.mblocks;
  mb = w - nb * P.mblocks;
  j = P.k + 1;
  long long cnt = P.nt - j - P.band - 1;
  while (q >= cnt) {
    q -= cnt;
    ++j;
    --cnt;
  }
  i = j + P.band + 1 + (int)q;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(sg::THREADS, 1)
split_gemm_kernel(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                  const __grid_constant__ CUtensorMap tm_c,
                  const __grid_constant__ SplitStep P) {
  using namespace sg;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  __shared__ int bail_flag;
  volatile int& bail = bail_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  const long long pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);    // the leader's producer (expect_tx of both CTAs' bytes)
      mbar_init(&empty[s], 1);   // the leader's MMA commit, in both CTAs
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);               // the leader's MMA commit, in both CTAs
      mbar_init(&acc_empty[b], 2 * EPI_WARPS);  // the epilogue warps of both CTAs (leader's copy)
    }
    bail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    // same warp and same slot offset in both CTAs
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  // both CTAs' barriers are initialised before any copy or arrive can reach them
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int ksteps = P.ts / BK;
  const int pf_kt = ksteps > PF_AHEAD ? ksteps - PF_AHEAD : 0;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      const int mm = P.nt - P.band - 1;
      for (long long L = pair; L < P.total && !bail; L += npairs) {
        int i, j, mb, nb;
        decode_item(P, L, i, j, mb, nb);
        const int arow = i * P.ts + mb * PM + (int)rank * BM, brow = j * P.ts + nb * BN + (int)rank * (BN / 2);
        for (int kt = 0; kt < ksteps; ++kt, ++it) {
          const uint32_t s = it % STAGES;
          if (it >= (uint32_t)STAGES && !mbar_wait(&empty[s], ((it / STAGES) & 1) ^ 1, P.err)) {
            bail = 1;
            break;
          }
          uint8_t* st = smem + s * STAGE_BYTES;
          if (leader) mbar_expect_tx(&full[s], 2 * STAGE_BYTES);
          const uint32_t fb = cluster_addr(&full[s], 0);
          const int x = kt * BK;
          tma_load_2d_pair(st, &tm_hi, fb, x, arow);
          tma_load_2d_pair(st + A_BYTES, &tm_lo, fb, x, arow);
          tma_load_2d_pair(st + 2 * A_BYTES, &tm_hi, fb, x, brow);
          tma_load_2d_pair(st + 2 * A_BYTES + B_BYTES, &tm_lo, fb, x, brow);
          if (kt == pf_kt) {
            // this CTA's C block (BM rows x BN columns of an FP32 tile) into L2
            const long long slot = tile_slot(i - P.band - 1, j, mm);
            tma_prefetch_l2_2d(&tm_c, mb * PM + (int)rank * BM, (int)(slot * P.ts + nb * BN));
          }
        }
      }
      // drain (leader): the stages issued last must land before either CTA may exit;
      // the peer's copies complete on the same barriers
      if (leader) {
        const uint32_t first = it > (uint32_t)STAGES ? it - STAGES : 0;
        for (uint32_t q = first; q < it; ++q) mbar_wait(&full[q % STAGES], (q / STAGES) & 1, P.err);
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      uint32_t it = 0;
      bool ok = true;
      for (long long L = pair; L < P.total && ok && !bail; L += npairs) {
        for (int kt = 0; kt < ksteps; ++kt, ++it) {
          // stage it accumulates into buffer it & 1 from zero
          const uint32_t ab = it & 1, s = it % STAGES;
          if (it >= 2 && !mbar_wait(&acc_empty[ab], ((it >> 1) & 1) ^ 1, P.err)) {
            ok = false;
            break;
          }
          if (!mbar_wait(&full[s], (it / STAGES) & 1, P.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dcol = tmem_base + ab * BN;
          const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t sal = sa + A_BYTES, sbh = sa + 2 * A_BYTES, sbl = sbh + B_BYTES;
          // corrections first (small partial sums), the main product last
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint32_t off = kk * 32;
            umma_f16_pair(dcol, sdesc_sw128(sa + off), sdesc_sw128(sbl + off), kk > 0 ? 1u : 0u);
            umma_f16_pair(dcol, sdesc_sw128(sal + off), sdesc_sw128(sbh + off), 1u);
          }
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint32_t off = kk * 32;
            umma_f16_pair(dcol, sdesc_sw128(sa + off), sdesc_sw128(sbh + off), 1u);
          }
          umma_commit_pair(&empty[s]);
          umma_commit_pair(&acc_full[ab]);
        }
      }
      if (!ok) bail = 1;
    }
  } else {
    // epilogue warps 2..9: TMEM lane quarter = warp % 4, column half by warp group
    const int quarter = warp & 3, half = (warp - 2) >> 2;
    const uint32_t tl = tmem_base + ((uint32_t)(quarter * 32) << 16) + half * HALF_COLS;
    uint32_t it = 0, red_count = 0;
    bool ok = true;
    for (long long L = pair; L < P.total && ok; L += npairs) {
      float acc[HALF_COLS];  // zero plus the first stage is that stage's value
#pragma unroll
      for (int c = 0; c < HALF_COLS; ++c) acc[c] = 0.f;
      for (int kt = 0; kt < ksteps; ++kt, ++it) {
        const uint32_t ab = it & 1;
        // one lane waits, the warp follows it uniformly (tcgen05.ld needs the whole warp)
        int w = 1;
        if (lane == 0) w = mbar_wait(&acc_full[ab], (it >> 1) & 1, P.err) ? 1 : 0;
        w = __shfl_sync(0xffffffffu, w, 0);
        if (!w) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int g = 0; g < HALF_COLS / 16; ++g) {
          float v[16];
          tmem_ld16(tl + ab * BN + g * 16, v);
#pragma unroll
          for (int c = 0; c < 16; ++c) acc[g * 16 + c] += v[c];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if (leader)
            mbar_arrive(&acc_empty[ab]);
          else
            mbar_arrive_remote(cluster_addr(&acc_empty[ab], 0));
        }
      }
      if (!ok) break;
      // C -= acc * inv_r * inv_c straight from the registers: per column, the
      // warp's 32 lanes (32 consecutive rows) reduce 128 contiguous bytes of the
      // column-major FP32 tile in L2 (red.global.add, round to nearest); nothing
      // waits for the reductions, so the epilogue turns to the next tile's
      // stages at once.  Each element of C has one writer per launch.
      int i, j, mb, nb;
      decode_item(P, L, i, j, mb, nb);
      const int mm = P.nt - P.band - 1;
      const long long slot = tile_slot(i - P.band - 1, j, mm);
      const int r0 = mb * PM + (int)rank * BM + quarter * 32;
      const int c0 = nb * BN + half * HALF_COLS;
      const float inv_r = P.inv_scale[(long long)i * P.ts + r0 + lane];
      float inv_c[HALF_COLS / 32];  // lane l holds the scales of columns l, l + 32, ...
#pragma unroll
      for (int q = 0; q < HALF_COLS / 32; ++q) inv_c[q] = __ldg(P.inv_scale + (long long)j * P.ts + c0 + q * 32 + lane);
      float* cp = P.c_pool + (slot * P.ts + c0) * (long long)P.ts + r0 + lane;
#pragma unroll
      for (int c = 0; c < HALF_COLS; ++c) {
        const float sc = __shfl_sync(0xffffffffu, inv_c[c >> 5], c & 31);
        red_add_f32(cp + (long long)c * P.ts, -(acc[c] * inv_r) * sc);
      }
    }
    if (!ok) bail = 1;
  }
  // neither CTA leaves (or frees its tensor memory) while the other may still
  // issue MMAs into it, read its shared memory or arrive on its barriers
  __syncwarp();
  tc_fence_before();
  cluster_sync_all();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

int split_tensor_map(void* storage, const __half* base, int ts, long long rows) {
  void* fn = nullptr;
  if (tensor_map_encoder(&fn) != EGS_OK) return EGS_ERR_CUDA;
  if (ts % 64 != 0 || ((uintptr_t)base & 15) != 0) return EGS_ERR_INVALID;
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  cuuint64_t dims[2] = {(cuuint64_t)ts, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ts * 2};
  cuuint32_t box[2] = {sg::BK, sg::BOX_ROWS};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(reinterpret_cast<CUtensorMap*>(storage), CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                      const_cast<__half*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed", "split_tensor_map");
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

// The off-band FP32 pool as a 2-D tensor (tile rows fastest, then every column
// of every slot) in BM x BN boxes: the C block of a CTA tile, prefetched to L2
// before the tile's last stages.
int split_c_map(void* storage, const float* c_pool, int ts, long long nslots) {
  constexpr int box_rows = sg::BM, box_cols = sg::BN;
  std::memset(storage, 0, 128);
  if (nslots <= 0) return EGS_OK;  // no off-band tile, no update launches
  void* fn = nullptr;
  if (tensor_map_encoder(&fn) != EGS_OK) return EGS_ERR_CUDA;
  if (ts % sg::BN != 0 || ((uintptr_t)c_pool & 15) != 0) return EGS_ERR_INVALID;
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  cuuint64_t dims[2] = {(cuuint64_t)ts, (cuuint64_t)(nslots * ts)};
  cuuint64_t strides[1] = {(cuuint64_t)ts * 4};
  cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(reinterpret_cast<CUtensorMap*>(storage), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                      const_cast<float*>(c_pool), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error("cuTensorMapEncodeTiled failed", "split_c_tensor_map");
    return EGS_ERR_CUDA;
  }
  return EGS_OK;
}

void launch_panel_split(const double* W, int ts, int t0, int ntiles, int row_tile0, float* inv_scale, __half* Ph,
                        __half* Pl, cudaStream_t st) {
  if (ntiles <= 0) return;
  panel_rowscale_kernel<<<dim3(ts / 64, ntiles), 256, 0, st>>>(W, ts, t0, row_tile0, inv_scale);
  panel_split_kernel<<<dim3(ts / 64, ts / 64, ntiles), 256, 0, st>>>(W, ts, t0, row_tile0, inv_scale, Ph, Pl);
}

// Number of off-band target tiles at step k.
long long split_targets(int nt, int band, int k) {
  long long n = 0;
  for (int j = k + 1; j < nt; ++j) {
    const int c = nt - j - band - 1;
    if (c > 0) n += c;
  }
  return n;
}

// Clusters of split_gemm_kernel that can be resident at once on the current
// device (once per device; half the SM count if the query fails).
static long long split_max_pairs() {
  static std::once_flag done[64];
  static long long pairs_of[64];
  int dev = 0;
  cudaGetDevice(&dev);
  auto query = [dev]() {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * 74, 1, 1);
    cfg.blockDim = dim3(sg::THREADS, 1, 1);
    cfg.dynamicSmemBytes = sg::SMEM_BYTES;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, split_gemm_kernel, &cfg) != cudaSuccess) {
      cudaGetLastError();
      n = gemm_num_sms() / 2;
    }
    if (dev >= 0 && dev < 64) pairs_of[dev] = n;
    return n;
  };
  if (dev < 0 || dev >= 64) return query();
  std::call_once(done[dev], query);
  return pairs_of[dev];
}

int launch_split_update(const void* tm_hi, const void* tm_lo, const void* tm_c, int ts, int nt,
                        int band, int k, float* c_pool, const float* inv_scale, int* err, cudaStream_t st,
                        int max_ctas) {
  using namespace sg;
  if (ts % BN != 0) return EGS_ERR_INVALID;
  const long long targets = split_targets(nt, band, k);
  if (targets == 0) return EGS_OK;
  static std::once_flag attr_done[64];
  once_per_device(attr_done,
                  []() { cudaFuncSetAttribute(split_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES); });
  SplitStep P;
  P.ts = ts;
  P.nt = nt;
  P.band = band;
  P.k = k;
  P.mblocks = ts / PM;
  P.nblocks = ts / BN;
  P.total = targets * P.mblocks * P.nblocks;
  P.c_pool = c_pool;
  P.inv_scale = inv_scale;
  P.err = err;
  // clusters of two CTAs: as many pairs as fit on the device at once (SMs of a
  // TPC pair up; a TPC with one usable SM runs none), at most one per pair tile
  long long pairs = split_max_pairs();
  if (pairs <= 0) {
    set_last_error("no CTA pair of the kernel fits on an SM pair (registers or shared memory)", "split_gemm_kernel");
    return EGS_ERR_CUDA;
  }
  if (max_ctas > 0 && max_ctas / 2 < pairs) pairs = max_ctas / 2 > 0 ? max_ctas / 2 : 1;
  if (P.total < pairs) pairs = P.total;
  const long long grid = 2 * pairs;
  split_gemm_kernel<<<(unsigned)grid, THREADS, SMEM_BYTES, st>>>(*reinterpret_cast<const CUtensorMap*>(tm_hi),
                                                                 *reinterpret_cast<const CUtensorMap*>(tm_lo),
                                                                 *reinterpret_cast<const CUtensorMap*>(tm_c), P);
  return launch_status("split_gemm_kernel");
}

}  // namespace egs

using namespace egs;

extern "C" int egs_split_update(int ts, int nt, int band, int k, const double* panel, float* offband, double* ms) {
  if (ts <= 0 || ts % sg::BN != 0 || nt <= 0 || band < 0 || k < -1 || k >= nt || !panel || !offband)
    return EGS_ERR_INVALID;
  const long long rows = (long long)nt * ts;
  __half *ph = nullptr, *pl = nullptr;
  float* inv = nullptr;
  int* err = nullptr;
  alignas(64) unsigned char tmh[128], tml[128], tmc[128];
  const long long mm = nt - band - 1 > 0 ? nt - band - 1 : 0;
  int rc = EGS_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&ph, rows * ts * sizeof(__half)) || cudaMalloc(&pl, rows * ts * sizeof(__half)) ||
      cudaMalloc(&inv, rows * sizeof(float)) || cudaMalloc(&err, sizeof(int))) {
    cudaGetLastError();
    rc = EGS_ERR_OOM;
    goto done;
  }
  cudaMemset(err, 0, sizeof(int));
  cudaMemset(inv, 0, rows * sizeof(float));
  cudaMemset(ph, 0, rows * ts * sizeof(__half));
  cudaMemset(pl, 0, rows * ts * sizeof(__half));
  if ((rc = split_tensor_map(tmh, ph, ts, rows)) != EGS_OK || (rc = split_tensor_map(tml, pl, ts, rows)) != EGS_OK ||
      (rc = split_c_map(tmc, offband, ts, mm * (mm + 1) / 2)) != EGS_OK)
    goto done;
  launch_panel_split(panel, ts, k + 1, nt - k - 1, 0, inv, ph, pl, 0);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, 0);
  if ((rc = launch_split_update(tmh, tml, tmc, ts, nt, band, k, offband, inv, err, 0)) != EGS_OK) goto done;
  cudaEventRecord(e1, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    rc = EGS_ERR_CUDA;
    set_last_error(cudaGetErrorString(cudaGetLastError()), "egs_split_update");
    goto done;
  }
  {
    int h = 0;
    cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
    if (h) {
      set_last_error("a device-side wait exceeded its limit", "egs_split_update");
      rc = EGS_ERR_TIMEOUT;
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(ph);
  cudaFree(pl);
  cudaFree(inv);
  cudaFree(err);
  return rc;
}
