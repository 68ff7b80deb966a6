// Split-precision products on the 5th-generation tensor cores (tcgen05) for the Cholesky route
// of the two-electron tensors.
//
// With Cholesky-factored integrals (mu nu|lam sig) = sum_P L^P[mu nu] L^P[lam sig], every
// four-index transform of the build, T(A,B,C,D)[p,q,r,s] = sum (mu nu|lam sig) A[mu,p] B[nu,q]
// C[lam,r] D[sig,s] (src/maths/eri.rs:258, the J and II tensors of
// src/nonorthogonalwicks/build.rs:261-313,876-917), becomes one dense product
//   T[pq][rs] = sum_P U[P][pq] V[P][rs],  U[P] = A^T L^P B,  V[P] = C^T L^P D,
// an (n^2 x naux) x (naux x n^2) GEMM.  This file runs that product on tcgen05 from FP64 factors
// in one of two split forms:
//   * NW_TRANSFORM_CHOL_BF16X6: each factor entry is cut into three BF16 pieces (hi, mid, lo) and the six
//     products of total order <= 2 are summed in FP32 in tensor memory (FP32-class result);
//   * NW_TRANSFORM_CHOL_INT8: Ozaki-style integer slices.  Each row of U (and of V) is scaled by a power of
//     two so its largest entry is at most 1/2, then cut into S signed 7-bit slices
//     x = sum_i a_i 2^(-7 (i + 1)); the products of slices with i + j = s are summed exactly in
//     INT32 in tensor memory (one accumulator per s), and the result is rebuilt in FP64 as
//     sum_s 2^(e_row + e_col - 7 (s + 2)) C_s.  With S = 8 the result is FP64-faithful.
//
// Kernel shape: persistent, one CTA of 320 threads per SM walking 128 x 64 tiles of T
// (cta_group::1, M = 128, N = 64).
// Operands are pre-tiled in global memory by the split kernels in the tcgen05 no-swizzle K-major
// layout (8-row x 16-byte core matrices, 64-byte-deep K tiles), so the K tile of one piece of an
// operand is one contiguous block moved by a single cp.async.bulk (no multicast).  A pipeline
// stage holds the K tile of EVERY piece of both operands (int8: 8 + 8 slices, 96 KB, two stages;
// BF16: 3 + 3 pieces, 36 KB, five stages), so each slice is read from L2 once per tile and all
// products of that K tile run from shared memory.  Warp 0 issues the copies (running ahead
// across tile boundaries), warp 1 the MMAs (tcgen05.mma, two 32-byte K steps per product and
// stage, then tcgen05.commit to free the stage; one more commit marks the tile's accumulators
// complete); each product (A piece, B piece) goes to its accumulator's 64 TMEM columns.  Eight
// epilogue warps (2..9) drain a tile: warp w reads TMEM lanes 32 (w % 4) .. + 31 and one half of
// the columns of every accumulator with one 32-column tcgen05.ld each, releases the TMEM to the
// next tile's MMAs, then rebuilds FP64 (exact int32 -> FP64 conversion by the 2^52 + 2^31
// offset, power-of-two scales built from the exponent bits) and stores T in the [p][r][q][s]
// order of the build's T4 buffers while the next tile is copied and multiplied.  Every
// mbarrier wait is bounded: on a timeout the CTA records an error flag, stops issuing work,
// waits (bounded) for what it issued, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "internal.cuh"

namespace nw {
namespace {

// warp 0: copies, warp 1: MMAs, warps 2..9: epilogue
constexpr int kTcThreads = 320;
constexpr int kEpiWarps = 8;
constexpr int kTileM = 128, kTileN = 64;
// Bytes of K per tile row and stage: 64 for both splits (int8: the 16 slices of a K tile take
// 96 KB, two stages; BF16: 6 pieces, 36 KB, five stages; 32-byte int8 tiles in four stages
// were measured slower, 336 against 279 us at n = 64, naux = 256).  A pre-tiled 64-row block
// holds 64 x that many bytes, a 128-row A tile two adjacent blocks; consecutive 8-row groups
// of a block are 8 x 16 x (K bytes / 16) bytes apart (the descriptor's stride offset).
constexpr int kbytes_of(int kind) { return kind == 1 ? 64 : 64; }
constexpr uint32_t block_bytes_of(int kind) { return 64u * (uint32_t)kbytes_of(kind); }
constexpr uint32_t sbo_of(int kind) { return 8u * 16u * (uint32_t)(kbytes_of(kind) / 16); }
constexpr int kMaxAcc = 8;                          // accumulators of 64 columns (512 TMEM columns)
constexpr uint32_t kWaitLimit = 1u << 24;           // try_wait rounds before a wait gives up

template <int kKind>
struct TcShape {
  static constexpr int kPieces = kKind == 1 ? kOzakiSlices : 3;
  static constexpr int kStages = kKind == 1 ? 2 : 5;
  static constexpr int kKBytes = kbytes_of(kKind);
  static constexpr uint32_t kBlockBytes = block_bytes_of(kKind);
  static constexpr uint32_t kTileABytes = kTileM * kKBytes, kTileBBytes = kTileN * kKBytes;
  static constexpr uint32_t kSbo = sbo_of(kKind);
  static constexpr uint32_t kStageA = kPieces * kTileABytes, kStageB = kPieces * kTileBBytes;
  // ring, barriers (full and empty per stage, tmem_full, tmem_empty), TMEM slot + abort flag
  static constexpr size_t kSmem = 1024 + (size_t)kStages * (kStageA + kStageB) + 8 * (2 * kStages + 2) + 8;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Waits for the phase of `parity` to complete; false after kWaitLimit unsuccessful rounds.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Shared-memory matrix descriptor, no swizzle: start, leading-dimension byte offset (between
// core matrices adjacent in K), stride byte offset (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D format (1 = F32, 2 = S32), A/B formats (kind::f16: 1 = BF16;
// kind::i8: 1 = signed), both operands K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t idesc(uint32_t dfmt, uint32_t abfmt, uint32_t m, uint32_t n) {
  return (dfmt << 4) | (abfmt << 7) | (abfmt << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

template <int kKind>  // 0: kind::f16 (BF16 in, F32 accumulate), 1: kind::i8 (S8 in, S32 accumulate)
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  if constexpr (kKind == 0) {
    constexpr uint32_t id = idesc(1, 1, kTileM, kTileN);
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(ad), "l"(bd), "r"(id), "r"(accumulate));
  } else {
    constexpr uint32_t id = idesc(2, 1, kTileM, kTileN);
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem),
        "l"(ad), "l"(bd), "r"(id), "r"(accumulate));
  }
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Exact int32 -> FP64: the low word of 2^52 + 2^31 + x, minus that offset (one DADD).
__device__ __forceinline__ double i32_to_f64(uint32_t x) {
  return __hiloint2double(0x43300000, (int)(x ^ 0x80000000u)) - 4503601774854144.0;
}

// v 2^e; a multiplication by the exact power of two when 2^e is a normal number (the same
// single rounding as ldexp), ldexp otherwise.
__device__ __forceinline__ double scale_pow2(double v, int e) {
  if (e >= -1022 && e <= 1023) return v * __longlong_as_double((long long)(e + 1023) << 52);
  return ldexp(v, e);
}

struct TcArgs {
  const uint8_t* a;        // pre-tiled A pieces: [piece][k tile][64-row block][4 KB]
  const uint8_t* b;        // pre-tiled B pieces, same layout
  long long a_piece, b_piece;  // bytes per piece
  int nkt;                 // K tiles per piece
  int nrt_a, nrt_b;        // 64-row blocks of each operand (rows padded to 128)
  int nprod;               // products
  int8_t pa[64], pb[64], pacc[64];  // per product: A piece, B piece, accumulator
  int8_t pfirst[64];       // 1 for the first product of its accumulator (starts it at K tile 0)
  int nacc;
  double acc_scale[kMaxAcc];   // per accumulator: 2^(-7 (s + 2)) (int8) or 1 (bf16)
  const int* erow;         // per row / column power-of-two exponents (int8), or null
  const int* ecol;
  int M, N;                // rows (pq) and columns (rs) of T
  int n;                   // orbital count: T[pq][rs] is stored at [p][r][q][s]
  int ntm, ntn;            // 128-row and 64-column tiles of T
  double* out;
  uint32_t* err;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Persistent kernel: each CTA takes tiles blockIdx.x, blockIdx.x + gridDim.x, ... (64-column
// tiles fastest, so the CTAs working at one time share their A tiles).  The copy warp runs
// ahead through the stage ring across tile boundaries; the MMA warp starts a tile once the
// epilogue has read the previous tile's accumulators out of TMEM (tmem_empty), and signals a
// finished tile with tcgen05.commit (tmem_full); the epilogue warps convert and store a tile
// while the next tile's copies and MMAs proceed.
template <int kKind>
__global__ void __launch_bounds__(kTcThreads, 1) tc_gemm_kernel(const __grid_constant__ TcArgs g) {
  using Sh = TcShape<kKind>;
  constexpr int kPieces = Sh::kPieces, kStages = Sh::kStages;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte aligned stage rings (A tiles, then B tiles); barriers after them
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sa = smem;
  uint8_t* sb = smem + kStages * Sh::kStageA;
  uint64_t* full = reinterpret_cast<uint64_t*>(sb + kStages * Sh::kStageB);
  uint64_t* empty = full + kStages;
  uint64_t* tmem_full = empty + kStages;
  uint64_t* tmem_empty = tmem_full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tmem_empty + 1);
  volatile uint32_t* abort_flag = tmem_slot + 1;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = g.ntm * g.ntn;
  const int mytiles = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const uint32_t ncols = (uint32_t)g.nacc * kTileN <= 64 ? 64u
                         : (uint32_t)g.nacc * kTileN <= 128 ? 128u
                         : (uint32_t)g.nacc * kTileN <= 256 ? 256u : 512u;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(tmem_full, 1);
    mbar_init(tmem_empty, kEpiWarps);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // copies: the K tile of every piece of both operands per stage, tile after tile
      int issued = 0;
      for (int i = 0; i < mytiles && !*abort_flag; ++i) {
        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
        const int tm = tile / g.ntn, tn = tile % g.ntn;
        for (int kt = 0; kt < g.nkt; ++kt) {
          const int t = i * g.nkt + kt;
          const int s = t % kStages, use = t / kStages;
          if (use > 0 && !mbar_wait(&empty[s], (uint32_t)(use - 1) & 1u)) {
            *abort_flag = 1;
            atomicOr(g.err, 1u);
            break;
          }
          if (*abort_flag) break;
          mbar_expect_tx(&full[s], Sh::kStageA + Sh::kStageB);
          // a 128-row A tile is the two adjacent 64-row blocks 2 tm, 2 tm + 1 of its K tile
          const long long aoff = ((long long)kt * g.nrt_a + 2 * tm) * Sh::kBlockBytes;
          const long long boff = ((long long)kt * g.nrt_b + tn) * Sh::kBlockBytes;
#pragma unroll
          for (int p = 0; p < kPieces; ++p)
            bulk_g2s(sa + s * Sh::kStageA + p * Sh::kTileABytes, g.a + p * g.a_piece + aoff, Sh::kTileABytes,
                     &full[s]);
#pragma unroll
          for (int p = 0; p < kPieces; ++p)
            bulk_g2s(sb + s * Sh::kStageB + p * Sh::kTileBBytes, g.b + p * g.b_piece + boff, Sh::kTileBBytes,
                     &full[s]);
          ++issued;
        }
      }
      // the copies of the last stages must have landed before the CTA may exit (on the normal
      // path these phases completed long ago; after an abort they bound the wait for them)
      for (int t = issued - kStages < 0 ? 0 : issued - kStages; t < issued; ++t)
        if (!mbar_wait(&full[t % kStages], (uint32_t)(t / kStages) & 1u)) atomicOr(g.err, 8u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMAs: every product of each stage, two 32-byte K steps each, into its accumulator
      for (int i = 0; i < mytiles && !*abort_flag; ++i) {
        // the epilogue has read the previous tile's accumulators
        if (i > 0 && !mbar_wait(tmem_empty, (uint32_t)(i - 1) & 1u)) {
          *abort_flag = 1;
          atomicOr(g.err, 16u);
          break;
        }
        tc_fence_after();
        bool ok = true;
        for (int kt = 0; kt < g.nkt; ++kt) {
          const int t = i * g.nkt + kt;
          const int s = t % kStages, use = t / kStages;
          if (!mbar_wait(&full[s], (uint32_t)use & 1u)) {
            *abort_flag = 1;
            atomicOr(g.err, 2u);
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t a_st = smem_u32(sa + s * Sh::kStageA), b_st = smem_u32(sb + s * Sh::kStageB);
          for (int p = 0; p < g.nprod; ++p) {
            const uint32_t dcol = tmem + (uint32_t)g.pacc[p] * kTileN;
            const bool first = kt == 0 && g.pfirst[p];
            const uint32_t a0 = a_st + (uint32_t)g.pa[p] * Sh::kTileABytes;
            const uint32_t b0 = b_st + (uint32_t)g.pb[p] * Sh::kTileBBytes;
#pragma unroll
            for (int k = 0; k < Sh::kKBytes / 32; ++k)
              mma<kKind>(dcol, smem_desc(a0 + k * 256, 128, Sh::kSbo), smem_desc(b0 + k * 256, 128, Sh::kSbo),
                         (first && k == 0) ? 0u : 1u);
          }
          mma_commit(&empty[s]);
        }
        if (!ok) break;
        mma_commit(tmem_full);  // arrives once every MMA of the tile has completed
      }
    }
  } else {
    // epilogue warps 2..9: warp w reads TMEM lanes 32 (w % 4) .. + 31 and columns 32 h .. + 31
    const int ew = warp - 2, quad = warp & 3, half = ew >> 2;
    for (int i = 0; i < mytiles; ++i) {
      const int tile = (int)blockIdx.x + i * (int)gridDim.x;
      const int tm = tile / g.ntn, tn = tile % g.ntn;
      const bool ok = mbar_wait(tmem_full, (uint32_t)i & 1u);
      tc_fence_after();
      // warp-uniform: tcgen05.ld is a whole-warp instruction
      if (!__all_sync(0xFFFFFFFFu, ok && !*abort_flag)) {
        if (lane == 0 && !ok) atomicOr(g.err, 4u);
        break;
      }
      __syncwarp();  // converged for the .sync.aligned TMEM loads
      const uint32_t base = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * 32);
      double v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = 0.0;
      for (int a = 0; a < g.nacc; ++a) {
        uint32_t r[32];
        tmem_ld32(base + (uint32_t)(a * kTileN), r);
        tmem_wait_ld();
        const double sc = g.acc_scale[a];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const double x = kKind == 0 ? (double)__uint_as_float(r[j]) : i32_to_f64(r[j]);
          v[j] += sc * x;
        }
      }
      // the accumulators are in registers: the next tile's MMAs may overwrite them
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_empty);
      const int row = tm * kTileM + quad * 32 + lane;
      if (row < g.M) {
        const int p = row / g.n, q = row % g.n;
        const int er = g.erow ? g.erow[row] : 0;
        double* out = g.out + (long long)p * g.n * g.n * g.n + (long long)q * g.n;
        // column rs of T -> offset r n^2 + s of [p][r][q][s], stepped from the first column
        const int c0 = tn * kTileN + half * 32;
        int r = c0 / g.n, sidx = c0 % g.n;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = c0 + j;
          if (col < g.N) {
            const int ec = g.ecol ? __ldg(g.ecol + col) : 0;
            out[(long long)r * g.n * g.n + sidx] = scale_pow2(v[j], er + ec);
          }
          if (++sidx == g.n) {
            sidx = 0;
            ++r;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

// ---------------------------------------------------------------------------------------
// Split kernels: FP64 factor F[k][row] (k < K, row < R; the K-major rows of the product) into
// pieces in one pre-tiled layout shared by both operands: piece c holds, for each 64-byte K
// tile kt and each 64-row block rt, the block's
// core matrices [row group of 8][16-byte K chunk][8 rows][16 bytes] at
// ((c * nkt + kt) * nrt + rt) * block bytes; rows are padded to a multiple of 128 with zeros, so
// a 128-row A tile is two adjacent 64-row blocks.
// ---------------------------------------------------------------------------------------
template <int kKind>
__device__ __forceinline__ long long chunk_offset(int row, int kc, int nrt) {
  constexpr int kChunks = kbytes_of(kKind) / 16;
  const int kt = kc / kChunks, c = kc % kChunks;
  return ((long long)kt * nrt + (row >> 6)) * block_bytes_of(kKind) + ((row & 63) >> 3) * sbo_of(kKind) + c * 128 +
         (row & 7) * 16;
}

// Per-row exponents e with max_k |F[k][row]| * 2^-e <= 1/2 (0 for an all-zero or padding row).
// A block takes 32 rows (one per lane, coalesced loads) and splits the K range over its 8
// warps; the per-warp maxima meet in shared memory.
__global__ void __launch_bounds__(256) row_exponent_kernel(const double* __restrict__ f, int K, int R, int rpad,
                                                           int* __restrict__ e) {
  __shared__ double part[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row = blockIdx.x * 32 + lane;
  double mx = 0.0;
  if (row < R)
    for (int k = warp; k < K; k += 8) mx = fmax(mx, fabs(f[(long long)k * R + row]));
  part[warp][lane] = mx;
  __syncthreads();
  if (warp == 0 && row < rpad) {
#pragma unroll
    for (int w = 1; w < 8; ++w) mx = fmax(mx, part[w][lane]);
    int ex = 0;
    if (mx > 0.0) {
      frexp(mx, &ex);   // mx = m 2^ex, m in [1/2, 1)
      ex += 1;          // mx 2^-ex in [1/4, 1/2)
    }
    e[row] = ex;
  }
}

// Ozaki slices of one 16-byte chunk (16 consecutive k of one row) per thread: x = F / 2^e
// (|x| <= 1/2), a_0 = rint(x 2^7), then a_i = rint(r_i 2^7) of the remainders (every slice fits
// a signed byte, |a_i| <= 64); one 16-byte store per slice.
__global__ void int8_slices_kernel(const double* __restrict__ f, int K, int R, int rpad, int nkt,
                                   const int* __restrict__ e, int S, long long piece_bytes, uint8_t* __restrict__ out) {
  const long long total = (long long)rpad * nkt * (kbytes_of(1) / 16);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t % rpad), kc = (int)(t / rpad);
    double x[16];
    const int ex = e[row];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int k = kc * 16 + j;
      x[j] = (row < R && k < K) ? ldexp(f[(long long)k * R + row], -ex) : 0.0;
    }
    const long long off = chunk_offset<1>(row, kc, rpad >> 6);
    for (int c = 0; c < S; ++c) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const double y = x[j] * 128.0;
        const double a = rint(y);
        x[j] = y - a;
        w[j >> 2] |= ((uint32_t)(int32_t)a & 0xFFu) << (8 * (j & 3));
      }
      *reinterpret_cast<uint4*>(out + c * piece_bytes + off) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// BF16 pieces hi, mid, lo (round to nearest at each step) of one 16-byte chunk (8 consecutive k
// of one row) per thread.
__global__ void bf16_pieces_kernel(const double* __restrict__ f, int K, int R, int rpad, int nkt,
                                   long long piece_bytes, uint8_t* __restrict__ out) {
  const long long total = (long long)rpad * nkt * (kbytes_of(0) / 16);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t % rpad), kc = (int)(t / rpad);
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = kc * 8 + j;
      x[j] = (row < R && k < K) ? f[(long long)k * R + row] : 0.0;
    }
    const long long off = chunk_offset<0>(row, kc, rpad >> 6);
    for (int c = 0; c < 3; ++c) {
      uint32_t w[4];
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        const __nv_bfloat16 h0 = __double2bfloat16(x[j]), h1 = __double2bfloat16(x[j + 1]);
        x[j] -= (double)__bfloat162float(h0);
        x[j + 1] -= (double)__bfloat162float(h1);
        w[j >> 1] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
      }
      *reinterpret_cast<uint4*>(out + c * piece_bytes + off) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

int pieces_of(int mode) { return mode == NW_TRANSFORM_CHOL_INT8 ? kOzakiSlices : 3; }

}  // namespace

size_t split_factor_bytes(int mode, int naux, int R) {
  const int kbytes = mode == NW_TRANSFORM_CHOL_INT8 ? naux : 2 * naux;
  const int kind = mode == NW_TRANSFORM_CHOL_INT8 ? 1 : 0, kb = kbytes_of(kind);
  const int nkt = (kbytes + kb - 1) / kb, rpad = (R + kTileM - 1) / kTileM * kTileM;
  return (size_t)pieces_of(mode) * nkt * (rpad / 64) * block_bytes_of(kind) + (size_t)rpad * sizeof(int) + 256;
}

cudaError_t split_factor(cudaStream_t st, int mode, const double* F, int naux, int R, void* buf, size_t bytes,
                         SplitFactor* out) {
  if (mode != NW_TRANSFORM_CHOL_INT8 && mode != NW_TRANSFORM_CHOL_BF16X6) return cudaErrorInvalidValue;
  if (bytes < split_factor_bytes(mode, naux, R)) return cudaErrorInvalidValue;
  const int kbytes = mode == NW_TRANSFORM_CHOL_INT8 ? naux : 2 * naux;
  SplitFactor f;
  f.mode = mode;
  f.R = R;
  f.rpad = (R + kTileM - 1) / kTileM * kTileM;
  const int kind = mode == NW_TRANSFORM_CHOL_INT8 ? 1 : 0, kb = kbytes_of(kind);
  f.nkt = (kbytes + kb - 1) / kb;
  f.piece_bytes = (long long)f.nkt * (f.rpad / 64) * block_bytes_of(kind);
  f.pieces = static_cast<uint8_t*>(buf);
  f.exps = reinterpret_cast<int*>(f.pieces + (size_t)pieces_of(mode) * f.piece_bytes);
  const long long chunks = (long long)f.rpad * f.nkt * (kb / 16);
  const int blocks = (int)std::min<long long>((chunks + 255) / 256, 148 * 16);
  if (mode == NW_TRANSFORM_CHOL_INT8) {
    row_exponent_kernel<<<(f.rpad + 31) / 32, 256, 0, st>>>(F, naux, R, f.rpad, f.exps);
    int8_slices_kernel<<<blocks, 256, 0, st>>>(F, naux, R, f.rpad, f.nkt, f.exps, kOzakiSlices, f.piece_bytes,
                                               f.pieces);
  } else {
    bf16_pieces_kernel<<<blocks, 256, 0, st>>>(F, naux, R, f.rpad, f.nkt, f.piece_bytes, f.pieces);
  }
  *out = f;
  return cudaGetLastError();
}

// T[p][r][q][s] = sum_k U[k][pq] V[k][rs] from two split factors (same mode) on tcgen05.
cudaError_t split_product(cudaStream_t st, const SplitFactor& A, const SplitFactor& B, int n, double* out,
                          uint32_t* err) {
  const int M = n * n, N = n * n;
  if (A.mode != B.mode || A.nkt != B.nkt || A.R != M || B.R != N) return cudaErrorInvalidValue;
  TcArgs g{};
  g.a = A.pieces;
  g.b = B.pieces;
  g.a_piece = A.piece_bytes;
  g.b_piece = B.piece_bytes;
  g.nkt = A.nkt;
  g.nrt_a = A.rpad / 64;
  g.nrt_b = B.rpad / 64;
  if (A.mode == NW_TRANSFORM_CHOL_INT8) {
    // products of slices i + j = s into accumulator s, for s < kOzakiSlices
    int np = 0;
    for (int s = 0; s < kOzakiSlices; ++s)
      for (int i = 0; i <= s; ++i) {
        g.pa[np] = (int8_t)i;
        g.pb[np] = (int8_t)(s - i);
        g.pacc[np] = (int8_t)s;
        ++np;
      }
    g.nprod = np;
    for (int p = 0; p < np; ++p) g.pfirst[p] = g.pa[p] == 0;  // (0, s) opens accumulator s
    g.nacc = kOzakiSlices;
    for (int s = 0; s < kOzakiSlices; ++s) g.acc_scale[s] = ldexp(1.0, -7 * (s + 2));
    g.erow = A.exps;
    g.ecol = B.exps;
  } else {
    // hi hi, hi mid, mid hi, hi lo, mid mid, lo hi: all into one FP32 accumulator
    static const int8_t pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
    for (int i = 0; i < 6; ++i) {
      g.pa[i] = pa[i];
      g.pb[i] = pb[i];
      g.pacc[i] = 0;
      g.pfirst[i] = i == 0;
    }
    g.nprod = 6;
    g.nacc = 1;
    g.acc_scale[0] = 1.0;
  }
  g.M = M;
  g.N = N;
  g.n = n;
  g.out = out;
  g.err = err;
  g.ntm = A.rpad / kTileM;
  g.ntn = B.rpad / kTileN;
  const int ntiles = g.ntm * g.ntn;
  const dim3 grid((unsigned)std::min(ntiles, 148));  // persistent: one CTA per SM
  cudaError_t e;
  if (A.mode == NW_TRANSFORM_CHOL_INT8) {
    e = cudaFuncSetAttribute(tc_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TcShape<1>::kSmem);
    if (e != cudaSuccess) return e;
    tc_gemm_kernel<1><<<grid, kTcThreads, TcShape<1>::kSmem, st>>>(g);
  } else {
    e = cudaFuncSetAttribute(tc_gemm_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TcShape<0>::kSmem);
    if (e != cudaSuccess) return e;
    tc_gemm_kernel<0><<<grid, kTcThreads, TcShape<0>::kSmem, st>>>(g);
  }
  return cudaGetLastError();
}

// Scratch of split_product_pqrs: both factors' pieces and exponents.
size_t split_product_scratch(int mode, int naux, int M, int N, int slices) {
  (void)slices;
  return split_factor_bytes(mode, naux, M) + split_factor_bytes(mode, naux, N);
}

// T[p][r][q][s] = sum_k U[k][pq] V[k][rs] with the split products on tcgen05 (both factors
// split here).
cudaError_t split_product_pqrs(cudaStream_t st, int mode, int slices, const double* U, const double* V, int naux, int n,
                               double* out, void* scratch, size_t scratch_bytes, uint32_t* err) {
  const int M = n * n, N = n * n;
  if (mode == NW_TRANSFORM_CHOL_INT8 && slices != kOzakiSlices) return cudaErrorInvalidValue;
  if (scratch_bytes < split_product_scratch(mode, naux, M, N, slices)) return cudaErrorInvalidValue;
  const size_t ba = split_factor_bytes(mode, naux, M);
  SplitFactor A, B;
  cudaError_t e = split_factor(st, mode, U, naux, M, scratch, ba, &A);
  if (e == cudaSuccess)
    e = split_factor(st, mode, V, naux, N, static_cast<char*>(scratch) + ba, scratch_bytes - ba, &B);
  if (e != cudaSuccess) return e;
  return split_product(st, A, B, n, out, err);
}

}  // namespace nw
