// FP64 GEMM of the intermediate build on the B200's FP64 tensor cores.
//
// The build's dense products (X/Y, the partial transforms cx/xc, J/K contractions, F/V
// intermediates, the quarter steps of the four-index transforms behind the J and II tensors,
// src/nonorthogonalwicks/build.rs:198-313,526-683,808-917 and src/maths/eri.rs:258) are FP64
// GEMMs: row-major C (M x N) = alpha op(A) op(B) + beta C, strided-batched.  tcgen05.mma has
// no FP64 kind, so on sm_100a the FP64 tensor path is the DMMA instruction
// mma.sync.aligned.m16n8k16.row.col.f64, issued here per warp.
//
// Tiling: a 64 x 64 tile of C per block of 128 threads (2 x 2 warps of 32 x 32, i.e. 2 x 4
// DMMA tiles of 16 x 8 per warp, 32 FP64 accumulators per thread), one m16n8k16 DMMA per tile
// and 16-deep K panel.  Panels move global -> shared with 8-byte cp.async (zero-fill past the
// matrix edges, so any M, N, K) through a three-stage ring, so two panels are in flight while
// the third feeds the tensor cores.  Each operand's panel keeps the operand's own contiguous
// direction (k-major rows of 16 + 4 doubles, or m/n-major rows of 64 + 4 doubles): the copies
// are coalesced, and the padded strides make every fragment load of a warp conflict-free.
// Operands may be transposed (op = ^T, a template parameter) and either batch stride may be 0
// (a shared operand).
#include <cuda_runtime.h>

#include "internal.cuh"

namespace nw {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;
constexpr int kThreads = 128;
constexpr int kStages = 3;
constexpr int kLdK = kBK + 4;   // k-contiguous panel rows (16 + 4 doubles)
constexpr int kLdMN = kBM + 4;  // m- or n-contiguous panel rows (64 + 4 doubles)
constexpr int kPanel = kBM * kLdK > kBK * kLdMN ? kBM * kLdK : kBK * kLdMN;  // doubles per panel
constexpr size_t kSmem = (size_t)kStages * 2 * kPanel * sizeof(double);

__device__ __forceinline__ void dmma16816(double (&d)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7, %8, %9, %10, %11}, "
      "{%12, %13, %14, %15}, {%0, %1, %2, %3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
        "d"(b[2]), "d"(b[3]));
}

// 8-byte asynchronous copy global -> shared; src_bytes = 0 writes a zero.
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

struct GemmArgs {
  const double* A;
  const double* B;
  double* C;
  long long sa, sb, sc;   // batch strides (elements)
  int M, N, K, lda, ldb, ldc;
  double alpha, beta;
};

// Panel element (i, k) of a kRows x kBK panel: row-major over k when the operand is k-contiguous
// in memory (KC), else k-major over the rows.
template <bool KC>
__device__ __forceinline__ int panel_index(int i, int k) {
  return KC ? i * kLdK + k : k * kLdMN + i;
}

// Issue the copies of K panel kt of op(A) (rows m0..) and op(B) (columns n0..) into stage st.
// TA: A stored K x M (m contiguous); TB: B stored N x K (k contiguous).
template <bool TA, bool TB>
__device__ __forceinline__ void load_panels(const GemmArgs& g, const double* A, const double* B, int m0, int n0,
                                            int kt, double* as, double* bs) {
  const int tid = threadIdx.x, k0 = kt * kBK;
#pragma unroll
  for (int u = 0; u < kBM * kBK / kThreads; ++u) {
    const int e = tid + u * kThreads;
    // consecutive threads take consecutive addresses of the operand's contiguous index
    const int m = TA ? e % kBM : e / kBK, k = TA ? e / kBM : e % kBK;
    const int gm = m0 + m, gk = k0 + k;
    const bool ok = gm < g.M && gk < g.K;
    const double* src = ok ? A + (TA ? (long long)gk * g.lda + gm : (long long)gm * g.lda + gk) : A;
    cp_async8(as + panel_index<!TA>(m, k), src, ok);
  }
#pragma unroll
  for (int u = 0; u < kBN * kBK / kThreads; ++u) {
    const int e = tid + u * kThreads;
    const int n = TB ? e / kBK : e % kBN, k = TB ? e % kBK : e / kBN;
    const int gn = n0 + n, gk = k0 + k;
    const bool ok = gn < g.N && gk < g.K;
    const double* src = ok ? B + (TB ? (long long)gn * g.ldb + gk : (long long)gk * g.ldb + gn) : B;
    cp_async8(bs + panel_index<TB>(n, k), src, ok);
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(kThreads) dgemm_kernel(GemmArgs g) {
  extern __shared__ __align__(16) double dsm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int grp = lane >> 2, tig = lane & 3;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const long long bz = blockIdx.z;
  const double* __restrict__ A = g.A + bz * g.sa;
  const double* __restrict__ B = g.B + bz * g.sb;
  double* __restrict__ C = g.C + bz * g.sc;
  const int nk = (g.K + kBK - 1) / kBK;

  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 4; ++h) acc[i][j][h] = 0.0;

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) load_panels<TA, TB>(g, A, B, m0, n0, s, dsm + (2 * s) * kPanel, dsm + (2 * s + 1) * kPanel);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<kStages - 2>();  // panel kt has landed (this thread's copies)
    __syncthreads();               // ... and every thread's; stage (kt - 1) % kStages is free
    {
      const int nx = kt + kStages - 1, st = nx % kStages;
      if (nx < nk) load_panels<TA, TB>(g, A, B, m0, n0, nx, dsm + (2 * st) * kPanel, dsm + (2 * st + 1) * kPanel);
      cp_async_commit();
    }
    const int st = kt % kStages;
    const double* as = dsm + (2 * st) * kPanel;
    const double* bs = dsm + (2 * st + 1) * kPanel;
    // fragments: A[row grp + 8 (i % 2)][col tig + 4 (i / 2)], B[row tig + 4 i][col grp]
    double af[2][8], bf[4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        af[mt][i] = as[panel_index<!TA>(wm + mt * 16 + grp + 8 * (i & 1), tig + 4 * (i >> 1))];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) bf[nt][i] = bs[panel_index<TB>(wn + nt * 8 + grp, tig + 4 * i)];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma16816(acc[mt][nt], af[mt], bf[nt]);
  }
  cp_async_wait<0>();
  // D fragment: rows grp, grp + 8 and columns 2 tig, 2 tig + 1 of each 16 x 8 tile
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const int gm = m0 + wm + mt * 16 + grp + 8 * (h >> 1), gn = n0 + wn + nt * 8 + 2 * tig + (h & 1);
        if (gm < g.M && gn < g.N) {
          double* c = C + (long long)gm * g.ldc + gn;
          const double v = g.alpha * acc[mt][nt][h];
          *c = g.beta == 0.0 ? v : v + g.beta * *c;
        }
      }
}

template <bool TA, bool TB>
cudaError_t launch(cudaStream_t stream, const GemmArgs& g, dim3 grid) {
  // the three-stage ring is above the 48 KB default; raised once per device
  static bool raised[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !raised[dev]) {
    e = cudaFuncSetAttribute(dgemm_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) raised[dev] = true;
  }
  dgemm_kernel<TA, TB><<<grid, kThreads, kSmem, stream>>>(g);
  return cudaGetLastError();
}

}  // namespace

cudaError_t dgemm_strided(cudaStream_t stream, bool ta, bool tb, int M, int N, int K, double alpha, const double* A,
                          int lda, long long sa, const double* B, int ldb, long long sb, double beta, double* C,
                          int ldc, long long sc, int batch) {
  if (M <= 0 || N <= 0 || batch <= 0) return cudaSuccess;
  if (K <= 0) return cudaErrorInvalidValue;
  const long long gx = (N + kBN - 1) / kBN, gy = (M + kBM - 1) / kBM;
  if (gy > 65535 || batch > 65535 || gx > 0x7FFFFFFFll) return cudaErrorInvalidValue;
  GemmArgs g{A, B, C, sa, sb, sc, M, N, K, lda, ldb, ldc, alpha, beta};
  const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)batch);
  if (ta) return tb ? launch<true, true>(stream, g, grid) : launch<true, false>(stream, g, grid);
  return tb ? launch<false, true>(stream, g, grid) : launch<false, false>(stream, g, grid);
}

}  // namespace nw

// FP64 GEMM entry point (see the header): row-major, strided-batched, on the caller's stream.
extern "C" nw_status nw_dgemm(int trans_a, int trans_b, int m, int n, int k, double alpha, const double* a, int lda,
                              long long stride_a, const double* b, int ldb, long long stride_b, double beta, double* c,
                              int ldc, long long stride_c, int batch, void* stream) {
  if (!a || !b || !c || m < 0 || n < 0 || k < 0 || batch < 0) return NW_ERR_INVALID;
  const cudaError_t e = nw::dgemm_strided(static_cast<cudaStream_t>(stream), trans_a != 0, trans_b != 0, m, n, k,
                                          alpha, a, lda, stride_a, b, ldb, stride_b, beta, c, ldc, stride_c, batch);
  if (e == cudaErrorInvalidValue) return NW_ERR_INVALID;
  return e == cudaSuccess ? NW_OK : NW_ERR_CUDA;
}
