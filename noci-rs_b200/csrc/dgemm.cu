// FP64 GEMM of the intermediate build on the B200's FP64 tensor cores.
//
// The build's dense products (X/Y, the partial transforms cx/xc, J/K contractions, F/V
// intermediates, the quarter steps of the four-index transforms behind the J and II tensors,
// src/nonorthogonalwicks/build.rs:198-313,526-683,808-917 and src/maths/eri.rs:258) are FP64
// GEMMs: row-major C (M x N) = alpha op(A) op(B) + beta C, strided-batched.  tcgen05.mma has
// no FP64 kind, so on sm_100a the FP64 tensor path is the DMMA instruction
// mma.sync.aligned.m8n8k4.row.col.f64, issued here per warp.
//
// Tiling: a 64 x 64 tile of C per block of 128 threads (2 x 2 warps of 32 x 32, i.e. 4 x 4
// DMMA tiles of 8 x 8 per warp, 32 FP64 accumulators per thread), K in steps of 16 staged
// through shared memory as [k][m] and [k][n] panels (both operands k-major, so each lane's
// fragment element is one aligned 8-byte load), with the next panel's global loads in flight
// in registers while the current panel feeds the tensor cores.  Operands may be transposed
// (op = ^T) and either batch stride may be 0 (a shared operand); edges are zero-filled, so any
// M, N, K is accepted.
#include <cuda_runtime.h>

#include "internal.cuh"

namespace nw {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 16;
constexpr int kThreads = 128;
constexpr int kPad = 8;                  // panel row stride kBM + 8 doubles: fragment loads of a
constexpr int kLdA = kBM + kPad;         // warp touch each bank pair at most twice
constexpr int kLdB = kBN + kPad;
constexpr int kPerThreadA = kBM * kBK / kThreads;  // 8
constexpr int kPerThreadB = kBK * kBN / kThreads;  // 8

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

struct GemmArgs {
  const double* A;
  const double* B;
  double* C;
  long long sa, sb, sc;   // batch strides (elements)
  int M, N, K, lda, ldb, ldc;
  double alpha, beta;
  int ta, tb;
};

// Element e of the A panel (kBM x kBK of op(A)) at k-tile k0: its (m, k) inside the tile.  The
// mapping follows the operand's contiguous index so that a warp's loads are consecutive.
__device__ __forceinline__ void a_coord(int e, int ta, int* m, int* k) {
  if (ta) {  // A stored K x M: m contiguous
    *k = e / kBM;
    *m = e % kBM;
  } else {   // A stored M x K: k contiguous
    *m = e / kBK;
    *k = e % kBK;
  }
}

__device__ __forceinline__ void b_coord(int e, int tb, int* k, int* n) {
  if (tb) {  // B stored N x K: k contiguous
    *n = e / kBK;
    *k = e % kBK;
  } else {   // B stored K x N: n contiguous
    *k = e / kBN;
    *n = e % kBN;
  }
}

__global__ void __launch_bounds__(kThreads) dgemm_kernel(GemmArgs g) {
  __shared__ double As[kBK][kLdA];
  __shared__ double Bs[kBK][kLdB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int grp = lane >> 2, tig = lane & 3;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const long long bz = blockIdx.z;
  const double* __restrict__ A = g.A + bz * g.sa;
  const double* __restrict__ B = g.B + bz * g.sb;
  double* __restrict__ C = g.C + bz * g.sc;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  double ra[kPerThreadA], rb[kPerThreadB];
  auto load = [&](int k0) {
#pragma unroll
    for (int u = 0; u < kPerThreadA; ++u) {
      int m, k;
      a_coord(tid + u * kThreads, g.ta, &m, &k);
      const int gm = m0 + m, gk = k0 + k;
      ra[u] = (gm < g.M && gk < g.K) ? __ldg(A + (g.ta ? (long long)gk * g.lda + gm : (long long)gm * g.lda + gk))
                                     : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kPerThreadB; ++u) {
      int k, n;
      b_coord(tid + u * kThreads, g.tb, &k, &n);
      const int gn = n0 + n, gk = k0 + k;
      rb[u] = (gn < g.N && gk < g.K) ? __ldg(B + (g.tb ? (long long)gn * g.ldb + gk : (long long)gk * g.ldb + gn))
                                     : 0.0;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int u = 0; u < kPerThreadA; ++u) {
      int m, k;
      a_coord(tid + u * kThreads, g.ta, &m, &k);
      As[k][m] = ra[u];
    }
#pragma unroll
    for (int u = 0; u < kPerThreadB; ++u) {
      int k, n;
      b_coord(tid + u * kThreads, g.tb, &k, &n);
      Bs[k][n] = rb[u];
    }
  };

  load(0);
  for (int k0 = 0; k0 < g.K; k0 += kBK) {
    store();
    __syncthreads();
    if (k0 + kBK < g.K) load(k0 + kBK);  // next panel's loads overlap this panel's DMMAs
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = As[kk + tig][wm + i * 8 + grp];   // A[row grp][col tig]
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bs[kk + tig][wn + j * 8 + grp];   // B[row tig][col grp]
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }
  // D fragment: row grp, columns 2 tig, 2 tig + 1 of each 8 x 8 tile
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gm = m0 + wm + i * 8 + grp, gn = n0 + wn + j * 8 + 2 * tig + h;
        if (gm < g.M && gn < g.N) {
          double* c = C + (long long)gm * g.ldc + gn;
          const double v = g.alpha * acc[i][j][h];
          *c = g.beta == 0.0 ? v : v + g.beta * *c;
        }
      }
}

}  // namespace

cudaError_t dgemm_strided(cudaStream_t stream, bool ta, bool tb, int M, int N, int K, double alpha, const double* A,
                          int lda, long long sa, const double* B, int ldb, long long sb, double beta, double* C,
                          int ldc, long long sc, int batch) {
  if (M <= 0 || N <= 0 || batch <= 0) return cudaSuccess;
  if (K <= 0) return cudaErrorInvalidValue;
  const long long gx = (N + kBN - 1) / kBN, gy = (M + kBM - 1) / kBM;
  if (gy > 65535 || batch > 65535 || gx > 0x7FFFFFFFll) return cudaErrorInvalidValue;
  GemmArgs g{A, B, C, sa, sb, sc, M, N, K, lda, ldb, ldc, alpha, beta, ta ? 1 : 0, tb ? 1 : 0};
  dgemm_kernel<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)batch), kThreads, 0, stream>>>(g);
  return cudaGetLastError();
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
