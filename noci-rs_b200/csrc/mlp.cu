// Small MLP of the learned QMC proposal: forward, backward and Adam kernels (FP32 compute,
// BF16 weight copies in the products, FP32 accumulation).  The network is tiny (din x 128,
// 128 x 128, 128 x nout) and runs once per training step and once per determinant when the
// proposal table is rebuilt, so one tiled product kernel serves every layer and pass; it runs
// on the tensor cores as split-TF32 mma.sync products.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.cuh"
#include "mlp.cuh"
#include "qmc_math.cuh"

namespace nw {
namespace {

constexpr int kT = 64;   // output tile
constexpr int kL = 16;   // reduction chunk
constexpr int kSplitMax = 32;  // k-split blocks of a weight-gradient product
constexpr int kPrefetch = 8;   // reduction chunks whose panels one block loads at once

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

enum Epi { kPlain = 0, kBiasRelu = 1, kBias = 2, kReluMask = 3 };

// TF32 tensor-core product with a split of each operand into a TF32 head and a TF32 tail:
// a b = a_h b_h + a_h b_t + a_t b_h + O(2^-22 |a b|), three m16n8k8 MMAs per step with FP32
// accumulation, so the products keep FP32-class accuracy (the BF16 weight copies are exact
// TF32 heads with a zero tail).
__device__ __forceinline__ void split_tf32(float x, uint32_t& h, uint32_t& t) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  const float r = x - __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(r));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
               "{%0, %1, %2, %3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M x N] = epi(A[M x L] B[L x N]); A[i][l] = A[i * asr + l * asc], B[l][j] = B[l * bsr + j * bsc].
// With gridDim.z > 1 the reduction range is split: block z covers [z * lsplit, (z + 1) * lsplit)
// and writes its plain partial product to C + z * M * ldc (summed by splitk_sum_kernel).
// A 64 x 64 tile per block of 8 warps (4 along M x 2 along N, each 16 x 32: four m16n8 tiles);
// the panels are staged in shared memory k-major.
template <typename TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int L, const float* __restrict__ A, long asr, long asc,
                                                   const TB* __restrict__ B, long bsr, long bsc, float* __restrict__ C,
                                                   int ldc, int epi, const float* __restrict__ bias,
                                                   const float* __restrict__ mask, int lsplit) {
  __shared__ float As[kL][kT + 8];  // row stride 72 floats: the fragment loads hit 32 distinct banks
  __shared__ float Bs[kL][kT + 8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
  const int row0 = blockIdx.y * kT, col0 = blockIdx.x * kT;
  const int lbeg = blockIdx.z * lsplit, lend = min(L, lbeg + lsplit);
  C += (size_t)blockIdx.z * M * ldc;
  float acc[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.0f;
  // The panels of up to kPrefetch chunks are loaded into registers at once (every load in
  // flight together: one memory latency per kPrefetch chunks instead of one per chunk, which
  // set the pace of these small products), then staged chunk by chunk.
  constexpr int kPer = kT * kL / 256;  // elements of a panel per thread and chunk (4)
  for (int p0 = lbeg; p0 < lend; p0 += kL * kPrefetch) {
    float ra[kPrefetch][kPer], rb[kPrefetch][kPer];
#pragma unroll
    for (int ch = 0; ch < kPrefetch; ++ch) {
      const int l0 = p0 + ch * kL;
#pragma unroll
      for (int i = 0; i < kPer; ++i) {
        const int e = threadIdx.x + 256 * i;
        const int ar = e / kL, ac = e % kL, agr = row0 + ar, agc = l0 + ac;
        ra[ch][i] = (agr < M && agc < lend) ? A[agr * asr + agc * asc] : 0.0f;
        const int br = e / kT, bc = e % kT, bgr = l0 + br, bgc = col0 + bc;
        rb[ch][i] = (bgr < lend && bgc < N) ? to_f(B[bgr * bsr + bgc * bsc]) : 0.0f;
      }
    }
#pragma unroll
    for (int ch = 0; ch < kPrefetch; ++ch) {
    if (p0 + ch * kL >= lend) break;  // block-uniform
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int e = threadIdx.x + 256 * i;
      As[e % kL][e / kL] = ra[ch][i];
      Bs[e / kT][e % kT] = rb[ch][i];
    }
    __syncthreads();
#pragma unroll
    for (int k0 = 0; k0 < kL; k0 += 8) {
      uint32_t ah[4], at[4];
      split_tf32(As[k0 + t][wm + g], ah[0], at[0]);
      split_tf32(As[k0 + t][wm + g + 8], ah[1], at[1]);
      split_tf32(As[k0 + t + 4][wm + g], ah[2], at[2]);
      split_tf32(As[k0 + t + 4][wm + g + 8], ah[3], at[3]);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        uint32_t bh[2], bt[2];
        split_tf32(Bs[k0 + t][wn + j * 8 + g], bh[0], bt[0]);
        split_tf32(Bs[k0 + t + 4][wn + j * 8 + g], bh[1], bt[1]);
        mma_tf32(acc[j], at, bh);
        mma_tf32(acc[j], ah, bt);
        mma_tf32(acc[j], ah, bh);
      }
    }
    __syncthreads();
    }
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = row0 + wm + g + (e >> 1) * 8, c = col0 + wn + j * 8 + 2 * t + (e & 1);
      if (r >= M || c >= N) continue;
      float v = acc[j][e];
      if (epi == kBiasRelu) v = fmaxf(v + bias[c], 0.0f);
      if (epi == kBias) v += bias[c];
      if (epi == kReluMask) v = mask[(size_t)r * ldc + c] > 0.0f ? v : 0.0f;
      C[(size_t)r * ldc + c] = v;
    }
}

// C[i] = sum_z P[z][i] over the k-split partial products (fixed order).
__global__ void splitk_sum_kernel(const float* __restrict__ part, int splits, size_t count, float* __restrict__ c) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * count + i];
    c[i] = s;
  }
}

// Partial column sums of a B x N matrix: block (x, y) sums rows [y * rows, (y + 1) * rows) of
// columns 32x .. 32x + 31 (32 columns x 8 row groups, coalesced across the columns) into
// out[y * N + j]; splitk_sum_kernel adds the row splits in a fixed order.
__global__ void __launch_bounds__(256) colsum_kernel(const float* __restrict__ x, int B, int N, int rows,
                                                     float* __restrict__ out) {
  __shared__ float part[8][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + tx;
  const int r0 = blockIdx.y * rows, r1 = min(B, r0 + rows);
  float s = 0.0f;
  if (j < N)
    for (int r = r0 + ty; r < r1; r += 8) s += x[(size_t)r * N + j];
  part[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && j < N) {
    float t = 0.0f;
#pragma unroll
    for (int g = 0; g < 8; ++g) t += part[g][tx];
    out[(size_t)blockIdx.y * N + j] = t;
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ p, size_t n, __nv_bfloat16* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(p[i]);
}

template <typename TB>
nw_status gemm(nw_ctx* ctx, int M, int N, int L, const float* A, long asr, long asc, const TB* B, long bsr, long bsc,
               float* C, int ldc, int epi, const float* bias, const float* mask, cudaStream_t s) {
  const dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT);
  gemm_kernel<TB><<<grid, 256, 0, s>>>(M, N, L, A, asr, asc, B, bsr, bsc, C, ldc, epi, bias, mask, L);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

// Weight gradients (few output tiles, long reduction over the batch): the reduction is split
// over kSplitMax blocks along z into m->part, then summed in a fixed order.
nw_status gemm_splitk(nw_ctx* ctx, Mlp* m, int M, int N, int L, const float* A, long asr, long asc, const float* B,
                      long bsr, long bsc, float* C, cudaStream_t s) {
  const int lsplit = std::max(kL, (L + kSplitMax - 1) / kSplitMax + kL - 1) / kL * kL;
  const int splits = (L + lsplit - 1) / lsplit;
  const dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT, splits);
  gemm_kernel<float><<<grid, 256, 0, s>>>(M, N, L, A, asr, asc, B, bsr, bsc, m->part, N, kPlain, nullptr, nullptr, lsplit);
  const size_t count = (size_t)M * N;
  splitk_sum_kernel<<<(int)std::min<size_t>((count + 255) / 256, 1184), 256, 0, s>>>(m->part, splits, count, C);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

// out[j] = sum_r X[r][j] through the split buffer m->part.
nw_status colsum(nw_ctx* ctx, Mlp* m, const float* x, int B, int N, float* out, cudaStream_t s) {
  const int rows = std::max(8, (B + kSplitMax - 1) / kSplitMax);
  const int splits = (B + rows - 1) / rows;
  colsum_kernel<<<dim3((N + 31) / 32, splits), 256, 0, s>>>(x, B, N, rows, m->part);
  splitk_sum_kernel<<<(N + 255) / 256, 256, 0, s>>>(m->part, splits, (size_t)N, out);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

// Descriptor of a determinant (din floats, zero-padded): one-hot parent reference, one-hot
// alpha and beta excitation ranks (0..4), and per spin the indicator of the orbitals whose
// occupation the excitation changes (its holes and particles).
__global__ void feature_kernel(const nw_det* __restrict__ dets, const uint32_t* __restrict__ rows, uint32_t row0,
                               int B, int din, int nref, int nmo, float* __restrict__ x) {
  const int r = blockIdx.x;
  if (r >= B) return;
  float* xr = x + (size_t)r * din;
  for (int j = threadIdx.x; j < din; j += blockDim.x) xr[j] = 0.0f;
  __syncthreads();
  if (threadIdx.x != 0) return;
  const uint32_t g = rows ? rows[r] : row0 + (uint32_t)r;
  const nw_det d = dets[g];
  xr[d.parent] = 1.0f;
  xr[nref + d.rank_a] = 1.0f;
  xr[nref + 5 + d.rank_b] = 1.0f;
  const int base_a = nref + 10, base_b = nref + 10 + nmo;
  for (int k = 0; k < d.rank_a; ++k) {
    xr[base_a + d.idx_a[k]] = 1.0f;
    xr[base_a + d.idx_a[4 + k]] = 1.0f;
  }
  for (int k = 0; k < d.rank_b; ++k) {
    xr[base_b + d.idx_b[k]] = 1.0f;
    xr[base_b + d.idx_b[4 + k]] = 1.0f;
  }
}

}  // namespace

int mlp_descriptor_width(int nref, int nmo) { return ((nref + 10 + 2 * nmo) + 31) / 32 * 32; }

nw_status mlp_features(nw_ctx* ctx, Mlp* m, const nw_det* dets, const uint32_t* rows, uint32_t row0, int B,
                       cudaStream_t s) {
  if (B < 1 || B > m->bcap || m->din < mlp_descriptor_width(ctx->nref, ctx->nmo))
    return fail(ctx, NW_ERR_INVALID, "descriptor batch does not fit the network");
  feature_kernel<<<B, 128, 0, s>>>(dets, rows, row0, B, m->din, ctx->nref, ctx->nmo, m->x);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

size_t mlp_param_count(int din, int nout) {
  return (size_t)kMlpWidth * din + kMlpWidth + (size_t)kMlpWidth * kMlpWidth + kMlpWidth + (size_t)nout * kMlpWidth +
         nout;
}

nw_status mlp_create(nw_ctx* ctx, Mlp* m, int din, int nout, int bcap, uint64_t seed) {
  m->din = din;
  m->nout = nout;
  m->bcap = bcap;
  m->nparams = mlp_param_count(din, nout);
  const size_t np = m->nparams;
  float** bufs[] = {&m->params, &m->grads, &m->adam_m, &m->adam_v};
  for (float** b : bufs)
    if (cudaMalloc(b, sizeof(float) * np) != cudaSuccess) return fail(ctx, NW_ERR_ALLOC, "MLP parameters");
  if (cudaMalloc(&m->wbf, sizeof(__nv_bfloat16) * np) != cudaSuccess) return fail(ctx, NW_ERR_ALLOC, "MLP weights");
  const size_t part = (size_t)kSplitMax * kMlpWidth * std::max(std::max(din, nout), kMlpWidth);
  if (cudaMalloc(&m->part, sizeof(float) * part) != cudaSuccess) return fail(ctx, NW_ERR_ALLOC, "MLP split-k partials");
  struct Act {
    float** p;
    size_t n;
  } acts[] = {{&m->x, (size_t)bcap * din},   {&m->h1, (size_t)bcap * kMlpWidth}, {&m->h2, (size_t)bcap * kMlpWidth},
              {&m->z, (size_t)bcap * nout}, {&m->d2, (size_t)bcap * kMlpWidth}, {&m->d1, (size_t)bcap * kMlpWidth}};
  for (const Act& a : acts)
    if (cudaMalloc(a.p, sizeof(float) * std::max<size_t>(a.n, 1)) != cudaSuccess)
      return fail(ctx, NW_ERR_ALLOC, "MLP activations");
  // uniform +-sqrt(6 / fan_in) weights, zero biases
  std::vector<float> h(np, 0.0f);
  struct Blk {
    size_t off, n;
    int fan_in;
  } w[] = {{m->off_w1(), (size_t)kMlpWidth * din, din},
           {m->off_w2(), (size_t)kMlpWidth * kMlpWidth, kMlpWidth},
           {m->off_w3(), (size_t)nout * kMlpWidth, kMlpWidth}};
  for (const Blk& b : w) {
    const double a = std::sqrt(6.0 / b.fan_in);
    for (size_t i = 0; i < b.n; ++i) h[b.off + i] = (float)((2.0 * nwq::uniform1(seed, 0, b.off + i, 7) - 1.0) * a);
  }
  NW_CUDA(ctx, cudaMemcpy(m->params, h.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemset(m->adam_m, 0, sizeof(float) * np));
  NW_CUDA(ctx, cudaMemset(m->adam_v, 0, sizeof(float) * np));
  NW_CUDA(ctx, cudaMemset(m->grads, 0, sizeof(float) * np));
  m->adam_t = 0;
  return mlp_sync_bf16(ctx, m, nullptr);
}

void mlp_destroy(Mlp* m) {
  void* bufs[] = {m->params, m->grads, m->adam_m, m->adam_v, m->wbf, m->x, m->h1, m->h2, m->z, m->d2, m->d1, m->part};
  for (void* p : bufs)
    if (p) cudaFree(p);
  *m = Mlp{};
}

nw_status mlp_sync_bf16(nw_ctx* ctx, Mlp* m, cudaStream_t s) {
  to_bf16_kernel<<<256, 256, 0, s>>>(m->params, m->nparams, m->wbf);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

nw_status mlp_forward(nw_ctx* ctx, Mlp* m, int B, cudaStream_t s) {
  const int W = kMlpWidth;
  const float* P = m->params;
  nw_status st = gemm(ctx, B, W, m->din, m->x, m->din, 1, m->wbf + m->off_w1(), 1, m->din, m->h1, W, kBiasRelu,
                      P + m->off_b1(), nullptr, s);
  if (st == NW_OK)
    st = gemm(ctx, B, W, W, m->h1, W, 1, m->wbf + m->off_w2(), 1, W, m->h2, W, kBiasRelu, P + m->off_b2(), nullptr, s);
  if (st == NW_OK)
    st = gemm(ctx, B, m->nout, W, m->h2, W, 1, m->wbf + m->off_w3(), 1, W, m->z, m->nout, kBias, P + m->off_b3(),
              nullptr, s);
  return st;
}

nw_status mlp_backward(nw_ctx* ctx, Mlp* m, int B, cudaStream_t s) {
  const int W = kMlpWidth, K = m->nout, D = m->din;
  float* G = m->grads;
  // layer 3: dW3 = dZ^T H2, db3 = colsum dZ, d2 = (dZ W3) o [H2 > 0]
  nw_status st = gemm_splitk(ctx, m, K, W, B, m->z, 1, K, m->h2, W, 1, G + m->off_w3(), s);
  if (st == NW_OK) st = colsum(ctx, m, m->z, B, K, G + m->off_b3(), s);
  if (st == NW_OK)
    st = gemm(ctx, B, W, K, m->z, K, 1, m->wbf + m->off_w3(), W, 1, m->d2, W, kReluMask, nullptr, m->h2, s);
  // layer 2
  if (st == NW_OK) st = gemm_splitk(ctx, m, W, W, B, m->d2, 1, W, m->h1, W, 1, G + m->off_w2(), s);
  if (st == NW_OK) st = colsum(ctx, m, m->d2, B, W, G + m->off_b2(), s);
  if (st == NW_OK)
    st = gemm(ctx, B, W, W, m->d2, W, 1, m->wbf + m->off_w2(), W, 1, m->d1, W, kReluMask, nullptr, m->h1, s);
  // layer 1
  if (st == NW_OK) st = gemm_splitk(ctx, m, W, D, B, m->d1, 1, W, m->x, D, 1, G + m->off_w1(), s);
  if (st == NW_OK) st = colsum(ctx, m, m->d1, B, W, G + m->off_b1(), s);
  if (st == NW_OK) NW_CUDA(ctx, cudaGetLastError());
  return st;
}

nw_status mlp_adam(nw_ctx* ctx, Mlp* m, float lr, cudaStream_t s) {
  m->adam_t += 1;
  const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, m->adam_t)));
  const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, m->adam_t)));
  adam_kernel<<<256, 256, 0, s>>>(m->params, m->grads, m->adam_m, m->adam_v, m->nparams, lr, c1, c2);
  NW_CUDA(ctx, cudaGetLastError());
  return mlp_sync_bf16(ctx, m, s);
}

}  // namespace nw
