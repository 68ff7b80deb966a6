// Learned SNOCI candidate screener (nw_screen_*): an MLP din -> 128 -> 128 -> 1 over the
// determinant descriptor of csrc/mlp.cu regresses the standardised log10 of the NOCI-PT2
// selection score |a_a V_a| (src/snoci/step.rs:436-441) of candidates that were scored
// exactly.  Trained on the GPU by the MLP kernels with a mean-squared-error loss; its
// predictions rank a candidate pool so that only the highest-ranked part enters the
// candidate matrix M and GMRES.  No counterpart in the reference, which scores every
// candidate (exhaustive screening).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"
#include "mlp.cuh"
#include "qmc_math.cuh"

namespace {

constexpr int kScreenBatch = 4096;

// Random minibatch (with replacement) of the training rows.
__global__ void screen_batch_kernel(const uint32_t* __restrict__ idx, const float* __restrict__ target, uint64_t n,
                                    uint64_t seed, uint64_t step, int B, uint32_t* __restrict__ rows,
                                    float* __restrict__ t) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  uint64_t k = (uint64_t)(nwq::uniform1(seed, step, (uint64_t)r, nwq::kDrawTrain) * (double)n);
  if (k >= n) k = n - 1;
  rows[r] = idx[k];
  t[r] = target[k];
}

// z[r] <- dL/dz[r] of L = mean_r (z_r - t_r)^2; the loss goes to *loss.
__global__ void mse_kernel(float* __restrict__ z, const float* __restrict__ t, int B, double* __restrict__ loss) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int r = threadIdx.x; r < B; r += blockDim.x) {
    const float d = z[r] - t[r];
    acc += (double)d * (double)d;
    z[r] = 2.0f * d / (float)B;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (double)B;
}

}  // namespace

struct nw_screen {
  nw_ctx* ctx = nullptr;
  nw::Mlp mlp{};
  uint64_t seed = 0;
  double mean = 0.0, scale = 1.0;  // target standardisation
  bool trained = false;
  uint32_t* rows = nullptr;
  float* t = nullptr;
  double* loss = nullptr;
};

namespace {

nw_status sfail(nw_screen* s, nw_status st, const std::string& m) { return nw::fail(s->ctx, st, m); }

void screen_release(nw_screen* s) {
  nw::mlp_destroy(&s->mlp);
  if (s->rows) cudaFree(s->rows);
  if (s->t) cudaFree(s->t);
  if (s->loss) cudaFree(s->loss);
  delete s;
}

nw_status check_rows(nw_screen* s, const uint32_t* idx, uint64_t n) {
  nw_ctx* ctx = s->ctx;
  if (!ctx->d_dets) return sfail(s, NW_ERR_STATE, "no determinant basis set");
  for (uint64_t i = 0; i < n; ++i)
    if (idx[i] >= ctx->ndet) return sfail(s, NW_ERR_INVALID, "determinant index out of range");
  return NW_OK;
}

}  // namespace

extern "C" {

nw_status nw_screen_create(nw_ctx* ctx, uint64_t seed, nw_screen** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!ctx) return NW_ERR_INVALID;
  if (!ctx->built) return nw::fail(ctx, NW_ERR_STATE, "intermediates not built");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw_screen* s = new (std::nothrow) nw_screen;
  if (!s) return NW_ERR_ALLOC;
  s->ctx = ctx;
  s->seed = seed;
  if (nw::mlp_create(ctx, &s->mlp, nw::mlp_descriptor_width(ctx->nref, ctx->nmo), 1, kScreenBatch, seed) != NW_OK ||
      cudaMalloc(&s->rows, sizeof(uint32_t) * kScreenBatch) != cudaSuccess ||
      cudaMalloc(&s->t, sizeof(float) * kScreenBatch) != cudaSuccess ||
      cudaMalloc(&s->loss, sizeof(double)) != cudaSuccess) {
    screen_release(s);
    return nw::fail(ctx, NW_ERR_ALLOC, "screener allocation failed");
  }
  *out = s;
  return NW_OK;
}

nw_status nw_screen_train(nw_screen* s, const uint32_t* idx, const double* target, uint64_t n, const nw_mlp_opts* opts,
                          nw_mlp_report* rep) {
  if (!s || !idx || !target || !opts || !rep || n == 0) return NW_ERR_INVALID;
  if (opts->epochs < 0 || opts->batch < 1 || opts->batch > kScreenBatch || !(opts->lr > 0.0))
    return sfail(s, NW_ERR_INVALID, "invalid training options (batch <= 4096)");
  if (n > 0xFFFFFFFFull) return sfail(s, NW_ERR_UNSUPPORTED, "too many training rows");
  nw_status st = check_rows(s, idx, n);
  if (st != NW_OK) return st;
  double sum = 0.0, sq = 0.0;
  for (uint64_t i = 0; i < n; ++i) {
    if (!std::isfinite(target[i])) return sfail(s, NW_ERR_INVALID, "non-finite target");
    sum += target[i];
    sq += target[i] * target[i];
  }
  // standardise with the first training set; later calls fine-tune on the same scale
  if (!s->trained) {
    s->mean = sum / (double)n;
    const double var = std::max(sq / (double)n - s->mean * s->mean, 0.0);
    s->scale = var > 1e-12 ? std::sqrt(var) : 1.0;
  }
  std::vector<float> tn(n);
  for (uint64_t i = 0; i < n; ++i) tn[i] = (float)((target[i] - s->mean) / s->scale);
  nw_ctx* ctx = s->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  uint32_t* didx = nullptr;
  float* dt = nullptr;
  if (cudaMalloc(&didx, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&dt, sizeof(float) * n) != cudaSuccess) {
    if (didx) cudaFree(didx);
    return sfail(s, NW_ERR_ALLOC, "training rows");
  }
  cudaStream_t stream = nullptr;
  st = NW_OK;
  if (cudaMemcpy(didx, idx, sizeof(uint32_t) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dt, tn.data(), sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    st = sfail(s, NW_ERR_CUDA, "training upload");
  std::memset(rep, 0, sizeof(*rep));
  rep->samples = n;
  const int B = (int)std::min<uint64_t>((uint64_t)opts->batch, n);
  const uint64_t steps = (uint64_t)opts->epochs * ((n + (uint64_t)B - 1) / (uint64_t)B);
  for (uint64_t step = 0; step < steps && st == NW_OK; ++step) {
    screen_batch_kernel<<<(B + 127) / 128, 128, 0, stream>>>(didx, dt, n, opts->seed, step, B, s->rows, s->t);
    if ((st = nw::mlp_features(ctx, &s->mlp, ctx->d_dets, s->rows, 0, B, stream)) != NW_OK) break;
    if ((st = nw::mlp_forward(ctx, &s->mlp, B, stream)) != NW_OK) break;
    mse_kernel<<<1, 256, 0, stream>>>(s->mlp.z, s->t, B, s->loss);
    if ((st = nw::mlp_backward(ctx, &s->mlp, B, stream)) != NW_OK) break;
    if ((st = nw::mlp_adam(ctx, &s->mlp, (float)opts->lr, stream)) != NW_OK) break;
    if (step == 0 || step + 1 == steps) {
      double l = 0.0;
      if (cudaMemcpy(&l, s->loss, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        st = sfail(s, NW_ERR_CUDA, "loss read");
        break;
      }
      if (step == 0) rep->loss_first = l;
      if (step + 1 == steps) rep->loss_last = l;
    }
  }
  if (st == NW_OK && cudaDeviceSynchronize() != cudaSuccess) st = sfail(s, NW_ERR_CUDA, "screener training");
  cudaFree(didx);
  cudaFree(dt);
  if (st != NW_OK) return st;
  rep->steps = (int32_t)steps;
  s->trained = true;
  return NW_OK;
}

nw_status nw_screen_predict(nw_screen* s, const uint32_t* idx, uint64_t n, double* out) {
  if (!s || (n && (!idx || !out))) return NW_ERR_INVALID;
  if (!s->trained) return sfail(s, NW_ERR_STATE, "screener not trained (nw_screen_train)");
  nw_status st = check_rows(s, idx, n);
  if (st != NW_OK) return st;
  nw_ctx* ctx = s->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  std::vector<float> z(kScreenBatch);
  for (uint64_t r0 = 0; r0 < n; r0 += kScreenBatch) {
    const int B = (int)std::min<uint64_t>(kScreenBatch, n - r0);
    NW_CUDA(ctx, cudaMemcpy(s->rows, idx + r0, sizeof(uint32_t) * B, cudaMemcpyHostToDevice));
    if ((st = nw::mlp_features(ctx, &s->mlp, ctx->d_dets, s->rows, 0, B, nullptr)) != NW_OK) return st;
    if ((st = nw::mlp_forward(ctx, &s->mlp, B, nullptr)) != NW_OK) return st;
    NW_CUDA(ctx, cudaMemcpy(z.data(), s->mlp.z, sizeof(float) * B, cudaMemcpyDeviceToHost));
    for (int r = 0; r < B; ++r) out[r0 + r] = (double)z[r] * s->scale + s->mean;
  }
  return NW_OK;
}

nw_status nw_screen_destroy(nw_screen* s) {
  if (!s) return NW_OK;
  cudaSetDevice(s->ctx->device);
  cudaDeviceSynchronize();
  screen_release(s);
  return NW_OK;
}

}  // extern "C"
