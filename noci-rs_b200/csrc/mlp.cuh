// Small MLP of the learned QMC proposal (csrc/mlp.cu): din -> 128 -> 128 -> nout, ReLU, FP32
// master parameters with BF16 copies of the weight matrices that the forward and backward
// products read (FP32 accumulation), Adam updates.  Parameter layout (floats):
//   W1 [128][din], b1 [128], W2 [128][128], b2 [128], W3 [nout][128], b3 [nout].
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/nociwick.h"

struct nw_ctx;

namespace nw {

constexpr int kMlpWidth = 128;

struct Mlp {
  int din = 0, nout = 0, bcap = 0;
  size_t nparams = 0;
  float* params = nullptr;  // master parameters
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  __nv_bfloat16* wbf = nullptr;  // BF16 copies of W1, W2, W3 (same offsets as in params, biases unused)
  float* x = nullptr;            // [bcap][din] features
  float* h1 = nullptr;           // [bcap][128]
  float* h2 = nullptr;           // [bcap][128]
  float* z = nullptr;            // [bcap][nout] logits, then dZ
  float* d2 = nullptr;           // [bcap][128]
  float* d1 = nullptr;           // [bcap][128]
  float* part = nullptr;         // k-split partial products of the weight gradients
  int adam_t = 0;
  size_t off_w1() const { return 0; }
  size_t off_b1() const { return (size_t)kMlpWidth * din; }
  size_t off_w2() const { return off_b1() + kMlpWidth; }
  size_t off_b2() const { return off_w2() + (size_t)kMlpWidth * kMlpWidth; }
  size_t off_w3() const { return off_b2() + kMlpWidth; }
  size_t off_b3() const { return off_w3() + (size_t)nout * kMlpWidth; }
};

size_t mlp_param_count(int din, int nout);
// Width of the determinant descriptor (rounded up to 32): nref + 10 + 2 nmo.
int mlp_descriptor_width(int nref, int nmo);
// Descriptors of dets[rows[r]] (or dets[row0 + r] when rows is null), r < B <= bcap, into m->x.
nw_status mlp_features(nw_ctx* ctx, Mlp* m, const nw_det* dets, const uint32_t* rows, uint32_t row0, int B,
                       cudaStream_t s);
// Allocates the MLP and initialises it (uniform +-sqrt(6 / fan_in) weights from a Philox stream
// of `seed`, zero biases).
nw_status mlp_create(nw_ctx* ctx, Mlp* m, int din, int nout, int bcap, uint64_t seed);
void mlp_destroy(Mlp* m);
// Refresh the BF16 weight copies from the master parameters.
nw_status mlp_sync_bf16(nw_ctx* ctx, Mlp* m, cudaStream_t s);
// Logits z[b] of features x[0..B) (activations kept for the backward pass).
nw_status mlp_forward(nw_ctx* ctx, Mlp* m, int B, cudaStream_t s);
// With m->z holding dL/dz: gradients of all parameters into m->grads (overwritten).
nw_status mlp_backward(nw_ctx* ctx, Mlp* m, int B, cudaStream_t s);
nw_status mlp_adam(nw_ctx* ctx, Mlp* m, float lr, cudaStream_t s);

}  // namespace nw
