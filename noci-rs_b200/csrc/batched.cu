// Per-reference-pair batched evaluation from caller-held excitation caches, and the host-buffer
// overlap entry point.
//
// nw_eval_hs_batched[_device] stands in for xw_hamiltonian_overlap_prepared_batched
// (src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:121-362): every request belongs to
// one ordered reference pair (lp, gp) and brings its bra and ket excitation caches
// (ExcitationCache, src/lib.rs:136-167) and the product of their excitation phases.  The
// caches are packed on the device into the engine's 32-byte determinant records (bra 2i with
// parent lp and the phase, ket 2i + 1 with parent gp and phase 1), each checked as nw_set_basis
// checks a resident basis (a request with an invalid cache gets NaN and is reported by the
// call, or by nw_sync for the device variant); the requests then go through the engine's sorted
// pipeline (classify by contraction-rank class, scan, scatter, the fixed-rank and m > 0
// evaluators) exactly as resident-basis pairs do.
#include <cuda_runtime.h>

#include <cmath>

#include "internal.cuh"

namespace nw {
namespace {

__device__ __forceinline__ bool spin_cache_ok(const nw_exc_spin& c, int nocc, int nmo) {
  const int r = c.rank;
  if (r > 4) return false;
  for (int k = 0; k < r; ++k) {
    if (c.indices[k] >= nocc) return false;
    if (c.indices[4 + k] < nocc || c.indices[4 + k] >= nmo) return false;
    if (k > 0 && (c.indices[k] <= c.indices[k - 1] || c.indices[4 + k] <= c.indices[3 + k])) return false;
  }
  return true;
}

__device__ __forceinline__ void pack_det(nw_det* d, uint16_t* desc, uint32_t parent, const nw_exc_cache& c,
                                         double phase) {
  nw_det r;
  r.parent = parent;
  r.rank_a = c.alpha.rank;
  r.rank_b = c.beta.rank;
  for (int k = 0; k < 8; ++k) {
    r.idx_a[k] = k % 4 < c.alpha.rank ? c.alpha.indices[k] : 0;
    r.idx_b[k] = k % 4 < c.beta.rank ? c.beta.indices[k] : 0;
  }
  r.pad[0] = r.pad[1] = 0;
  r.phase = phase;
  *d = r;
  *desc = (uint16_t)det_desc(parent, c.alpha.rank, c.beta.rank);
}

// Request i -> records 2i (bra) and 2i + 1 (ket) and pair (2i, 2i + 1); an invalid request
// gets an out-of-range pair, which the classify kernel turns into NaN and the error flag.
__global__ void pack_batched_kernel(uint32_t lp, uint32_t gp, const nw_exc_cache* __restrict__ x,
                                    const nw_exc_cache* __restrict__ w, const double* __restrict__ phase,
                                    uint64_t n, int nocc_a, int nocc_b, int nmo, nw_det* __restrict__ dets,
                                    uint16_t* __restrict__ desc, uint2* __restrict__ pairs) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const nw_exc_cache cx = x[i], cw = w[i];
    const double ph = phase[i];
    const bool ok = spin_cache_ok(cx.alpha, nocc_a, nmo) && spin_cache_ok(cx.beta, nocc_b, nmo) &&
                    spin_cache_ok(cw.alpha, nocc_a, nmo) && spin_cache_ok(cw.beta, nocc_b, nmo) && isfinite(ph);
    pack_det(dets + 2 * i, desc + 2 * i, lp, cx, ph);
    pack_det(dets + 2 * i + 1, desc + 2 * i + 1, gp, cw, 1.0);
    pairs[i] = ok ? make_uint2((uint32_t)(2 * i), (uint32_t)(2 * i + 1)) : make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
  }
}

nw_status eval_batched(nw_ctx* ctx, EvalMode mode, int lp, int gp, const nw_exc_cache* x, const nw_exc_cache* w,
                       const double* phase, uint64_t n, double* hs, cudaStream_t s) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (mode == EvalMode::kFS && !ctx->fock_ready) return fail(ctx, NW_ERR_STATE, "Fock tables not set (nw_update_fock)");
  if (lp < 0 || gp < 0 || lp >= ctx->nref || gp >= ctx->nref) return fail(ctx, NW_ERR_INVALID, "reference index out of range");
  if (n == 0) return NW_OK;
  if (n >= 0x7FFFFFFFull) return fail(ctx, NW_ERR_UNSUPPORTED, "at most 2^31 - 2 requests per call");
  nw_status st;
  if ((st = ensure(ctx, ctx->bt_dets, 2 * n * sizeof(nw_det))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->bt_desc, 2 * n * sizeof(uint16_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->bt_pairs, n * sizeof(uint2))) != NW_OK) return st;
  nw_det* dets = static_cast<nw_det*>(ctx->bt_dets.p);
  uint16_t* desc = static_cast<uint16_t*>(ctx->bt_desc.p);
  uint2* pairs = static_cast<uint2*>(ctx->bt_pairs.p);
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 8);
  pack_batched_kernel<<<(unsigned)blocks, 256, 0, s>>>((uint32_t)lp, (uint32_t)gp, x, w, phase, n, ctx->nocc_a,
                                                       ctx->nocc_b, ctx->nmo, dets, desc, pairs);
  NW_CUDA(ctx, cudaGetLastError());
  EvalParams P = make_params(ctx);
  P.dets = dets;
  P.desc = desc;
  P.ndet = 2 * n;
  return eval_pairs_on(ctx, P, reinterpret_cast<const uint32_t*>(pairs), n, hs, mode, s);
}

// Host-buffer form: stage the caches and phases, evaluate, copy the results back (width
// doubles per request), synchronise and report invalid requests.
nw_status eval_batched_host(nw_ctx* ctx, EvalMode mode, int lp, int gp, const nw_exc_cache* x, const nw_exc_cache* w,
                            const double* phase, uint64_t npairs, double* out, cudaStream_t s) {
  if (npairs == 0) return NW_OK;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  if (npairs >= 0x7FFFFFFFull) return fail(ctx, NW_ERR_UNSUPPORTED, "at most 2^31 - 2 requests per call");
  const int width = mode == EvalMode::kS ? 1 : 2;
  // staging: x caches | w caches | phases (8-byte aligned) | results (16-byte aligned)
  const size_t cache_bytes = npairs * sizeof(nw_exc_cache);
  const size_t off_ph = (2 * cache_bytes + 15) / 16 * 16;
  const size_t off_out = (off_ph + npairs * sizeof(double) + 15) / 16 * 16;
  nw_status st = ensure(ctx, ctx->bt_in, off_out + npairs * width * sizeof(double));
  if (st != NW_OK) return st;
  if ((st = ensure(ctx, ctx->flag, 256)) != NW_OK) return st;
  char* base = static_cast<char*>(ctx->bt_in.p);
  nw_exc_cache* dx = reinterpret_cast<nw_exc_cache*>(base);
  nw_exc_cache* dw = reinterpret_cast<nw_exc_cache*>(base + cache_bytes);
  double* dph = reinterpret_cast<double*>(base + off_ph);
  double* dout = reinterpret_cast<double*>(base + off_out);
  NW_CUDA(ctx, cudaMemcpyAsync(dx, x, cache_bytes, cudaMemcpyHostToDevice, s));
  NW_CUDA(ctx, cudaMemcpyAsync(dw, w, cache_bytes, cudaMemcpyHostToDevice, s));
  NW_CUDA(ctx, cudaMemcpyAsync(dph, phase, npairs * sizeof(double), cudaMemcpyHostToDevice, s));
  if ((st = eval_batched(ctx, mode, lp, gp, dx, dw, dph, npairs, dout, s)) != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpyAsync(out, dout, npairs * width * sizeof(double), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaMemcpyAsync(ctx->h_flag, ctx->flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaStreamSynchronize(s));
  if (*ctx->h_flag) return fail(ctx, NW_ERR_INVALID, "invalid excitation cache or phase in a request");
  return NW_OK;
}

}  // namespace
}  // namespace nw

extern "C" {

nw_status nw_eval_hs_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                    const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs,
                                    double* hs_dev, void* stream) {
  if (!ctx || (npairs && (!x_dev || !w_dev || !phase_dev || !hs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::eval_batched(ctx, nw::EvalMode::kHS, lp, gp, x_dev, w_dev, phase_dev, npairs, hs_dev,
                          static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_hs_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                             const double* phase, uint64_t npairs, double* hs_out, void* stream) {
  if (!ctx || (npairs && (!x || !w || !phase || !hs_out))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_batched_host(ctx, nw::EvalMode::kHS, lp, gp, x, w, phase, npairs, hs_out,
                               static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_s_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                   const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs, double* s_dev,
                                   void* stream) {
  if (!ctx || (npairs && (!x_dev || !w_dev || !phase_dev || !s_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::eval_batched(ctx, nw::EvalMode::kS, lp, gp, x_dev, w_dev, phase_dev, npairs, s_dev,
                          static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_s_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                            const double* phase, uint64_t npairs, double* s_out, void* stream) {
  if (!ctx || (npairs && (!x || !w || !phase || !s_out))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_batched_host(ctx, nw::EvalMode::kS, lp, gp, x, w, phase, npairs, s_out,
                               static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_fs_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                    const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs,
                                    double* fs_dev, void* stream) {
  if (!ctx || (npairs && (!x_dev || !w_dev || !phase_dev || !fs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::eval_batched(ctx, nw::EvalMode::kFS, lp, gp, x_dev, w_dev, phase_dev, npairs, fs_dev,
                          static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_fs_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                             const double* phase, uint64_t npairs, double* fs_out, void* stream) {
  if (!ctx || (npairs && (!x || !w || !phase || !fs_out))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_batched_host(ctx, nw::EvalMode::kFS, lp, gp, x, w, phase, npairs, fs_out,
                               static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_s_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* s_host, void* stream) {
  if (!ctx || (npairs && (!pairs_host || !s_host))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  if (npairs == 0) return NW_OK;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw_status st = nw::ensure(ctx, ctx->io_pairs, npairs * 2 * sizeof(uint32_t));
  if (st != NW_OK) return st;
  if ((st = nw::ensure(ctx, ctx->io_hs, npairs * sizeof(double))) != NW_OK) return st;
  uint32_t* dp = static_cast<uint32_t*>(ctx->io_pairs.p);
  double* ds = static_cast<double*>(ctx->io_hs.p);
  NW_CUDA(ctx, cudaMemcpyAsync(dp, pairs_host, npairs * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  if ((st = nw::eval_pairs(ctx, dp, npairs, ds, nw::EvalMode::kS, s)) != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpyAsync(s_host, ds, npairs * sizeof(double), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaMemcpyAsync(ctx->h_flag, ctx->flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaStreamSynchronize(s));
  if (*ctx->h_flag) return nw::fail(ctx, NW_ERR_INVALID, "pair index out of range of the determinant basis");
  return NW_OK;
}

}  // extern "C"
