// C ABI of the engine (declared in include/nociwick.h): context lifetime, input validation,
// and the host/device entry points.
#include <cuda_runtime.h>
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"

namespace nw {

nw_status fail(nw_ctx* ctx, nw_status st, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return st;
}

nw_status cuda_fail(nw_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, NW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

nw_status ensure(nw_ctx* ctx, DevBuf& b, size_t bytes) {
  if (b.bytes >= bytes) return NW_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  size_t want = bytes + bytes / 4 + 256;
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) {
    b.p = nullptr;
    return fail(ctx, NW_ERR_ALLOC, std::string("scratch allocation failed: ") + cudaGetErrorString(e));
  }
  b.bytes = want;
  return NW_OK;
}

}  // namespace nw

namespace {

void free_buf(nw::DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
}

nw_status upload(nw_ctx* ctx, double** dst, const double* src, size_t count) {
  if (cudaMalloc(dst, count * sizeof(double)) != cudaSuccess)
    return nw::fail(ctx, NW_ERR_ALLOC, "device allocation for inputs failed");
  NW_CUDA(ctx, cudaMemcpy(*dst, src, count * sizeof(double), cudaMemcpyHostToDevice));
  return NW_OK;
}

bool finite_all(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// Page-locked host memory (cudaHostAlloc / cudaHostRegister): only such buffers let the copy
// engines run asynchronously, so only they take the pipelined path.
bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

nw_status pipe_setup(nw_ctx* ctx) {
  if (ctx->s_in) return NW_OK;
  NW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_in, cudaStreamNonBlocking));
  NW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_comp, cudaStreamNonBlocking));
  NW_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->s_out, cudaStreamNonBlocking));
  NW_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_start, cudaEventDisableTiming));
  for (int i = 0; i < 2; ++i) {
    NW_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_in[i], cudaEventDisableTiming));
    NW_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_comp[i], cudaEventDisableTiming));
  }
  return NW_OK;
}

// Waits for everything the pipeline queued (the caller's host buffers must not be touched by
// copies after the call returns, also on error paths).
cudaError_t pipe_drain(nw_ctx* ctx) {
  cudaError_t first = cudaSuccess;
  for (cudaStream_t q : {ctx->s_in, ctx->s_comp, ctx->s_out}) {
    if (!q) continue;
    const cudaError_t e = cudaStreamSynchronize(q);
    if (first == cudaSuccess) first = e;
  }
  return first;
}

// Host-buffer evaluation as a three-stage pipeline over chunks of the request: chunk k+1 is
// copied in (copy engine, host -> device) while chunk k is evaluated and chunk k-1 is copied
// out (second copy engine, device -> host), so PCIe transfer in both directions overlaps the
// kernels.  Starts after the work already queued on `caller` and returns when the results
// are in hs_host.
nw_status eval_hs_pipelined(nw_ctx* ctx, nw::EvalMode mode, const uint32_t* pairs_host, uint64_t npairs,
                            double* hs_host, uint32_t* dp, double* dh, cudaStream_t caller) {
  nw_status st = pipe_setup(ctx);
  if (st != NW_OK) return st;
  if ((st = nw::ensure(ctx, ctx->flag, 256)) != NW_OK) return st;
  uint32_t* flag = static_cast<uint32_t*>(ctx->flag.p);
  NW_CUDA(ctx, cudaEventRecord(ctx->ev_start, caller));
  for (cudaStream_t q : {ctx->s_in, ctx->s_comp, ctx->s_out}) NW_CUDA(ctx, cudaStreamWaitEvent(q, ctx->ev_start, 0));
  NW_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(uint32_t), ctx->s_comp));
  uint64_t chunk = (npairs + nw::kPipeChunks - 1) / nw::kPipeChunks;
  chunk = std::max<uint64_t>(nw::kPipeMinChunk, (chunk + 255) / 256 * 256);
  uint64_t k = 0;
  for (uint64_t o = 0; o < npairs; o += chunk, ++k) {
    const uint64_t nk = std::min(chunk, npairs - o);
    const int slot = (int)(k & 1);
    cudaError_t e = cudaMemcpyAsync(dp + 2 * o, pairs_host + 2 * o, nk * 2 * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, ctx->s_in);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_in[slot], ctx->s_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_comp, ctx->ev_in[slot], 0);
    if (e != cudaSuccess) {
      pipe_drain(ctx);
      return nw::cuda_fail(ctx, e, "pipelined copy-in");
    }
    st = nw::eval_pairs(ctx, dp + 2 * o, nk, dh + 2 * o, mode, ctx->s_comp, false);
    if (st != NW_OK) {
      pipe_drain(ctx);
      return st;
    }
    e = cudaEventRecord(ctx->ev_comp[slot], ctx->s_comp);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_out, ctx->ev_comp[slot], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hs_host + 2 * o, dh + 2 * o, nk * 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->s_out);
    if (e != cudaSuccess) {
      pipe_drain(ctx);
      return nw::cuda_fail(ctx, e, "pipelined copy-out");
    }
  }
  cudaError_t e = cudaMemcpyAsync(ctx->h_flag, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->s_comp);
  const cudaError_t ed = pipe_drain(ctx);
  if (e != cudaSuccess) return nw::cuda_fail(ctx, e, "pipelined flag read");
  if (ed != cudaSuccess) return nw::cuda_fail(ctx, ed, "pipelined evaluation");
  NW_CUDA(ctx, cudaGetLastError());
  if (*ctx->h_flag) return nw::fail(ctx, NW_ERR_INVALID, "pair index out of range of the determinant basis");
  return NW_OK;
}

// Host-buffer evaluation (H, S) or (F, S): copy in, evaluate, copy out, synchronise.
nw_status eval_host(nw_ctx* ctx, nw::EvalMode mode, const uint32_t* pairs_host, uint64_t npairs, double* out_host,
                    void* stream) {
  if (!ctx || (npairs && (!pairs_host || !out_host))) return NW_ERR_INVALID;
  if (npairs == 0) return NW_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw_status st = nw::ensure(ctx, ctx->io_pairs, npairs * 2 * sizeof(uint32_t));
  if (st != NW_OK) return st;
  if ((st = nw::ensure(ctx, ctx->io_hs, npairs * 2 * sizeof(double))) != NW_OK) return st;
  uint32_t* dp = static_cast<uint32_t*>(ctx->io_pairs.p);
  double* dh = static_cast<double*>(ctx->io_hs.p);
  if (npairs >= 2 * nw::kPipeMinChunk && is_pinned(pairs_host) && is_pinned(out_host))
    return eval_hs_pipelined(ctx, mode, pairs_host, npairs, out_host, dp, dh, s);
  NW_CUDA(ctx, cudaMemcpyAsync(dp, pairs_host, npairs * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  if ((st = nw::eval_pairs(ctx, dp, npairs, dh, mode, s)) != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpyAsync(out_host, dh, npairs * 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaMemcpyAsync(ctx->h_flag, ctx->flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NW_CUDA(ctx, cudaStreamSynchronize(s));
  if (*ctx->h_flag) return nw::fail(ctx, NW_ERR_INVALID, "pair index out of range of the determinant basis");
  return NW_OK;
}

}  // namespace

extern "C" {

const char* nw_status_string(nw_status st) {
  switch (st) {
    case NW_OK:
      return "ok";
    case NW_ERR_INVALID:
      return "invalid argument";
    case NW_ERR_CUDA:
      return "CUDA error";
    case NW_ERR_ALLOC:
      return "allocation failed";
    case NW_ERR_UNSUPPORTED:
      return "unsupported input";
    case NW_ERR_STATE:
      return "call out of order";
    case NW_ERR_NO_DEVICE:
      return "no CUDA device";
    case NW_ERR_IO:
      return "cache file input/output failed";
  }
  return "unknown status";
}

const char* nw_last_error(const nw_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

}  // extern "C"

namespace {

// Shared part of nw_ctx_create / nw_ctx_create_cholesky: validation of everything but the
// two-electron integrals, the context, its streams and the uploads of S, h and the orbitals.
nw_status create_base(int nao, int nmo, double enuc, const double* s, const double* h, const nw_refs* refs,
                      const nw_opts* opts, nw_ctx** out) {
  if (!s || !h || !refs || !opts || !refs->c_alpha || !refs->c_beta) return NW_ERR_INVALID;
  const int nref = refs->nref;
  if (nao <= 0 || nmo <= 0 || nmo > 128 || nref <= 0 || nref > 256) return NW_ERR_UNSUPPORTED;
  if (refs->nocc_a < 0 || refs->nocc_b < 0 || refs->nocc_a > nmo || refs->nocc_b > nmo) return NW_ERR_INVALID;
  if (refs->nocc_a > 64 || refs->nocc_b > 64) return NW_ERR_UNSUPPORTED;
  if (!(opts->tol >= 0.0) || !std::isfinite(opts->tol) || !std::isfinite(enuc)) return NW_ERR_INVALID;
  if (opts->convention != NW_CONVENTION_REFERENCE && opts->convention != NW_CONVENTION_EXACT) return NW_ERR_INVALID;
  const size_t n2 = (size_t)nao * nao;
  if (!finite_all(s, n2) || !finite_all(h, n2) || !finite_all(refs->c_alpha, (size_t)nref * nao * nmo) ||
      !finite_all(refs->c_beta, (size_t)nref * nao * nmo))
    return NW_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return NW_ERR_NO_DEVICE;
  if (opts->device < 0 || opts->device >= ndev) return NW_ERR_INVALID;
  nw_ctx* ctx = new (std::nothrow) nw_ctx();
  if (!ctx) return NW_ERR_ALLOC;
  ctx->device = opts->device;
  ctx->nao = nao;
  ctx->nmo = nmo;
  ctx->nref = nref;
  ctx->nocc_a = refs->nocc_a;
  ctx->nocc_b = refs->nocc_b;
  ctx->enuc = enuc;
  ctx->tol = opts->tol;
  ctx->convention = opts->convention;
  nw_status st = NW_OK;
  if (cudaSetDevice(ctx->device) != cudaSuccess) st = NW_ERR_CUDA;
  if (st == NW_OK && cublasCreate(&ctx->blas) != CUBLAS_STATUS_SUCCESS) st = NW_ERR_CUDA;
  if (st == NW_OK) st = upload(ctx, &ctx->d_s, s, n2);
  if (st == NW_OK) st = upload(ctx, &ctx->d_h, h, n2);
  if (st == NW_OK) st = upload(ctx, &ctx->d_ca, refs->c_alpha, (size_t)nref * nao * nmo);
  if (st == NW_OK) st = upload(ctx, &ctx->d_cb, refs->c_beta, (size_t)nref * nao * nmo);
  if (st == NW_OK && cudaMallocHost(&ctx->h_flag, sizeof(uint32_t)) != cudaSuccess) st = NW_ERR_ALLOC;
  for (int i = 0; i < 3 && st == NW_OK; ++i)
    if (cudaStreamCreateWithFlags(&ctx->s_aux[i], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming) != cudaSuccess)
      st = NW_ERR_CUDA;
  if (st == NW_OK && cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess) st = NW_ERR_CUDA;
  if (st == NW_OK && cudaEventCreateWithFlags(&ctx->ev_free, cudaEventDisableTiming) != cudaSuccess) st = NW_ERR_CUDA;
  if (st != NW_OK) {
    nw_ctx_destroy(ctx);
    return st;
  }
  *out = ctx;
  return NW_OK;
}

}  // namespace

extern "C" {

nw_status nw_ctx_create(const nw_system* sys, const nw_refs* refs, const nw_opts* opts, nw_ctx** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!sys || !sys->eri) return NW_ERR_INVALID;
  const size_t n2 = (size_t)std::max(sys->nao, 0) * std::max(sys->nao, 0);
  if (sys->nao > 0 && sys->nao <= 128 && !finite_all(sys->eri, n2 * n2)) return NW_ERR_INVALID;
  nw_ctx* ctx = nullptr;
  nw_status st = create_base(sys->nao, sys->nmo, sys->enuc, sys->s, sys->h, refs, opts, &ctx);
  if (st != NW_OK) return st;
  if ((st = upload(ctx, &ctx->d_eri, sys->eri, n2 * n2)) != NW_OK) {
    nw_ctx_destroy(ctx);
    return st;
  }
  *out = ctx;
  return NW_OK;
}

nw_status nw_ctx_create_cholesky(const nw_system_cd* sys, const nw_refs* refs, const nw_opts* opts, nw_ctx** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!sys || !sys->chol || sys->naux <= 0) return NW_ERR_INVALID;
  if (sys->naux > 65536) return NW_ERR_UNSUPPORTED;
  const int nao = sys->nao;
  const size_t n2 = (size_t)std::max(nao, 0) * std::max(nao, 0);
  if (nao > 0 && nao <= 128 && !finite_all(sys->chol, (size_t)sys->naux * n2)) return NW_ERR_INVALID;
  nw_ctx* ctx = nullptr;
  nw_status st = create_base(nao, sys->nmo, sys->enuc, sys->s, sys->h, refs, opts, &ctx);
  if (st != NW_OK) return st;
  // (mu nu|lam sig) = sum_P L[P][mu nu] L[P][lam sig]: E = L^T L with L as naux x n^2, on the
  // engine's FP64 GEMM; the factors stay resident
  ctx->naux = sys->naux;
  st = upload(ctx, &ctx->d_chol, sys->chol, (size_t)sys->naux * n2);
  if (st == NW_OK && cudaMalloc(&ctx->d_eri, n2 * n2 * sizeof(double)) != cudaSuccess) st = NW_ERR_ALLOC;
  if (st == NW_OK) {
    const cudaError_t e = nw::dgemm_strided(0, true, false, (int)n2, (int)n2, sys->naux, 1.0, ctx->d_chol, (int)n2, 0,
                                            ctx->d_chol, (int)n2, 0, 0.0, ctx->d_eri, (int)n2, 0, 1);
    if (e != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = nw::cuda_fail(ctx, e, "Cholesky integrals");
  }
  if (st != NW_OK) {
    nw_ctx_destroy(ctx);
    return st;
  }
  *out = ctx;
  return NW_OK;
}

nw_status nw_set_transform(nw_ctx* ctx, int32_t mode) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (mode < NW_TRANSFORM_FP64 || mode > NW_TRANSFORM_CHOL_BF16X6) return nw::fail(ctx, NW_ERR_INVALID, "unknown transform");
  if (mode != NW_TRANSFORM_FP64 && !ctx->d_chol)
    return nw::fail(ctx, NW_ERR_STATE, "Cholesky transforms need a context from nw_ctx_create_cholesky");
  // int8 slice sums stay exact in INT32 while (s + 1) naux 64^2 < 2^31
  if (mode == NW_TRANSFORM_CHOL_INT8 && ctx->naux > 16384)
    return nw::fail(ctx, NW_ERR_UNSUPPORTED, "int8 split products take at most 16384 Cholesky vectors");
  ctx->transform = mode;
  return NW_OK;
}

nw_status nw_transform_product(int32_t mode, const double* u, const double* v, int32_t naux, int32_t n, double* t4,
                               void* stream) {
  if (!u || !v || !t4 || naux <= 0 || n <= 0 || n > 128) return NW_ERR_INVALID;
  if (mode != NW_TRANSFORM_CHOL_FP64 && mode != NW_TRANSFORM_CHOL_INT8 && mode != NW_TRANSFORM_CHOL_BF16X6)
    return NW_ERR_INVALID;
  if (mode == NW_TRANSFORM_CHOL_INT8 && naux > 16384) return NW_ERR_UNSUPPORTED;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n2 = n * n;
  void* work = nullptr;
  const size_t scratch = mode == NW_TRANSFORM_CHOL_FP64 ? (size_t)n2 * n2 * sizeof(double)
                                                         : nw::split_product_scratch(mode, naux, n2, n2, nw::kOzakiSlices);
  if (cudaMalloc(&work, scratch + 256) != cudaSuccess) return NW_ERR_ALLOC;
  uint32_t* err = reinterpret_cast<uint32_t*>(static_cast<char*>(work) + scratch);
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) {
    if (mode == NW_TRANSFORM_CHOL_FP64) {
      e = nw::dgemm_strided(s, true, false, n2, n2, naux, 1.0, u, n2, 0, v, n2, 0, 0.0, static_cast<double*>(work), n2,
                            0, 1);
      if (e == cudaSuccess) e = nw::swap_qr(s, static_cast<const double*>(work), n, t4);
    } else {
      e = nw::split_product_pqrs(s, mode, nw::kOzakiSlices, u, v, naux, n, t4, work, scratch, err);
    }
  }
  uint32_t herr = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(work);
  if (e != cudaSuccess) return NW_ERR_CUDA;
  return herr ? NW_ERR_CUDA : NW_OK;
}

nw_status nw_build_intermediates(nw_ctx* ctx) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::build_all(ctx, nullptr);
}

nw_status nw_pair_zero_counts(const nw_ctx* ctx, int32_t* m) {
  if (!ctx || !m) return NW_ERR_INVALID;
  if (!ctx->built) return NW_ERR_STATE;
  std::memcpy(m, ctx->m_counts.data(), sizeof(int32_t) * ctx->m_counts.size());
  return NW_OK;
}

nw_status nw_set_basis(nw_ctx* ctx, const nw_det* basis, uint64_t ndet) {
  if (!ctx || (!basis && ndet)) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (ndet >= 0xFFFFFFFFull) return nw::fail(ctx, NW_ERR_UNSUPPORTED, "at most 2^32 - 2 determinants");
  if (ctx->live_qmc > 0)
    return nw::fail(ctx, NW_ERR_STATE, "a QMC object uses the resident basis (nw_qmc_destroy it first)");
  // Validate every record: parent in range, ranks <= 4, holes ascending in the occupied
  // block, particles ascending in the virtual block.
  for (uint64_t i = 0; i < ndet; ++i) {
    const nw_det& d = basis[i];
    if (d.parent >= (uint32_t)ctx->nref) return nw::fail(ctx, NW_ERR_INVALID, "determinant parent out of range");
    if (!std::isfinite(d.phase)) return nw::fail(ctx, NW_ERR_INVALID, "non-finite determinant phase");
    for (int spin = 0; spin < 2; ++spin) {
      const int r = spin ? d.rank_b : d.rank_a;
      const uint8_t* idx = spin ? d.idx_b : d.idx_a;
      const int nocc = spin ? ctx->nocc_b : ctx->nocc_a;
      if (r > 4) return nw::fail(ctx, NW_ERR_UNSUPPORTED, "excitation rank above 4 per spin");
      for (int k = 0; k < r; ++k) {
        if (idx[k] >= nocc) return nw::fail(ctx, NW_ERR_INVALID, "hole index not occupied in the parent");
        if (idx[4 + k] < nocc || idx[4 + k] >= ctx->nmo)
          return nw::fail(ctx, NW_ERR_INVALID, "particle index not virtual in the parent");
        if (k > 0 && (idx[k] <= idx[k - 1] || idx[4 + k] <= idx[3 + k]))
          return nw::fail(ctx, NW_ERR_INVALID, "hole/particle indices must be strictly ascending");
      }
    }
  }
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw::overlap_plan_free(ctx->ovl);
  ctx->ovl = nullptr;
  if (ctx->d_dets) cudaFree(ctx->d_dets);
  if (ctx->d_desc) cudaFree(ctx->d_desc);
  ctx->d_dets = nullptr;
  ctx->d_desc = nullptr;
  ctx->ndet = 0;
  if (ndet == 0) return NW_OK;
  std::vector<uint16_t> desc(ndet);
  for (uint64_t i = 0; i < ndet; ++i) desc[i] = (uint16_t)nw::det_desc(basis[i].parent, basis[i].rank_a, basis[i].rank_b);
  if (cudaMalloc(&ctx->d_dets, ndet * sizeof(nw_det)) != cudaSuccess ||
      cudaMalloc(&ctx->d_desc, ndet * sizeof(uint16_t)) != cudaSuccess)
    return nw::fail(ctx, NW_ERR_ALLOC, "basis allocation failed");
  NW_CUDA(ctx, cudaMemcpy(ctx->d_dets, basis, ndet * sizeof(nw_det), cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_desc, desc.data(), ndet * sizeof(uint16_t), cudaMemcpyHostToDevice));
  ctx->ndet = ndet;
  return NW_OK;
}

nw_status nw_eval_hs_pairs_blocked(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* hs_dev,
                                   uint64_t slab_budget, uint32_t* nblocks, void* stream) {
  if (!ctx || (npairs && (!pairs_dev || !hs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  if (ctx->live_qmc > 0)
    return nw::fail(ctx, NW_ERR_STATE, "a QMC object uses the intermediates (nw_qmc_destroy it first)");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::eval_blocked(ctx, pairs_dev, npairs, hs_dev, slab_budget, static_cast<cudaStream_t>(stream), nblocks);
}

nw_status nw_eval_hs_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* hs_dev,
                                  void* stream) {
  if (!ctx || (npairs && (!pairs_dev || !hs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_pairs(ctx, pairs_dev, npairs, hs_dev, nw::EvalMode::kHS, static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_hs_pairs_noalloc(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* hs_dev,
                                   void* stream) {
  if (!ctx || (npairs && (!pairs_dev || !hs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_pairs_noalloc(ctx, pairs_dev, npairs, hs_dev, static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_s_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* s_dev,
                                 void* stream) {
  if (!ctx || (npairs && (!pairs_dev || !s_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_pairs(ctx, pairs_dev, npairs, s_dev, nw::EvalMode::kS, static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_hs_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* hs_host, void* stream) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return eval_host(ctx, nw::EvalMode::kHS, pairs_host, npairs, hs_host, stream);
}

nw_status nw_update_fock(nw_ctx* ctx, const double* fock_a, const double* fock_b) {
  if (!ctx || !fock_a || !fock_b) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  const size_t n2 = (size_t)ctx->nao * ctx->nao;
  if (!finite_all(fock_a, n2) || !finite_all(fock_b, n2)) return nw::fail(ctx, NW_ERR_INVALID, "non-finite Fock matrix");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  return nw::update_fock(ctx, fock_a, fock_b);
}

nw_status nw_eval_fs_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* fs_dev,
                                  void* stream) {
  if (!ctx || (npairs && (!pairs_dev || !fs_dev))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return nw::eval_pairs(ctx, pairs_dev, npairs, fs_dev, nw::EvalMode::kFS, static_cast<cudaStream_t>(stream));
}

nw_status nw_eval_fs_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* fs_host, void* stream) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  return eval_host(ctx, nw::EvalMode::kFS, pairs_host, npairs, fs_host, stream);
}

nw_status nw_build_hs_matrix(nw_ctx* ctx, const uint32_t* left, uint64_t nl, const uint32_t* right, uint64_t nr,
                             int symmetric, double* h_out, double* s_out) {
  if (!ctx || (nl && !left) || (nr && !right) || (nl && nr && (!h_out || !s_out))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  return nw::build_matrix(ctx, nw::EvalMode::kHS, left, nl, right, nr, symmetric != 0, h_out, s_out);
}

nw_status nw_build_fs_matrix(nw_ctx* ctx, const uint32_t* left, uint64_t nl, const uint32_t* right, uint64_t nr,
                             int symmetric, double* f_out, double* s_out) {
  if (!ctx || (nl && !left) || (nr && !right) || (nl && nr && (!f_out || !s_out))) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (!ctx->fock_ready) return nw::fail(ctx, NW_ERR_STATE, "Fock tables not set (nw_update_fock)");
  return nw::build_matrix(ctx, nw::EvalMode::kFS, left, nl, right, nr, symmetric != 0, f_out, s_out);
}

nw_status nw_general_evp(nw_ctx* ctx, int32_t n, const double* h, const double* s, int project, double tol,
                         double* evals, double* c, int32_t* nkept) {
  if (!ctx || n <= 0 || !h || !s || !evals || !c || !nkept) return NW_ERR_INVALID;
  if (!(tol >= 0.0) || !std::isfinite(tol)) return NW_ERR_INVALID;
  const size_t n2 = (size_t)n * n;
  if (!finite_all(h, n2) || !finite_all(s, n2)) return nw::fail(ctx, NW_ERR_INVALID, "non-finite matrix entry");
  int k = 0;
  const nw_status st = nw::general_evp(ctx, n, h, s, project != 0, tol, evals, c, &k);
  *nkept = k;
  return st;
}

nw_status nw_sync(nw_ctx* ctx, void* stream) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  if (ctx->flag.p) {
    NW_CUDA(ctx, cudaMemcpyAsync(ctx->h_flag, ctx->flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  }
  NW_CUDA(ctx, cudaStreamSynchronize(s));
  if (ctx->flag.p && *ctx->h_flag) return nw::fail(ctx, NW_ERR_INVALID, "pair index out of range of the determinant basis");
  return NW_OK;
}

nw_status nw_set_timing(nw_ctx* ctx, int enable) {
  if (!ctx) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  if (enable < 0 || enable > 2) return NW_ERR_INVALID;
  if (enable && !ctx->ev[0]) {
    for (int i = 0; i < 8; ++i) NW_CUDA(ctx, cudaEventCreate(&ctx->ev[i]));
  }
  if (enable == 2 && !ctx->evc[0]) {
    for (int i = 0; i < 6; ++i) NW_CUDA(ctx, cudaEventCreate(&ctx->evc[i]));
  }
  ctx->timing = enable != 0;
  ctx->serial_classes = enable == 2;
  ctx->timed_valid = false;
  ctx->timed_classes = false;
  return NW_OK;
}

nw_status nw_last_class_timings(nw_ctx* ctx, float* ms) {
  if (!ctx || !ms) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (!ctx->timed_valid || !ctx->timed_classes)
    return nw::fail(ctx, NW_ERR_STATE, "no serially timed evaluation recorded (nw_set_timing(ctx, 2))");
  NW_CUDA(ctx, cudaEventSynchronize(ctx->evc[5]));
  for (int i = 0; i < 5; ++i) NW_CUDA(ctx, cudaEventElapsedTime(&ms[i], ctx->evc[i], ctx->evc[i + 1]));
  return NW_OK;
}

nw_status nw_last_timings(nw_ctx* ctx, float* ms) {
  if (!ctx || !ms) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (!ctx->timed_valid) return nw::fail(ctx, NW_ERR_STATE, "no timed evaluation recorded");
  NW_CUDA(ctx, cudaEventSynchronize(ctx->ev[5]));
  for (int i = 0; i < 4; ++i) NW_CUDA(ctx, cudaEventElapsedTime(&ms[i], ctx->ev[i], ctx->ev[i + 1]));
  ms[4] = 0.0f;
  if (ctx->timed_gen) NW_CUDA(ctx, cudaEventElapsedTime(&ms[4], ctx->ev[6], ctx->ev[7]));
  return NW_OK;
}

nw_status nw_ctx_info(const nw_ctx* ctx, nw_info* out) {
  if (!ctx || !out) return NW_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->nref = ctx->nref;
  out->nmo = ctx->nmo;
  out->ngeneric = ctx->built ? ctx->nresident - ctx->nfast : 0;
  out->slab_bytes = ctx->slab_bytes;
  out->ndet = ctx->ndet;
  return NW_OK;
}

nw_status nw_ctx_destroy(nw_ctx* ctx) {
  if (!ctx) return NW_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  double* bufs[] = {ctx->d_s, ctx->d_h, ctx->d_eri, ctx->d_chol, ctx->d_ca, ctx->d_cb, ctx->d_slab};
  for (double* b : bufs)
    if (b) cudaFree(b);
  if (ctx->d_fast) cudaFree(ctx->d_fast);
  if (ctx->d_gen) cudaFree(ctx->d_gen);
  if (ctx->d_order) cudaFree(ctx->d_order);
  if (ctx->d_dets) cudaFree(ctx->d_dets);
  if (ctx->d_desc) cudaFree(ctx->d_desc);
  nw::overlap_plan_free(ctx->ovl);
  for (double* b : {ctx->d_fbase, ctx->d_fock, ctx->d_fslab})
    if (b) cudaFree(b);
  if (ctx->d_fockp) cudaFree(ctx->d_fockp);
  free_buf(ctx->build_work);
  free_buf(ctx->bt_dets);
  free_buf(ctx->bt_desc);
  free_buf(ctx->bt_pairs);
  free_buf(ctx->bt_in);
  free_buf(ctx->keys);
  free_buf(ctx->ranks);
  free_buf(ctx->tsum);
  free_buf(ctx->perm);
  free_buf(ctx->counts);
  free_buf(ctx->offsets);
  free_buf(ctx->flag);
  free_buf(ctx->io_pairs);
  free_buf(ctx->io_hs);
  if (ctx->h_flag) cudaFreeHost(ctx->h_flag);
  for (int i = 0; i < 8; ++i)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  for (int i = 0; i < 6; ++i)
    if (ctx->evc[i]) cudaEventDestroy(ctx->evc[i]);
  for (cudaStream_t q : {ctx->s_in, ctx->s_comp, ctx->s_out, ctx->s_aux[0], ctx->s_aux[1], ctx->s_aux[2]})
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t e : {ctx->ev_start, ctx->ev_in[0], ctx->ev_in[1], ctx->ev_comp[0], ctx->ev_comp[1], ctx->ev_fork,
                        ctx->ev_join[0], ctx->ev_join[1], ctx->ev_join[2], ctx->ev_free})
    if (e) cudaEventDestroy(e);
  if (ctx->blas) cublasDestroy(ctx->blas);
  if (ctx->solver) cusolverDnDestroy(ctx->solver);
  delete ctx;
  return NW_OK;
}

}  // extern "C"
