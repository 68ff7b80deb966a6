// Internal types of the B200 Wick engine: device-side pair tables, the context, and the
// small dense linear algebra used by the pair evaluators.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <stdint.h>

#include <mutex>

#include <string>
#include <vector>

#include "../../include/nociwick.h"
#include "wick_math.cuh"

namespace nw {

constexpr int kMaxL = 8;          // largest contraction-determinant dimension per spin
constexpr int kClasses = kRankClasses;  // (L_alpha, L_beta) in 0..4 x 0..4, plus one "other" class
constexpr uint32_t kSkipKey = 0xFFFFFFFFu;

struct EvalParams {
  const nw_det* dets;
  uint64_t ndet;
  const FastPair* fast;    // indexed by ordered pair x*nref + w
  const GenPair* gen;      // indexed by ordered pair x*nref + w
  const int32_t* order;    // ordered pair -> sort position (fast pairs first)
  int32_t nref, n, nocc_a, nocc_b;
  int32_t nfast;           // number of fast ordered pairs (sort positions 0..nfast-1)
  int32_t exact;
  const uint16_t* desc;    // per-determinant class descriptor (det_desc)
  const FockPair* fock;    // Fock tables (after nw_update_fock), indexed like fast/gen
  uint32_t nbucket;        // sort keys per rank class for fast pairs (pair_sort_key)
  int32_t shift;
  double enuc, tol;
};

// ---------------------------------------------------------------------------------------
// Context.
// ---------------------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// Spin-factorised overlap action over the resident basis (overlap.cu).
struct OverlapPlan;

}  // namespace nw

struct nw_ctx {
  int device = 0;
  int nao = 0, nmo = 0, nref = 0, nocc_a = 0, nocc_b = 0;
  double enuc = 0.0, tol = 1e-8;
  int convention = NW_CONVENTION_REFERENCE;
  bool built = false;

  // inputs on the device
  double* d_s = nullptr;
  double* d_h = nullptr;
  double* d_eri = nullptr;
  double* d_chol = nullptr; // naux x nao x nao Cholesky vectors (nw_ctx_create_cholesky), else null
  int naux = 0;
  int transform = NW_TRANSFORM_FP64;  // four-index transform of the build (nw_set_transform)
  nw::DevBuf chol_work;     // Cholesky-route factors, split pieces and error word of the build
  double* d_ca = nullptr;   // nref x nao x nmo
  double* d_cb = nullptr;

  // intermediates
  double* d_slab = nullptr;
  size_t slab_bytes = 0;
  size_t slab_capacity = 0;        // bytes allocated at d_slab (>= slab_bytes)
  nw::DevBuf build_work;           // workspace of the build, kept for rebuilds
  nw::FastPair* d_fast = nullptr;
  nw::GenPair* d_gen = nullptr;
  int32_t* d_order = nullptr;
  int nfast = 0;
  int nresident = 0;               // ordered pairs whose slab pieces are built (sort positions)
  bool partial = false;            // the slab holds one block of a blocked evaluation
  bool allow_partial = false;      // set by the blocked evaluation while it evaluates a block
  std::vector<int32_t> m_counts;   // 2 per ordered pair
  std::vector<int32_t> order_host; // ordered pair -> sort position

  // resident basis
  nw_det* d_dets = nullptr;
  uint16_t* d_desc = nullptr;      // det_desc of every record
  uint64_t ndet = 0;
  nw::OverlapPlan* ovl = nullptr;  // factor tables of the overlap action, built on first use

  // evaluation scratch (grown on demand)
  nw::DevBuf keys, perm, counts, offsets, flag, ranks, tsum;
  uint32_t* h_flag = nullptr;      // pinned mirror of the device error flag
  nw::DevBuf io_pairs, io_hs;      // staging for the host-buffer entry point
  // determinant records, descriptors and pairs packed from caller excitation caches
  // (nw_eval_hs_batched), and their device staging for host-buffer calls
  nw::DevBuf bt_dets, bt_desc, bt_pairs, bt_in;
  // copy-in / evaluate / copy-out streams and chunk events of the pipelined host-buffer path
  cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
  // class evaluators forked off the launching stream (medium ranks; heavy and runtime ranks;
  // the zero-overlap generic evaluator)
  cudaStream_t s_aux[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_start = nullptr;
  // Calls on one context from several host threads (each on its own stream) are serialised:
  // the guard holds mtx while a call enqueues its work, and the work of one call waits for the
  // previous call's (ev_free, recorded on that call's stream), since both use the context's
  // scratch buffers.
  std::recursive_mutex mtx;
  cudaEvent_t ev_free = nullptr;
  bool ev_free_used = false;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr};

  // Fock (F + S) path: per (pair, spin) [M^(0), M^(1), cx^(0), cx^(1), xc^(0), xc^(1)] kept
  // from the build, the AO Fock matrices, their per-pair tables and records
  double* d_fbase = nullptr;        // 2 nref^2 x 6 x n^2
  double* d_fock = nullptr;         // F_alpha, F_beta (nao x nao each)
  double* d_fslab = nullptr;
  nw::FockPair* d_fockp = nullptr;  // nref^2
  bool fock_ready = false;
  std::vector<nw::FastPair> fast_host;
  std::vector<nw::GenPair> gen_host;
  std::vector<char> generic_host;  // per ordered pair: m_alpha + m_beta > 0

  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;  // created by the first generalised eigensolve
  std::string last_error;

  // optional per-phase timing of the evaluation pipeline; serial_classes runs the class
  // evaluators one after another on the launching stream, each between two of evc[0..5]
  bool timing = false;
  bool serial_classes = false;
  // launch configuration chosen by nw_autotune (0: defaults)
  double tune_keys_per_pair = 0.0;  // fine sort-key budget of nw_eval_hs_pairs* per pair
  int live_qmc = 0;                 // QMC objects evaluating against the resident basis
  int tune_per_sm = 0;            // blocks per SM of classify / scatter / light evaluator
  bool timed_valid = false;
  bool timed_gen = false;           // the last timed call ran the m > 0 evaluator (ev[6], ev[7])
  // phase events: ev[0..5] on the launching stream, ev[6] / ev[7] around the m > 0 evaluator on
  // its forked stream
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t evc[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool timed_classes = false;       // the last timed call recorded evc (serial_classes)
};

namespace nw {

// Serialises one entry point's use of a context (see nw_ctx::mtx): the stream of the call first
// waits for the work of the previous call on the context, and the call's end is recorded for
// the next one.
struct CtxGuard {
  nw_ctx* ctx;
  cudaStream_t stream;
  CtxGuard(nw_ctx* c, cudaStream_t s) : ctx(c), stream(s) {
    ctx->mtx.lock();
    if (ctx->ev_free_used) cudaStreamWaitEvent(stream, ctx->ev_free, 0);
  }
  ~CtxGuard() {
    if (ctx->ev_free && cudaEventRecord(ctx->ev_free, stream) == cudaSuccess) ctx->ev_free_used = true;
    ctx->mtx.unlock();
  }
  CtxGuard(const CtxGuard&) = delete;
  CtxGuard& operator=(const CtxGuard&) = delete;
};


// Pipelined host-buffer path: about kPipeChunks chunks of at least kPipeMinChunk pairs.
constexpr uint64_t kPipeChunks = 16;
constexpr uint64_t kPipeMinChunk = 1ull << 18;

// Records an error on the context and returns the status.
nw_status fail(nw_ctx* ctx, nw_status st, const std::string& msg);
nw_status cuda_fail(nw_ctx* ctx, cudaError_t e, const char* what);
nw_status ensure(nw_ctx* ctx, DevBuf& b, size_t bytes);

// Row-major, strided-batched FP64 GEMM on the FP64 tensor cores (dgemm.cu):
// C[b] (M x N) = alpha op(A[b]) op(B[b]) + beta C[b], op(X) = X^T when the flag is set
// (A stored K x M, B stored N x K); a batch stride of 0 shares the operand.
cudaError_t dgemm_strided(cudaStream_t stream, bool ta, bool tb, int M, int N, int K, double alpha, const double* A,
                          int lda, long long sa, const double* B, int ldb, long long sb, double beta, double* C,
                          int ldc, long long sc, int batch);

// Cholesky-route product on tcgen05 (tc_gemm.cu): t4[p][r][q][s] = sum_k U[k][pq] V[k][rs] with
// mode NW_TRANSFORM_CHOL_INT8 (8 int8 Ozaki slices) or NW_TRANSFORM_CHOL_BF16X6 (3 BF16 pieces).
constexpr int kOzakiSlices = 8;
// A factor F[k][row] (naux x R) split into pre-tiled pieces (and, for int8, per-row exponents).
struct SplitFactor {
  int mode, R, rpad, nkt;
  long long piece_bytes;
  uint8_t* pieces;
  int* exps;
};
size_t split_factor_bytes(int mode, int naux, int R);
cudaError_t split_factor(cudaStream_t st, int mode, const double* F, int naux, int R, void* buf, size_t bytes,
                         SplitFactor* out);
cudaError_t split_product(cudaStream_t st, const SplitFactor& A, const SplitFactor& B, int n, double* out,
                          uint32_t* err);
size_t split_product_scratch(int mode, int naux, int M, int N, int slices);
cudaError_t split_product_pqrs(cudaStream_t st, int mode, int slices, const double* U, const double* V, int naux, int n,
                               double* out, void* scratch, size_t scratch_bytes, uint32_t* err);
// [p][q][r][s] -> [p][r][q][s] of an n^4 tensor (build.cu).
cudaError_t swap_qr(cudaStream_t st, const double* src, int n, double* dst);

// Build (build.cu).
// Build of the intermediates of every ordered reference pair, or of the pairs flagged in
// `subset` (nref^2 flags; the others get sort position -1 and are skipped by the evaluators).
nw_status build_all(nw_ctx* ctx, const std::vector<char>* subset = nullptr);
// Slab doubles of one ordered reference pair with zero-overlap counts (ma, mb).
size_t pair_slab_doubles(int n, int ma, int mb);
// Blocked evaluation of (H, S) over blocks of reference pairs whose slab fits `budget` bytes.
nw_status eval_blocked(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* hs, uint64_t budget,
                       cudaStream_t stream, uint32_t* nblocks);
// On-disk cache of the built intermediates (storage.cu).
nw_status save_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path);
nw_status load_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path);
// Fock tables from AO Fock matrices (build.cu).
nw_status update_fock(nw_ctx* ctx, const double* fa, const double* fb);

// What a pair evaluation produces.
enum class EvalMode { kHS, kS, kFS };

// Evaluation (eval.cu).
// clear_flag = false keeps the out-of-range flag of earlier calls (chunked host path).
nw_status eval_pairs(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* out, EvalMode mode,
                     cudaStream_t stream, bool clear_flag = true);
// The same over a caller-supplied determinant table (P.dets / P.desc / P.ndet), e.g. the records
// packed from excitation caches by nw_eval_hs_batched.
nw_status eval_pairs_on(nw_ctx* ctx, EvalParams P, const uint32_t* pairs, uint64_t npairs, double* out, EvalMode mode,
                        cudaStream_t stream, bool clear_flag = true);
// Dense matrices over left x right determinant blocks and the generalised eigenproblem (matrix.cu).
nw_status build_matrix(nw_ctx* ctx, EvalMode mode, const uint32_t* left, uint64_t nl, const uint32_t* right,
                       uint64_t nr, bool symmetric, double* a_host, double* s_host);
nw_status general_evp(nw_ctx* ctx, int n, const double* h, const double* s, bool project, double tol, double* evals,
                      double* c, int* nkept);

// Device scratch of one sorted evaluation (classify -> scan -> scatter -> evaluate).
struct SortScratch {
  uint32_t* keys;     // npairs
  uint32_t* ranks;    // npairs
  uint32_t* sidx;     // npairs
  uint32_t* counts;   // nkeys
  uint32_t* offsets;  // nkeys + 1
  uint32_t* tsum;     // nkeys / 4096 + 1
  uint32_t* flag;
  uint32_t* work;     // chunk counter of the m > 0 evaluators (a word of the flag buffer, >= 64 bytes)
};

// Fine-key budget of the sort (pair_sort_key): at most kFineMax counters, and at most about one
// per pair of the request so the counter memset and scan stay small next to the evaluation.
constexpr uint64_t kFineMax = 1ull << 23;
constexpr uint64_t kFineMin = 1ull << 14;

EvalParams make_params(const nw_ctx* ctx);
// Number of sort keys with at most `cap` counters for the fast classes; fills P.nbucket/P.shift.
uint64_t plan_keys(const nw_ctx* ctx, EvalParams& P, uint64_t cap);
// classify -> scan -> scatter -> evaluate on `stream` (no allocation, no host synchronisation).
// With npairs_dev the number of pairs is read on the device (at most npairs, the capacity the
// launch is sized for); ev (eight events or null) brackets the phases.  With classified the
// caller has already cleared S.counts and written S.keys / S.ranks (and the outputs of
// skipped pairs), e.g. the fused QMC spawn kernel, and the pipeline starts at the scan.
nw_status launch_sorted(nw_ctx* ctx, const EvalParams& P, uint64_t nkeys, const uint32_t* pairs, uint64_t npairs,
                        double* out, const SortScratch& S, cudaStream_t stream, cudaEvent_t* ev,
                        EvalMode mode = EvalMode::kHS, const uint32_t* npairs_dev = nullptr,
                        bool classified = false);

// Exclusive scan of n counters into offsets[0..n] (offsets[n] = total); tsum holds n / 4096 + 1.
nw_status scan_exclusive(nw_ctx* ctx, const uint32_t* counts, uint64_t n, uint32_t* offsets, uint32_t* tsum,
                         cudaStream_t stream);

// Overlap action y += S x over the resident basis (overlap.cu): the plan (spin components,
// factor tables, work buffers) is built on first use, allocates and synchronises `stream`, and
// stays with the context until the basis changes; an apply only launches kernels.
nw_status overlap_plan_get(nw_ctx* ctx, cudaStream_t stream, OverlapPlan** out);
nw_status overlap_apply(nw_ctx* ctx, const OverlapPlan* plan, const double* x, double* y, cudaStream_t stream);
void overlap_plan_free(OverlapPlan* plan);

// Same evaluation with its scratch in a fixed device array (no device allocation).
nw_status eval_pairs_noalloc(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* out, cudaStream_t stream);

}  // namespace nw

#define NW_CUDA(ctx, call)                                  \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return nw::cuda_fail(ctx, e_, #call); \
  } while (0)
