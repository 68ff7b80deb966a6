/*
 * nociwick.h - C ABI of the B200 nonorthogonal Wick matrix-element engine.
 *
 * The engine evaluates overlap and Hamiltonian matrix elements (H_ij, S_ij) between
 * nonorthogonal determinants by the extended nonorthogonal Wick theorem, on one NVIDIA
 * B200 (sm_100a), with the per-reference-pair intermediates resident in HBM.  It replaces
 * the hot path of dy-cl/noci-rs, src/nonorthogonalwicks (Wick build + evaluators) and
 * src/noci/hs.rs (batched pair dispatch); each entry point names the reference interface it
 * stands in for.
 *
 * Conventions
 *  - Matrices are row-major FP64.  AO integrals are chemists' (mu nu|lam sig) stored as
 *    eri[((mu*n + nu)*n + lam)*n + sig], the PySCF int2e s1 order read by noci-rs.
 *  - Orbital coefficients C[mu][p] (nao x nmo).  A reference's occupied orbitals are the
 *    first nocc columns (noci-rs contraction_orbitals assumes the same).
 *  - A determinant is an nw_det record: parent reference, per-spin excitation rank and the
 *    first four hole then particle orbital indices (noci-rs ExcitationSpinCache), and the
 *    product of both spins' fermionic excitation phases (ReducedTwoSpinDetState.phase).
 *  - Pair (a, b) puts determinant a in the bra and b in the ket; results are written as
 *    hs[2*i] = H, hs[2*i + 1] = S.
 *  - Every call returns an nw_status; NW_OK is 0.  Nothing aborts the process.
 *  - A context owns its device memory.  Its entry points may be called from several host
 *    threads, each with its own stream: calls on one context are serialised (a per-context
 *    lock while a call enqueues its work, and on the device each call's work waits for the
 *    previous call's, since they share the context's scratch buffers); different contexts are
 *    independent.  nw_ctx_destroy must not race with other calls on the context, and calls of
 *    nw_eval_hs_pairs_noalloc must not overlap at all (its scratch is per process).
 */
#ifndef NOCIWICK_H
#define NOCIWICK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__) || defined(__clang__)
#define NW_API __attribute__((visibility("default")))
#else
#define NW_API
#endif

typedef enum {
    NW_OK = 0,
    NW_ERR_INVALID = 1,      /* bad argument or inconsistent input data            */
    NW_ERR_CUDA = 2,         /* a CUDA runtime or cuBLAS call failed               */
    NW_ERR_ALLOC = 3,        /* device or pinned host allocation failed            */
    NW_ERR_UNSUPPORTED = 4,  /* input outside what this build supports             */
    NW_ERR_STATE = 5,        /* call out of order (e.g. evaluate before build)     */
    NW_ERR_NO_DEVICE = 6,    /* no usable CUDA device                              */
    NW_ERR_IO = 7            /* a cache file could not be created, read or written  */
} nw_status;

/* Matrix-element conventions for reference pairs with zero-overlap orbital pairs (m > 0).
 * NW_CONVENTION_REFERENCE reproduces noci-rs xw_hamiltonian_overlap_gen_prepared
 * (src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:20550-20966) including its
 * treatment of singular mixed determinants, its (0,1)+(1,0) scalar term and the omitted
 * E_nuc*S.  NW_CONVENTION_EXACT returns the exact matrix element (checked against a
 * brute-force Fock-space evaluation).  Pairs without zero-overlap orbitals agree in both. */
typedef enum { NW_CONVENTION_REFERENCE = 0, NW_CONVENTION_EXACT = 1 } nw_convention;

/* One determinant (32 bytes).  Replaces noci-rs ExcitationCache + ReducedTwoSpinDetState
 * (src/lib.rs:136-167, :230-266) as the per-determinant input of the batched evaluator. */
typedef struct {
    uint32_t parent;     /* reference index                                          */
    uint8_t rank_a;      /* alpha excitation rank (0..4)                             */
    uint8_t idx_a[8];    /* alpha holes [0..3] then particles [4..7], ascending      */
    uint8_t rank_b;      /* beta excitation rank (0..4)                              */
    uint8_t idx_b[8];    /* beta holes then particles                                */
    uint8_t pad[2];
    double phase;        /* alpha phase * beta phase relative to the parent          */
} nw_det;

/* Excitation cache of one spin (noci-rs ExcitationSpinCache, src/lib.rs:151-167): rank and the
 * first four holes [0..3] then particles [4..7], ascending. */
typedef struct {
    uint8_t rank;
    uint8_t indices[8];
} nw_exc_spin;

/* Both spins of a determinant's excitation from its parent (noci-rs ExcitationCache,
 * src/lib.rs:136-149), the per-request input of xw_hamiltonian_overlap_prepared_batched. */
typedef struct {
    nw_exc_spin alpha;
    nw_exc_spin beta;
} nw_exc_cache;

/* AO data (noci-rs AoData, src/lib.rs:52-76): only the fields the Wick path reads. */
typedef struct {
    int32_t nao;         /* AO basis size                                            */
    int32_t nmo;         /* orbitals per spin per reference (== nao in noci-rs)      */
    double enuc;         /* nuclear repulsion energy                                 */
    const double* s;     /* nao x nao overlap                                        */
    const double* h;     /* nao x nao core Hamiltonian                               */
    const double* eri;   /* nao^4 Coulomb integrals (mu nu|lam sig)                  */
} nw_system;

/* AO data with the two-electron integrals in Cholesky-factored form:
 * (mu nu|lam sig) = sum_P chol[P][mu][nu] chol[P][lam][sig], each chol[P] symmetric, naux of
 * them.  The reference reads the full eri_coul tensor (AoData.eri_coul, src/read.rs:28-61);
 * this is the factored input of the same integrals. */
typedef struct {
    int32_t nao;
    int32_t nmo;
    int32_t naux;        /* Cholesky vectors                                         */
    int32_t pad;
    double enuc;
    const double* s;     /* nao x nao overlap                                        */
    const double* h;     /* nao x nao core Hamiltonian                               */
    const double* chol;  /* naux x nao x nao                                         */
} nw_system_cd;

/* Reference determinants (noci-rs DetState ca/cb/oa/ob, src/scalar.rs:30-61). */
typedef struct {
    int32_t nref;
    int32_t nocc_a;      /* occupied alpha orbitals per reference (first nocc_a)     */
    int32_t nocc_b;
    const double* c_alpha;  /* nref x nao x nmo                                      */
    const double* c_beta;   /* nref x nao x nmo                                      */
} nw_refs;

typedef struct {
    double tol;          /* singular values |s| <= tol are zero-overlap pairs (noci-rs tol) */
    int32_t convention;  /* nw_convention                                           */
    int32_t device;      /* CUDA device ordinal                                     */
} nw_opts;

typedef struct {
    int32_t nref;
    int32_t nmo;
    int32_t ngeneric;            /* ordered reference pairs with m_alpha + m_beta > 0   */
    int32_t pad;
    uint64_t slab_bytes;         /* device bytes held for intermediates                 */
    uint64_t ndet;               /* determinants in the resident basis                  */
} nw_info;

typedef struct nw_ctx nw_ctx;

/* Create a context: copies the AO data and reference orbitals to the device.
 * Replaces the inputs of noci-rs build_wicks_shared (src/noci/wicks.rs:133-139). */
NW_API nw_status nw_ctx_create(const nw_system* sys, const nw_refs* refs, const nw_opts* opts, nw_ctx** out);

/* The same from Cholesky-factored integrals: the factors are copied to the device and kept, and
 * the Coulomb tensor is formed there as L^T L on the engine's FP64 GEMM (nw_dgemm).  Every
 * other call works on such a context as on one made by nw_ctx_create. */
NW_API nw_status nw_ctx_create_cholesky(const nw_system_cd* sys, const nw_refs* refs, const nw_opts* opts,
                                        nw_ctx** out);

/* Build every ordered reference-pair intermediate on the GPU (Loewdin pairing by an FP64
 * Jacobi SVD, M^(0)/M^(1), X/Y, F, V, J and II tensors).
 * Replaces build_wicks_shared / build_wicks_pair (src/noci/wicks.rs:37-279) and
 * SameSpinBuild::new / DiffSpinBuild::new (src/nonorthogonalwicks/build.rs:86-926). */
NW_API nw_status nw_build_intermediates(nw_ctx* ctx);

/* How nw_build_intermediates forms the four-index J and II tensors (build.rs:261-313, :876-917,
 * eri_ao2mo_into, src/maths/eri.rs:258).  The Cholesky routes need a context made by
 * nw_ctx_create_cholesky: T(A,B,C,D)[pq][rs] = sum_P (A^T L^P B)[pq] (C^T L^P D)[rs], one
 * naux-deep product per tensor instead of four n^5 quarter transforms. */
typedef enum {
    NW_TRANSFORM_FP64 = 0,         /* four FP64 quarter transforms of the Coulomb tensor (default) */
    NW_TRANSFORM_CHOL_FP64 = 1,    /* Cholesky route, FP64 product on the FP64 tensor cores      */
    NW_TRANSFORM_CHOL_INT8 = 2,    /* Cholesky route on tcgen05: 8 signed int8 slices per factor
                                      (Ozaki split, exact int32 sums), rebuilt in FP64; at most
                                      16384 Cholesky vectors                                       */
    NW_TRANSFORM_CHOL_BF16X6 = 3   /* Cholesky route on tcgen05: 3 BF16 pieces per factor, the 6
                                      leading products summed in FP32 (FP32-class accuracy)        */
} nw_transform;

/* Select the transform of the next nw_build_intermediates (NW_ERR_STATE for a Cholesky mode on
 * a context without Cholesky factors). */
NW_API nw_status nw_set_transform(nw_ctx* ctx, int32_t mode);

/* The Cholesky-route product alone: t4[p][r][q][s] = sum_P u[P][p*n + q] v[P][r*n + s] for
 * P < naux, p, q, r, s < n, with mode NW_TRANSFORM_CHOL_FP64, _INT8 or _BF16X6 (device buffers,
 * synchronous).  No counterpart in the reference; exposed for checks of the split products. */
NW_API nw_status nw_transform_product(int32_t mode, const double* u, const double* v, int32_t naux, int32_t n,
                                      double* t4, void* stream);

/* Zero-overlap counts (m_alpha, m_beta) of ordered pair x*nref + w, as planned by
 * plan_wicks_pairs (src/noci/wicks.rs:90-121).  m must hold 2*nref*nref ints. */
/* Blocked (out-of-core) evaluation for systems whose intermediates exceed the device memory
 * (at n = 64 each ordered reference pair without zero-overlap orbitals holds 0.4 GB, so about
 * 20 references fill 180 GB): the ordered reference pairs are cut, in index order, into blocks
 * whose slab fits slab_budget bytes (0: the free device memory less 8 GB); each block is built
 * and the whole request evaluated against it, each block writing the (H, S) of its own
 * reference pairs.  Results equal one full build's bit for bit.  Device buffers, synchronous;
 * *nblocks (if not null) receives the number of blocks.  Afterwards the context holds the last
 * block, and the other evaluation, matrix, QMC, PT2 and cache calls return NW_ERR_STATE until
 * nw_build_intermediates (unless one block held every reference pair).  NW_ERR_ALLOC when one
 * reference pair alone exceeds the budget. */
NW_API nw_status nw_eval_hs_pairs_blocked(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* hs_dev,
                                          uint64_t slab_budget, uint32_t* nblocks, void* stream);

/* On-disk cache of the built intermediates (the counterpart of the reference's wicks.bin /
 * wicks.meta, src/nonorthogonalwicks/storage.rs:19,164-240): nw_save_intermediates writes the
 * slab (and the Fock basis the build keeps) to slab_path and the versioned per-reference-pair
 * tables to meta_path; nw_load_intermediates restores them into a context created with the same
 * system and options instead of nw_build_intermediates.  Loading checks the format version, the
 * geometry, tol, convention, transform and a hash of every input of the build (S, h, the
 * two-electron integrals or Cholesky vectors, the reference orbitals): a cache of another system
 * gives NW_ERR_INVALID, an unreadable file NW_ERR_IO.  The format is this engine's own slab
 * layout, not the reference's. */
NW_API nw_status nw_save_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path);
NW_API nw_status nw_load_intermediates(nw_ctx* ctx, const char* slab_path, const char* meta_path);

NW_API nw_status nw_pair_zero_counts(const nw_ctx* ctx, int32_t* m);

/* Upload the determinant basis once (host array of ndet records); it stays resident.
 * Replaces the reduced_basis argument of calculate_hs_pairs_wicks_batched (src/noci/hs.rs:72-78).
 * Returns NW_ERR_STATE while a QMC object of the context exists (it evaluates against the
 * resident basis every cycle). */
NW_API nw_status nw_set_basis(nw_ctx* ctx, const nw_det* basis, uint64_t ndet);

/* (H, S) for npairs requests (a_i, b_i) = pairs[2i], pairs[2i+1] into the resident basis,
 * with device-resident pairs and output.  Same-parent pairs more than a double excitation
 * apart give exactly (0, 0); every other pair goes through the Wick path.  The call is
 * asynchronous on `stream` (a cudaStream_t, or NULL for the legacy stream).
 * Replaces calculate_hs_pairs_wicks_batched (src/noci/hs.rs:72-130) and
 * xw_hamiltonian_overlap_prepared_batched (preparehamiltonianoverlap.rs:121-362). */
NW_API nw_status nw_eval_hs_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs,
                                  double* hs_dev, void* stream);

/* The same with host buffers: copies pairs in, evaluates, copies (H, S) out, and returns
 * when the results are in hs_host.  Pinned host memory gives the full transfer rate. */
NW_API nw_status nw_eval_hs_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* hs_host,
                           void* stream);

/* (H, S) exactly as nw_eval_hs_pairs_device, but without allocating device memory: for callers
 * that cannot call cudaMalloc while they evaluate pairs (a host whose memory pool already owns
 * nearly all of HBM, or a latency-critical loop that cannot take cudaMalloc's implicit
 * synchronisation or its failure path).  No counterpart in the reference.
 * Limits: at most 1,048,576 pairs per call and at most 64 references (larger requests return
 * NW_ERR_UNSUPPORTED).  The per-call scratch lives in one fixed device array of about 16 MB that
 * every GPU loading this library holds until the process exits; its device address is looked
 * up on the first call on each device, so make that first call before any stream capture.
 * All calls share the array: calls whose work overlaps on the GPU race and must be serialised.
 * Pair indices out of range of the basis give NaN results (this variant does not report them
 * through nw_sync). */
NW_API nw_status nw_eval_hs_pairs_noalloc(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs,
                                          double* hs_dev, void* stream);

/* Overlap only, S for each pair (hs_dev[i]), device buffers.
 * Replaces xw_overlap (src/nonorthogonalwicks/eval/overlap.rs:42-65) times the phases. */
NW_API nw_status nw_eval_s_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs, double* s_dev,
                                 void* stream);

/* The same with host buffers (copies in, evaluates, copies S out, returns when done); pair
 * indices out of range give NW_ERR_INVALID.  Replaces xw_overlap_same_f64_batched
 * (src/nonorthogonalwicks/eval/overlap.rs:2572-2856) as called by calculate_s_pair /
 * src/noci/overlap.rs:162-186. */
NW_API nw_status nw_eval_s_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* s_host,
                                 void* stream);

/* Overlap action over the resident basis: y_dev[w] += sum_x S_wx x_dev[x] for every determinant
 * w (device buffers of ndet doubles; y_dev must not alias x_dev).  S_wx is the same overlap as
 * nw_eval_s_pairs*, computed from single-spin factors: the determinants of one parent share their
 * alpha and beta strings, S_wx = A[a_w][a_x] B[b_w][b_x] for parents Q != P with A, B the
 * single-spin overlaps det(C_Q[:,occ]^T S C_P[:,occ]) of the two parents' strings, and the
 * determinants of one parent are orthonormal.  The first call on a basis builds the factor tables
 * (allocates about 8 (na_Q na_P + nb_Q nb_P) bytes per ordered pair of parents with na / nb
 * distinct alpha / beta strings per parent, and synchronises the stream; call it once before any
 * stream capture); later calls only launch kernels.  At most 16 occupied orbitals per spin.
 * Needs the resident basis (nw_set_basis), not the built intermediates.
 * Replaces SpinFactorisation::apply_overlap_sparse with build_overlap_factors
 * (src/noci/factorise/overlap.rs:280-498), as applied by apply_overlap_population_changes
 * (src/stochastic/metric.rs:97-232). */
NW_API nw_status nw_apply_overlap_device(nw_ctx* ctx, const double* x_dev, double* y_dev, void* stream);

/* (H, S) for npairs requests of one ordered reference pair (bra reference lp, ket reference gp)
 * from caller-held excitation caches: request i is the bra x[i] (a determinant of reference lp)
 * against the ket w[i] (of reference gp), with phase[i] the product of both determinants'
 * excitation phases; hs[2i] = H, hs[2i + 1] = S.  Host buffers; returns when the results are in
 * hs_out.  Caches are checked like a resident basis (ranks <= 4, holes ascending in the
 * occupied block, particles ascending in the virtual block, finite phase); a request that fails
 * gets NaN and the call returns NW_ERR_INVALID.  On a diagonal block (lp == gp) requests more
 * than a double excitation apart give exactly (0, 0).  Replaces
 * xw_hamiltonian_overlap_prepared_batched (src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:121-129)
 * with its requests' ExcitationCache pairs, and xw_hamiltonian_overlap_prepared (:53-61) for
 * one request. */
NW_API nw_status nw_eval_hs_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                                    const double* phase, uint64_t npairs, double* hs_out, void* stream);
/* The same with device buffers, asynchronous on `stream`; failed requests are reported by
 * nw_sync. */
NW_API nw_status nw_eval_hs_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                           const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs,
                                           double* hs_dev, void* stream);
/* Overlap only for the same per-reference-pair request blocks: s_out[i] = S.  Replaces
 * xw_overlap_same_f64_batched (src/nonorthogonalwicks/eval/overlap.rs:2572-2856) and
 * xw_overlap (:42-65) with the excitation phases. */
NW_API nw_status nw_eval_s_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                                   const double* phase, uint64_t npairs, double* s_out, void* stream);
NW_API nw_status nw_eval_s_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                          const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs,
                                          double* s_dev, void* stream);
/* Fock one-body element with the overlap for the same request blocks (after nw_update_fock):
 * fs_out[2i] = F, fs_out[2i + 1] = S.  Replaces xw_f_overlap_prepared
 * (src/nonorthogonalwicks/eval/prepareonebodyoverlap.rs:57) and xw_f (eval/onebody.rs:40). */
NW_API nw_status nw_eval_fs_batched(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x, const nw_exc_cache* w,
                                    const double* phase, uint64_t npairs, double* fs_out, void* stream);
NW_API nw_status nw_eval_fs_batched_device(nw_ctx* ctx, int32_t lp, int32_t gp, const nw_exc_cache* x_dev,
                                           const nw_exc_cache* w_dev, const double* phase_dev, uint64_t npairs,
                                           double* fs_dev, void* stream);

/* Fock tables for the (F, S) path from the AO Fock matrices of each spin (row-major nao x nao,
 * host memory): F^(mi,mj) = cx^(mi)^T F xc^(mj) and F_0^(m) = tr(M^(m) F) for every ordered
 * reference pair, from the pairing kept by nw_build_intermediates.  Call again whenever the
 * Fock matrices change (each SNOCI iteration).
 * Replaces update_wicks_fock (src/noci/wicks.rs:290-330) and
 * SameSpinBuild::construct_f_scalar (src/nonorthogonalwicks/build.rs:564-617). */
NW_API nw_status nw_update_fock(nw_ctx* ctx, const double* fock_a, const double* fock_b);

/* (F, S) per pair into fs_dev[2i], fs_dev[2i+1]: the Fock one-body element <x|F|w> and the
 * overlap, device buffers, asynchronous on `stream`.  The SNOCI operator element is
 * M = F - E0 S.  Same-parent pairs more than a double excitation apart give (0, 0).
 * Replaces xw_f_overlap_prepared (src/nonorthogonalwicks/eval/prepareonebodyoverlap.rs:57-100),
 * xw_f (eval/onebody.rs:40) and calculate_m_pair_wicks (src/noci/m.rs:160-197) before its
 * E0 shift. */
NW_API nw_status nw_eval_fs_pairs_device(nw_ctx* ctx, const uint32_t* pairs_dev, uint64_t npairs,
                                         double* fs_dev, void* stream);

/* The same with host buffers (copies in, evaluates, copies out, returns when done). */
NW_API nw_status nw_eval_fs_pairs(nw_ctx* ctx, const uint32_t* pairs_host, uint64_t npairs, double* fs_host,
                                  void* stream);

/* Dense (H, S) matrices of a block of the resident basis: h_out[i*nr + j] = H(left[i], right[j]),
 * likewise s_out (host, row-major nl x nr).  With symmetric != 0 (nl == nr) only j >= i is
 * evaluated and mirrored.  Pairs are generated and evaluated on the device in row blocks.
 * Replaces build_noci_hs with calculate_matrix_elements / scatter_matrix_elements
 * (src/noci/matrix.rs:39-110). */
NW_API nw_status nw_build_hs_matrix(nw_ctx* ctx, const uint32_t* left, uint64_t nl, const uint32_t* right,
                                    uint64_t nr, int symmetric, double* h_out, double* s_out);

/* The same for (F, S) after nw_update_fock.  Replaces build_noci_fock (src/noci/matrix.rs:124-175). */
NW_API nw_status nw_build_fs_matrix(nw_ctx* ctx, const uint32_t* left, uint64_t nl, const uint32_t* right,
                                    uint64_t nr, int symmetric, double* f_out, double* s_out);

/* Generalised eigenproblem H C = S C e in FP64 on the GPU (host row-major n x n inputs; only
 * the lower triangles enter the eigensolves, the full H enters X^T H X).  With project != 0 the
 * orthogonaliser is X = U_+ diag(lambda_+^-1/2) over the overlap eigenvalues > tol, else
 * X = U diag(lambda^-1/2) U^T.  Writes nkept = k eigenvalues (ascending) to evals and the
 * row-major n x k eigenvectors C = X U to c (room for n*n doubles).
 * Replaces general_evp / loewdin_x / positive_subspace (src/maths/linalg.rs:180-256). */
NW_API nw_status nw_general_evp(nw_ctx* ctx, int32_t n, const double* h, const double* s, int project, double tol,
                                double* evals, double* c, int32_t* nkept);

/* ---------------------------------------------------------------------------------------
 * NOCI-QMC on the GPU: signed real walkers over the resident basis, uniform excitation
 * generator, FRI sampling and spawn rounding, shift control.  The whole report block (ncycles
 * cycles of sample -> spawn -> (H, S) of every attempt -> rounding -> accumulation, then the
 * population update, statistics and shift update) runs on the device and is replayed as one
 * CUDA graph, with no host synchronisation inside a run.
 * Replaces qmc_step for the signed-walker propagators (src/stochastic/walkers.rs:101-441) with
 * propagate_iteration (src/stochastic/metric.rs:378-473), spawning / resolve_batched_spawning
 * with the uniform generator (src/stochastic/state.rs:537-726), sample_populations / fri
 * (metric.rs:579-699) and update_shift (metric.rs:729-751), and qmc_step of the direct-overlap
 * propagator (metric.rs:766-1087: the same cycles, then N += S Phi(Delta) per report through the
 * overlap action of nw_apply_overlap_device, inside the graph).  Random numbers come from a
 * counter-based Philox4x32-10 stream per (seed, cycle, index), so runs are reproducible for a
 * given seed but are not the reference's SmallRng sequence.
 * --------------------------------------------------------------------------------------- */
typedef enum nw_propagator {
    NW_PROP_UNSHIFTED = 0,       /* U = 1 - dt (H - E_s S)                      */
    NW_PROP_SHIFTED = 1,         /* U = (1 + dt E_s) - dt (H - E_s S)           */
    NW_PROP_DOUBLY_SHIFTED = 2,  /* as SHIFTED with E_s = E_s^S (the default)   */
    NW_PROP_DDS_U1 = 3,          /* difference doubly shifted, variant 1        */
    NW_PROP_DDS_U2 = 4,          /* difference doubly shifted, variant 2        */
    NW_PROP_DIRECT_OVERLAP = 5   /* real metric population N (N_0 = S c_0 scaled), cycles as
                                    UNSHIFTED, each report's change applied as N += S Phi(Delta)
                                    (qmc_step of src/stochastic/metric.rs:766-1087)            */
} nw_propagator;

typedef struct nw_qmc_opts {
    double dt;                  /* imaginary time step                                       */
    double initial_population;  /* 1-norm of the initial populations (scaled c0)             */
    double target_population;   /* 1-norm from which on the shift is updated                 */
    double sampling_cutoff;     /* FRI cutoff of the sampled populations (0: exact sampling) */
    double spawn_cutoff;        /* FRI cutoff of spawned amplitudes (0: none)                 */
    double shift_damping;       /* shift damping factor                                       */
    double initial_shift;       /* E_s at the start (noci-rs uses the first reference energy) */
    int32_t ncycles;            /* cycles per report block                                    */
    int32_t propagator;         /* nw_propagator                                              */
    uint64_t seed;
    uint64_t max_attempts;      /* spawning attempts one cycle can hold (0: 16 x the larger of
                                   the target and initial populations + 2 ndet + 2^20)        */
    double update_cutoff;       /* NW_PROP_DIRECT_OVERLAP: FRI cutoff of a report's accumulated
                                   change before the overlap is applied (sampling_cutoff2 of
                                   noci-rs; 0: none); ignored by the other propagators        */
} nw_qmc_opts;

typedef struct nw_qmc_report {
    double shift;               /* E_s after the block's update                               */
    double eproj_num;           /* projected energy = eproj_num / eproj_den                   */
    double eproj_den;
    double nw;                  /* 1-norm of the populations after the block                  */
    double nref;                /* 1-norm on the reference determinants                       */
    double sampled_norm;        /* 1-norm of the last cycle's sampled populations             */
    uint64_t nocc;              /* determinants with a non-zero sampled population            */
    uint64_t nattempts;         /* spawning attempts in the block                             */
} nw_qmc_report;

typedef struct nw_qmc nw_qmc;

/* Set up a run over the resident basis: diagonal (H, S), the projected-energy couplings
 * sum_i c0_i (H_iw, S_iw) over the reference determinants ref_idx, and the initial populations
 * initial_population * c0 / |c0|_1 (c0 has one entry per determinant).
 * Replaces the setup of qmc_step (walkers.rs:101-330) and initialise_populations (walkers.rs:27-48). */
NW_API nw_status nw_qmc_create(nw_ctx* ctx, const nw_qmc_opts* opts, const double* c0, const uint32_t* ref_idx,
                               uint64_t nref_idx, nw_qmc** out);
/* Run nreports report blocks; reports[k] receives block k's statistics (host array).
 * NW_ERR_UNSUPPORTED if a cycle needed more spawning attempts than max_attempts. */
NW_API nw_status nw_qmc_run(nw_qmc* q, int32_t nreports, nw_qmc_report* reports);
/* Replace the current shift E_s (restart, or an equilibration estimate). */
NW_API nw_status nw_qmc_set_shift(nw_qmc* q, double shift);
/* Device time of the report blocks of the last nw_qmc_run (CUDA events around the graph
 * launches on the run's stream), in milliseconds. */
NW_API nw_status nw_qmc_last_run_ms(const nw_qmc* q, float* ms);
/* Current populations (one per determinant), and replacing them (restart). */
NW_API nw_status nw_qmc_populations(nw_qmc* q, double* populations);
NW_API nw_status nw_qmc_set_populations(nw_qmc* q, const double* populations);
/* One cycle's population change from the current populations without applying it (for checks
 * of the estimator): delta = -dt (H - E^S S - E^I) sampled populations, stochastically. */
NW_API nw_status nw_qmc_cycle_delta(nw_qmc* q, uint64_t cycle, double* delta);
NW_API nw_status nw_qmc_destroy(nw_qmc* q);

/* Learned spawning proposal (no counterpart in the reference, which offers uniform,
 * heat-bath and overlap-weighted generators, src/input/qmc.rs:10).  Children are grouped into
 * bins (child reference x (rank_a, rank_b) class); a small MLP (descriptor of the parent:
 * one-hot reference, one-hot ranks, changed orbitals -> 128 -> 128 -> bins, ReLU, BF16 weights,
 * FP32 accumulation) gives p(bin | parent); a child is drawn from the mixture
 *   pgen = mix / (N - 1) + (1 - mix) p(bin | parent) / |bin without the parent|,
 * so every attempt still carries its exact generation probability and the spawn stays
 * unbiased.  The network is trained on the GPU (own forward, backward and Adam kernels) by the
 * weighted cross entropy -sum w log p(bin | parent) over harvested attempts with
 * w = |H - E^S S| / ((N - 1) pgen), whose minimiser puts each bin's probability in proportion
 * to its coupling mass.  Needs at most 8 references. */
typedef struct nw_mlp_opts {
    int32_t epochs;             /* passes over the harvested attempts                         */
    int32_t batch;              /* rows per Adam step (<= 4096)                               */
    double lr;                  /* Adam learning rate                                         */
    uint64_t seed;              /* minibatch draws                                            */
} nw_mlp_opts;

typedef struct nw_mlp_report {
    double loss_first;          /* loss of the first and last minibatch                        */
    double loss_last;
    uint64_t samples;           /* harvested attempts used                                     */
    int32_t steps;
    int32_t pad;
} nw_mlp_report;

/* Record (parent, child bin, weight) of the attempts of the following runs, each with
 * probability keep_probability in (0, 1] (an unbiased thinning, so that a long stretch of steps
 * fits the buffer); enable = 1 clears the buffer of 4,194,304 attempts, attempts beyond it are
 * not recorded. */
NW_API nw_status nw_qmc_harvest(nw_qmc* q, int32_t enable, double keep_probability);
/* Train the proposal network on the harvested attempts and rebuild p(bin | parent) for every
 * determinant. */
NW_API nw_status nw_qmc_train_proposal(nw_qmc* q, const nw_mlp_opts* opts, nw_mlp_report* rep);
/* Uniform generator (learned = 0) or the learned mixture with uniform weight mix in (0, 1]. */
NW_API nw_status nw_qmc_set_generator(nw_qmc* q, int32_t learned, double mix);
/* Network shape, parameters (layout W1[128][din], b1, W2[128][128], b2, W3[nbin][128], b3),
 * and the loss and parameter gradients of a given batch (for checks of the kernels). */
NW_API nw_status nw_qmc_proposal_dims(nw_qmc* q, int32_t* din, int32_t* nbin, uint64_t* nparams);
NW_API nw_status nw_qmc_mlp_params(nw_qmc* q, float* params);
NW_API nw_status nw_qmc_set_mlp_params(nw_qmc* q, const float* params);
NW_API nw_status nw_qmc_mlp_loss_grad(nw_qmc* q, const uint32_t* parents, const uint32_t* bins, const float* w,
                                      int32_t n, double* loss, float* grads);
/* p(bin | det) of the current network (nbin values; bins without a child of det are 0). */
NW_API nw_status nw_qmc_proposal_probs(nw_qmc* q, uint32_t det, double* probs);

/* Learned SNOCI candidate screener (no counterpart in the reference, which scores every
 * candidate of the pool by the exhaustive NOCI-PT2 solve, src/snoci/step.rs:330-460, and
 * selects with select_candidates, src/snoci/operators.rs:1064).  An MLP over the same
 * determinant descriptor as the learned proposal (din -> 128 -> 128 -> 1, ReLU, BF16 weight
 * copies, FP32 accumulation, Adam) regresses a target per determinant -- the caller passes
 * log10 of the selection score |a_a V_a| of candidates it scored exactly -- with a
 * mean-squared-error loss, trained on the GPU by the engine's own kernels.  Its predictions
 * rank a pool so that only its highest-ranked part enters the candidate matrix M and GMRES.
 * Indices refer to the context's resident basis at the time of the call (nw_set_basis). */
typedef struct nw_screen nw_screen;
NW_API nw_status nw_screen_create(nw_ctx* ctx, uint64_t seed, nw_screen** out);
/* Train (or, after the first call, fine-tune) on n rows; targets are standardised with the
 * mean and spread of the first call's targets. */
NW_API nw_status nw_screen_train(nw_screen* s, const uint32_t* idx, const double* target, uint64_t n,
                                 const nw_mlp_opts* opts, nw_mlp_report* rep);
/* Predicted targets of n resident determinants. */
NW_API nw_status nw_screen_predict(nw_screen* s, const uint32_t* idx, uint64_t n, double* out);
NW_API nw_status nw_screen_destroy(nw_screen* s);

/* ---------------------------------------------------------------------------------------
 * NOCI-PT2 / SNOCI linear solve: the candidate-candidate shifted Fock matrix M = F - E0 S
 * stored on the device (packed upper triangle, n (n + 1) / 2 doubles), its mat-vec, and
 * restarted right-preconditioned GMRES on the projected operator
 *   M^Omega x = M x - f_a0 (s_0a . x) - s_a0 (f_0a . x) + 2 E0 s_a0 (s_0a . x),
 * all in FP64.  Replaces build_candidate_m / fill_candidate_m and apply_candidate_m /
 * apply_omega_m (src/snoci/operators.rs:205-296, 375-488, 696-955), Preconditioner
 * (src/snoci/types.rs:138-288) and gmres (src/snoci/gmres.rs:406-544) for real states with no
 * imaginary shift.
 * --------------------------------------------------------------------------------------- */
typedef enum { NW_PRECOND_DIAG = 0, NW_PRECOND_WOODBURY = 1 } nw_preconditioner;

typedef struct nw_pt2_projection {
    double e0;                  /* zeroth-order energy E0                                    */
    const double* s_a0;         /* <Phi_a|Psi_0> per candidate (host, n)                     */
    const double* s_0a;         /* <Psi_0|Phi_a>                                             */
    const double* f_a0;         /* <Phi_a|F|Psi_0>                                           */
    const double* f_0a;         /* <Psi_0|F|Phi_a>                                           */
} nw_pt2_projection;

typedef struct nw_gmres_opts {
    int32_t max_iter;           /* total Arnoldi steps (noci-rs default 100)                  */
    int32_t restart;            /* Krylov dimension per cycle (default 200)                   */
    double res_tol;             /* |b - A x| / sqrt(n) at convergence (default 1e-8)          */
    int32_t preconditioner;     /* nw_preconditioner (noci-rs default Woodbury)               */
    int32_t pad;
} nw_gmres_opts;

typedef struct nw_gmres_info {
    double residual_rms;        /* true residual |b - A x| / sqrt(n)                          */
    int32_t iterations;
    int32_t converged;
} nw_gmres_info;

typedef struct nw_pt2 nw_pt2;

/* Build M = F - E0 S over candidates cand[0..n) of the resident basis (after nw_update_fock). */
NW_API nw_status nw_pt2_create(nw_ctx* ctx, const uint32_t* cand, uint64_t n, double e0, nw_pt2** out);
/* The same operator without storing M: every product (nw_pt2_apply_m, and each GMRES step of
 * nw_pt2_solve) evaluates the n (n + 1) / 2 upper-triangle (F, S) pairs again through the pair
 * pipeline in blocks of 2^26 and accumulates M x directly, so the device holds O(n) instead of
 * the n^2 / 2 doubles of the packed matrix.  Replaces apply_candidate_m without a cached matrix
 * (src/snoci/operators.rs:424-471). */
NW_API nw_status nw_pt2_create_matrix_free(nw_ctx* ctx, const uint32_t* cand, uint64_t n, double e0, nw_pt2** out);
/* y = M x (host vectors of n), the unprojected candidate mat-vec (apply_candidate_m). */
NW_API nw_status nw_pt2_apply_m(nw_pt2* p, const double* x, double* y);
/* Device time of the last nw_pt2_apply_m product (CUDA events), in milliseconds. */
NW_API nw_status nw_pt2_last_apply_ms(const nw_pt2* p, float* ms);
/* Solve M^Omega x = rhs by GMRES from x = 0 (host vectors). */
NW_API nw_status nw_pt2_solve(nw_pt2* p, const nw_pt2_projection* proj, const double* rhs, const nw_gmres_opts* opts,
                              double* x, nw_gmres_info* info);
NW_API nw_status nw_pt2_destroy(nw_pt2* p);

/* The engine's FP64 GEMM on the B200's FP64 tensor cores (DMMA), the product behind every dense
 * contraction of nw_build_intermediates: row-major, strided-batched, device buffers, asynchronous
 * on `stream`:  C[b] (m x n) = alpha op(A[b]) op(B[b]) + beta C[b]  for b < batch, where
 * op(A) = A^T when trans_a != 0 (A stored k x m, leading dimension lda) and likewise B (stored
 * n x k when transposed); a stride of 0 shares that operand across the batch.  Stands in for
 * the dense products of src/nonorthogonalwicks/build.rs (construct_xy, build_cx_xc,
 * build_j_coulomb / build_k_exchange, the F and V intermediates) and the four-index transform
 * eri_ao2mo_into (src/maths/eri.rs:258).  NW_ERR_INVALID for null pointers, negative sizes,
 * k == 0 with m, n > 0, more than 65535 batches or ceil(m / 64) > 65535. */
NW_API nw_status nw_dgemm(int trans_a, int trans_b, int m, int n, int k, double alpha, const double* a, int lda,
                          long long stride_a, const double* b, int ldb, long long stride_b, double beta, double* c,
                          int ldc, long long stride_c, int batch, void* stream);

/* Wait for the work queued on `stream` and report pair indices that were out of range in an
 * earlier device-buffer call (those outputs are NaN). */
NW_API nw_status nw_sync(nw_ctx* ctx, void* stream);

/* Autotuner (no counterpart in the reference): times nw_eval_hs_pairs_device on the caller's
 * device pairs (npairs of them, results into hs) for fine sort-key budgets 2^14 .. 2^23 and
 * 4 / 8 / 16 blocks per SM of the grid-stride kernels, against the defaults, and keeps the
 * fastest for the later calls on this context, the budget as keys per pair so that calls of
 * other sizes scale it (budget 0 and blocks 0 in the report mean the defaults won).
 * Synchronises `stream`. */
typedef struct nw_tune_report {
    uint64_t key_budget;        /* chosen fine-key budget (0: default, min(2^23, max(2^14, npairs))) */
    int32_t blocks_per_sm;      /* chosen blocks per SM (0: default 8)                           */
    int32_t trials;             /* configurations timed                                         */
    float best_ms;              /* per call, chosen configuration                               */
    float default_ms;           /* per call, defaults                                           */
} nw_tune_report;
NW_API nw_status nw_autotune(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* hs, void* stream,
                             nw_tune_report* rep);

/* Per-phase device times of the most recent nw_eval_hs_pairs* call, measured with CUDA events
 * recorded on its stream while timing is enabled: ms[0] classify, ms[1] scan, ms[2] scatter,
 * ms[3] the evaluators (the m = 0 classes and the m > 0 generic evaluator run concurrently on
 * forked streams, so they are timed together), ms[4] the m > 0 generic evaluator alone (events
 * on its forked stream; 0 when the call had no such pair).  nw_last_timings waits for that call.
 * enable = 2 is a profiling mode: the class evaluators run one after another on the call's
 * stream (same kernels and work, no overlap), and nw_last_class_timings gives each one's device
 * time: ms[0] light, ms[1] medium, ms[2] heavy, ms[3] runtime rank, ms[4] the m > 0 generic
 * evaluator (the F+S path has no medium and runtime-rank kernels: 0 there). */
NW_API nw_status nw_set_timing(nw_ctx* ctx, int enable);
NW_API nw_status nw_last_timings(nw_ctx* ctx, float* ms);
NW_API nw_status nw_last_class_timings(nw_ctx* ctx, float* ms);

NW_API nw_status nw_ctx_info(const nw_ctx* ctx, nw_info* out);
NW_API nw_status nw_ctx_destroy(nw_ctx* ctx);
NW_API const char* nw_status_string(nw_status st);
/* Text of the last error recorded on ctx (empty string if none). */
NW_API const char* nw_last_error(const nw_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* NOCIWICK_H */
