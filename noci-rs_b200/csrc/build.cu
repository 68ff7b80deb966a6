// GPU build of the per-reference-pair Wick intermediates (FP64).
//
// For every ordered reference pair (x, w) and spin this computes, on the device:
//   Loewdin pairing of the occupied overlap by a Jacobi SVD      build.rs:401-424
//   M^(0) = W + P_xw + P_ww, M^(1) = P_xw                          build.rs:447-503
//   X^(m), Y^(m) in the contraction row/column spaces              build.rs:526-542
//   cx^(m), xc^(m) partial transforms                              build.rs:944-991
//   JK^(m) = J(M^(m)) - K(M^(m)), J(M^(m)) (Coulomb only)          build.rs:627-683
//   F0, F^(mi,mj), V0, V^(mi,mj,mk), V^alpha, V^beta, V_ab,0        build.rs:198-259, :808-874
//   J^(m1..m4) and II^(ma0,maz,mb0,mby) four-index tensors         build.rs:261-313, :876-917
// and packs them into the evaluator layout: pairs without zero-overlap orbitals get the
// fast layout (records {X0|Y0, hcol0}, antisymmetrised J^(0000), II^(0000)); the others keep
// the full reference-ordered set.  Dense products run on the engine's FP64 tensor-core GEMM
// (dgemm.cu); pairing, contractions and layout transforms are kernels in this file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "internal.cuh"
#include "wick_math.cuh"

namespace nw {
namespace {

#define NW_DG(ctx, call)                                                               \
  do {                                                                                 \
    const cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) return nw::cuda_fail(ctx, e_, #call);                       \
  } while (0)

// Row-major C(MxN) = op(A)(MxK) op(B)(KxN) on the engine's FP64 tensor-core GEMM (dgemm.cu),
// on the build's stream.
inline cudaError_t gemm(cudaStream_t h, bool ta, bool tb, int M, int N, int K, double alpha, const double* A, int lda,
                        const double* B, int ldb, double beta, double* C, int ldc) {
  return dgemm_strided(h, ta, tb, M, N, K, alpha, A, lda, 0, B, ldb, 0, beta, C, ldc, 0, 1);
}

inline cudaError_t gemm_b(cudaStream_t h, bool ta, bool tb, int M, int N, int K, double alpha, const double* A,
                          int lda, long long sa, const double* B, int ldb, long long sb, double beta, double* C,
                          int ldc, long long sc, int batch) {
  return dgemm_strided(h, ta, tb, M, N, K, alpha, A, lda, sa, B, ldb, sb, beta, C, ldc, sc, batch);
}

// y[b][i] += alpha x[b][i] for a batch of vectors at strides sx, sy.
__global__ void axpy_batched_kernel(double alpha, const double* __restrict__ x, long long sx, double* __restrict__ y,
                                    long long sy, long long n) {
  const double* xb = x + blockIdx.y * sx;
  double* yb = y + blockIdx.y * sy;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    yb[i] += alpha * xb[i];
}

// Bump allocator over one device buffer, 256-byte aligned pieces.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  double* take(size_t ndouble) {
    const size_t bytes = ((ndouble * sizeof(double) + 255) / 256) * 256;
    if (used + bytes > cap) return nullptr;
    double* p = reinterpret_cast<double*>(base + used);
    used += bytes;
    return p;
  }
};

struct PairSpinMeta {
  double phase, tsp;
  int m, o;
};

// One block per (ordered pair, spin): occupied overlap, Jacobi SVD, canonical null gauge,
// phase det(U) det(V), rotated occupied orbitals.
__global__ void pairing_kernel(const double* __restrict__ S, const double* __restrict__ Ca,
                               const double* __restrict__ Cb, int nref, int nao, int nmo, int oa, int ob, double tol,
                               int omax, double* __restrict__ ctx_out, double* __restrict__ ctw_out,
                               double* __restrict__ sv_out, PairSpinMeta* __restrict__ meta) {
  const int ps = blockIdx.x;
  const int p = ps >> 1, spin = ps & 1;
  const int x = p / nref, w = p % nref;
  const int o = spin ? ob : oa;
  const double* Cx = (spin ? Cb : Ca) + (size_t)x * nao * nmo;
  const double* Cw = (spin ? Cb : Ca) + (size_t)w * nao * nmo;
  extern __shared__ double sm[];
  double* scw = sm;            // nao * o
  double* A = scw + nao * o;   // o * o
  double* U = A + o * o;
  double* V = U + o * o;
  double* s = V + o * o;       // o
  for (int idx = threadIdx.x; idx < nao * o; idx += blockDim.x) {
    const int mu = idx / o, k = idx % o;
    double acc = 0.0;
    for (int nu = 0; nu < nao; ++nu) acc += S[(size_t)mu * nao + nu] * Cw[(size_t)nu * nmo + k];
    scw[idx] = acc;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < o * o; idx += blockDim.x) {
    const int i = idx / o, k = idx % o;
    double acc = 0.0;
    for (int mu = 0; mu < nao; ++mu) acc += Cx[(size_t)mu * nmo + i] * scw[mu * o + k];
    A[idx] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    jacobi_svd(o, A, U, V, s, tol);
    canonical_null_columns(o, U, s, tol);
    canonical_null_columns(o, V, s, tol);
    // det(U) det(V) with A as LU scratch
    for (int i = 0; i < o * o; ++i) A[i] = U[i];
    const double du = det_lu_inplace(A, o);
    for (int i = 0; i < o * o; ++i) A[i] = V[i];
    const double dv = det_lu_inplace(A, o);
    double tsp = 1.0;
    int m = 0;
    for (int k = 0; k < o; ++k) {
      if (fabs(s[k]) > tol)
        tsp *= s[k];
      else
        ++m;
    }
    meta[ps].phase = du * dv;
    meta[ps].tsp = tsp;
    meta[ps].m = m;
    meta[ps].o = o;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nao * o; idx += blockDim.x) {
    const int mu = idx / o, k = idx % o;
    double ax = 0.0, aw = 0.0;
    for (int i = 0; i < o; ++i) {
      ax += Cx[(size_t)mu * nmo + i] * U[i * o + k];
      aw += Cw[(size_t)mu * nmo + i] * V[i * o + k];
    }
    ctx_out[((size_t)ps * nao + mu) * omax + k] = ax;
    ctw_out[((size_t)ps * nao + mu) * omax + k] = aw;
  }
  for (int k = threadIdx.x; k < o; k += blockDim.x) sv_out[(size_t)ps * omax + k] = s[k];
}

// M^(0), M^(1) for every (pair, spin); M laid out [ps][2][nao][nao].
__global__ void m_kernel(const double* __restrict__ ctx, const double* __restrict__ ctw, const double* __restrict__ sv,
                         const PairSpinMeta* __restrict__ meta, int nao, int omax, double tol, double* __restrict__ M) {
  const int ps = blockIdx.y;
  const int o = meta[ps].o;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nao * nao; idx += gridDim.x * blockDim.x) {
    const int mu = idx / nao, nu = idx % nao;
    double m0 = 0.0, m1 = 0.0;
    for (int k = 0; k < o; ++k) {
      const double sk = sv[(size_t)ps * omax + k];
      const double cw = ctw[((size_t)ps * nao + mu) * omax + k];
      const double cx = ctx[((size_t)ps * nao + nu) * omax + k];
      if (fabs(sk) > tol) {
        m0 += cw * (1.0 / sk) * cx;
      } else {
        const double cwn = ctw[((size_t)ps * nao + nu) * omax + k];
        m0 += cw * cwn + cw * cx;
        m1 += cw * cx;
      }
    }
    M[((size_t)ps * 2 + 0) * nao * nao + idx] = m0;
    M[((size_t)ps * 2 + 1) * nao * nao + idx] = m1;
  }
}

// Row/column orbital spaces (build.rs:1008-1031) and per-(pair, spin) copies of C_x, C_w.
__global__ void spaces_kernel(const double* __restrict__ Ca, const double* __restrict__ Cb, int nref, int nao,
                              int nmo, int oa, int ob, double* __restrict__ rowc, double* __restrict__ colc,
                              double* __restrict__ cxs, double* __restrict__ cws) {
  const int ps = blockIdx.y;
  const int p = ps >> 1, spin = ps & 1;
  const int x = p / nref, w = p % nref;
  const int o = spin ? ob : oa;
  const double* Cx = (spin ? Cb : Ca) + (size_t)x * nao * nmo;
  const double* Cw = (spin ? Cb : Ca) + (size_t)w * nao * nmo;
  const int nv = nmo - o;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nao * nmo; idx += gridDim.x * blockDim.x) {
    const int mu = idx / nmo, c = idx % nmo;
    const size_t off = (size_t)ps * nao * nmo + idx;
    rowc[off] = (c < nv) ? Cx[(size_t)mu * nmo + o + c] : Cw[(size_t)mu * nmo + (c - nv)];
    colc[off] = (c < o) ? Cx[(size_t)mu * nmo + c] : Cw[(size_t)mu * nmo + c];
    cxs[off] = Cx[(size_t)mu * nmo + c];
    cws[off] = Cw[(size_t)mu * nmo + c];
  }
}

// cx^(m) = [ (M^T S C_x - (1-m) C_x)[:, o:] | (M^T S C_w)[:, :o] ],
// xc^(m) = [ (M S C_x)[:, :o] | (M S C_w - (1-m) C_w)[:, o:] ]   (build.rs:944-991).
__global__ void cxxc_kernel(const double* __restrict__ mtsx, const double* __restrict__ mtsw,
                            const double* __restrict__ msx, const double* __restrict__ msw,
                            const double* __restrict__ cxs, const double* __restrict__ cws, int nao, int nmo, int oa,
                            int ob, double* __restrict__ cx, double* __restrict__ xc) {
  const int psm = blockIdx.y;  // (ps, m)
  const int ps = psm >> 1, m = psm & 1;
  const int spin = ps & 1;
  const int o = spin ? ob : oa;
  const int nv = nmo - o;
  const double f = (double)(1 - m);
  const size_t base = (size_t)psm * nao * nmo;
  const size_t cbase = (size_t)ps * nao * nmo;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nao * nmo; idx += gridDim.x * blockDim.x) {
    const int mu = idx / nmo, c = idx % nmo;
    double l, r;
    if (c < nv) {
      const int j = o + c;
      l = mtsx[base + (size_t)mu * nmo + j] - f * cxs[cbase + (size_t)mu * nmo + j];
    } else {
      const int j = c - nv;
      l = mtsw[base + (size_t)mu * nmo + j];
    }
    if (c < o) {
      r = msx[base + (size_t)mu * nmo + c];
    } else {
      r = msw[base + (size_t)mu * nmo + c] - f * cws[cbase + (size_t)mu * nmo + c];
    }
    cx[base + idx] = l;
    xc[base + idx] = r;
  }
}

// G[(s,t),(mu,nu)] = (st|mu nu) - (s mu|nu t)
__global__ void g_kernel(const double* __restrict__ eri, int n, double* __restrict__ G) {
  const size_t n2 = (size_t)n * n, n4 = n2 * n2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n4; idx += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(idx / (n2 * n));
    const int t = (int)((idx / n2) % n);
    const int mu = (int)((idx / n) % n);
    const int nu = (int)(idx % n);
    G[idx] = eri[idx] - eri[(((size_t)s * n + mu) * n + nu) * n + t];
  }
}

// sum_{ab} A[b][a] B[a][b] for a batch of (A, B) pointer pairs, one block each.
__global__ void trace_kernel(const double* const* __restrict__ as, const double* const* __restrict__ bs, int n,
                             double* __restrict__ out) {
  const double* A = as[blockIdx.x];
  const double* B = bs[blockIdx.x];
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
    const int a = idx / n, b = idx % n;
    acc += A[(size_t)b * n + a] * B[idx];
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// Fock records: frecx = {X0, F^(00)}, frecy = {Y0, F^(00)} from the Hamiltonian records.
__global__ void fock_records_kernel(const double2* __restrict__ recx, const double2* __restrict__ recy,
                                    const double* __restrict__ ff00, int n, double2* __restrict__ frecx,
                                    double2* __restrict__ frecy) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const double f = ff00[idx];
    frecx[idx] = make_double2(recx[idx].x, f);
    frecy[idx] = make_double2(recy[idx].x, f);
  }
}

// dst[c][r] = src[r][c] (n x n)
__global__ void transpose_kernel(const double* __restrict__ src, int n, double* __restrict__ dst) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const int r = idx / n, c = idx % n;
    dst[(size_t)c * n + r] = src[idx];
  }
}

// Fast-layout records: recx = {X0, hcol0}, recy = {Y0, hcol0}.
__global__ void records_kernel(const double* __restrict__ X0, const double* __restrict__ Y0,
                               const double* __restrict__ F, const double* __restrict__ V,
                               const double* __restrict__ Vd, int n, double2* __restrict__ recx,
                               double2* __restrict__ recy) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const double hc = F[idx] + V[idx] + Vd[idx];
    recx[idx] = make_double2(X0[idx], hc);
    recy[idx] = make_double2(Y0[idx], hc);
  }
}

// T4 layout [p][r][q][s] holds T(A,B,C,D)[p,q,r,s].
//   jas[a,b,c,d] = T4dir[c][a][d][b] - T4exc[c][d][a][b] - T4dir[c][a][b][d] + T4exc[c][b][a][d]
__global__ void jas_kernel(const double* __restrict__ td, const double* __restrict__ te, int n,
                           double* __restrict__ out) {
  const size_t n2 = (size_t)n * n, n3 = n2 * n, n4 = n2 * n2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n4; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t a = idx / n3, b = (idx / n2) % n, c = (idx / n) % n, d = idx % n;
    out[idx] = jas_at(td, te, n, a, b, c, d);
  }
}

//   J stored [a,b,c,d] = T4dir[c][a][d][b] - T4exc[c][d][a][b]   (layout.rs:367-392 order)
__global__ void jstored_kernel(const double* __restrict__ td, const double* __restrict__ te, int n,
                               double* __restrict__ out) {
  const size_t n2 = (size_t)n * n, n3 = n2 * n, n4 = n2 * n2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n4; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t a = idx / n3, b = (idx / n2) % n, c = (idx / n) % n, d = idx % n;
    out[idx] = jstored_at(td, te, n, a, b, c, d);
  }
}

//   II stored [r,c,i,j] = T4[r][i][c][j]
__global__ void ii_kernel(const double* __restrict__ t4, int n, double* __restrict__ out) {
  const size_t n2 = (size_t)n * n, n3 = n2 * n, n4 = n2 * n2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n4; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t r = idx / n3, c = (idx / n2) % n, i = (idx / n) % n, j = idx % n;
    out[idx] = ii_at(t4, n, r, c, i, j);
  }
}

// [p][q][r][s] -> [p][r][q][s]
__global__ void swap_qr_kernel(const double* __restrict__ src, int n, double* __restrict__ dst) {
  const size_t n2 = (size_t)n * n, n3 = n2 * n, n4 = n2 * n2;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n4; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t p = idx / n3, r = (idx / n2) % n, q = (idx / n) % n, s = idx % n;
    dst[idx] = src[p * n3 + q * n2 + r * n + s];
  }
}

// Cholesky-route workspace: W = L^P B (naux x n^2), a small cache of factors U = A^T L^P B keyed
// by the (A, B) pair they come from (FP64 for NW_TRANSFORM_CHOL_FP64, split pieces for the
// tcgen05 modes: a pair's J and II tensors share six distinct factors, so each is computed and
// split once), and the error word of the split products.
constexpr int kFactorCache = 6;
struct CholWork {
  double* W = nullptr;
  double* F = nullptr;                     // FP64 factor scratch before splitting
  double* fac[kFactorCache] = {};          // FP64 factors (CHOL_FP64)
  char* split[kFactorCache] = {};          // split pieces (tcgen05 modes)
  SplitFactor sf[kFactorCache] = {};
  const double* ka[kFactorCache] = {};
  const double* kb[kFactorCache] = {};
  int next = 0;
  size_t split_bytes = 0;
  uint32_t* err = nullptr;
};

nw_status chol_work(nw_ctx* ctx, int n, CholWork* w) {
  const size_t fac = (size_t)ctx->naux * n * n, fb = fac * sizeof(double);
  const bool fp64 = ctx->transform == NW_TRANSFORM_CHOL_FP64;
  const size_t split = fp64 ? 0 : (split_factor_bytes(ctx->transform, ctx->naux, n * n) + 255) / 256 * 256;
  const size_t per = fp64 ? fb : split;
  const size_t bytes = 2 * fb + kFactorCache * per + 1024;
  nw_status st = ensure(ctx, ctx->chol_work, bytes);
  if (st != NW_OK) return st;
  char* base = static_cast<char*>(ctx->chol_work.p);
  *w = CholWork{};
  w->W = reinterpret_cast<double*>(base);
  w->F = w->W + fac;
  char* q = base + 2 * fb;
  for (int i = 0; i < kFactorCache; ++i, q += per) {
    if (fp64)
      w->fac[i] = reinterpret_cast<double*>(q);
    else
      w->split[i] = q;
  }
  w->split_bytes = split;
  w->err = reinterpret_cast<uint32_t*>(q);
  NW_CUDA(ctx, cudaMemsetAsync(w->err, 0, sizeof(uint32_t)));
  return NW_OK;
}

// Index of the cached factor A^T L^P B, computed (and split) on a miss; `keep` is never evicted.
nw_status chol_factor(nw_ctx* ctx, int n, const double* A, const double* B, CholWork& w, int keep, int* out) {
  for (int i = 0; i < kFactorCache; ++i)
    if (w.ka[i] == A && w.kb[i] == B) {
      *out = i;
      return NW_OK;
    }
  int i = w.next;
  if (i == keep) i = (i + 1) % kFactorCache;
  w.next = (i + 1) % kFactorCache;
  const cudaStream_t h = 0;
  const long long n2 = (long long)n * n;
  const int naux = ctx->naux;
  const bool fp64 = ctx->transform == NW_TRANSFORM_CHOL_FP64;
  double* U = fp64 ? w.fac[i] : w.F;
  NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, ctx->d_chol, n, n2, B, n, 0, 0.0, w.W, n, n2, naux));
  NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, A, n, 0, w.W, n, n2, 0.0, U, n, n2, naux));
  if (!fp64) NW_DG(ctx, split_factor(h, ctx->transform, U, naux, (int)n2, w.split[i], w.split_bytes, &w.sf[i]));
  w.ka[i] = A;
  w.kb[i] = B;
  *out = i;
  return NW_OK;
}

// The Cholesky route of T(A,B,C,D), result in [p][r][q][s] in t4 (t1 is n^4 scratch):
// U[P] = A^T L^P B, V[P] = C^T L^P D (batched FP64 products, cached), T[pq][rs] = sum_P
// U[P][pq] V[P][rs] in FP64 (NW_TRANSFORM_CHOL_FP64) or as split products on tcgen05 (tc_gemm.cu).
nw_status transform4_chol(nw_ctx* ctx, int n, const double* A, const double* B, const double* C, const double* D,
                          double* t1, double* t4, CholWork& w) {
  const cudaStream_t h = 0;
  const long long n2 = (long long)n * n;
  int iu = -1, iv = -1;
  nw_status st = chol_factor(ctx, n, A, B, w, -1, &iu);
  if (st == NW_OK) st = chol_factor(ctx, n, C, D, w, iu, &iv);
  if (st != NW_OK) return st;
  if (ctx->transform == NW_TRANSFORM_CHOL_FP64) {
    NW_DG(ctx, gemm(h, true, false, (int)n2, (int)n2, ctx->naux, 1.0, w.fac[iu], (int)n2, w.fac[iv], (int)n2, 0.0, t1,
                    (int)n2));
    swap_qr_kernel<<<148 * 16, 256>>>(t1, n, t4);
    NW_CUDA(ctx, cudaGetLastError());
    return NW_OK;
  }
  NW_DG(ctx, split_product(h, w.sf[iu], w.sf[iv], n, t4, w.err));
  return NW_OK;
}

// Four quarter transforms T(A,B,C,D)[p,q,r,s] = sum (mu nu|lam sig) A[mu,p] B[nu,q] C[lam,r] D[sig,s],
// result in layout [p][r][q][s] in t4.  t1 is scratch of n^4 doubles (nao == nmo here).  A
// Cholesky transform mode takes the factored route instead.
nw_status transform4(nw_ctx* ctx, const double* eri, int n, const double* A, const double* B, const double* C,
                     const double* D, double* t1, double* t4, CholWork* cw = nullptr) {
  if (cw) return transform4_chol(ctx, n, A, B, C, D, t1, t4, *cw);
  const cudaStream_t h = 0;  // the build runs on the legacy default stream
  const long long n2 = (long long)n * n, n3 = n2 * n;
  // T1[p][nu lam sig] = A^T (n x n) * E (n x n^3)
  NW_DG(ctx, gemm(h, true, false, n, (int)n3, n, 1.0, A, n, eri, (int)n3, 0.0, t1, (int)n3));
  // T2[p][lam sig][q] = T1[p]^T (n^2 x n) * B (n x n)
  NW_DG(ctx, gemm_b(h, true, false, (int)n2, n, n, 1.0, t1, (int)n2, n3, B, n, 0, 0.0, t4, n, n3, n));
  // T3[p][r][sig q] = C^T (n x n) * T2[p] (n x n^2)
  NW_DG(ctx, gemm_b(h, true, false, n, (int)n2, n, 1.0, C, n, 0, t4, (int)n2, n3, 0.0, t1, (int)n2, n3, n));
  // T4[p r][q][s] = T3[pr]^T (n x n) * D (n x n)
  NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, t1, n, n2, D, n, 0, 0.0, t4, n, n2, (int)n2));
  return NW_OK;
}

inline int grid_for(size_t work, int block = 256) {
  size_t g = (work + block - 1) / block;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

cudaError_t swap_qr(cudaStream_t st, const double* src, int n, double* dst) {
  swap_qr_kernel<<<148 * 16, 256, 0, st>>>(src, n, dst);
  return cudaGetLastError();
}

nw_status build_all(nw_ctx* ctx, const std::vector<char>* subset) {
  const int n = ctx->nmo, nao = ctx->nao, nref = ctx->nref;
  const int npair = nref * nref, nps = 2 * npair;
  const int oa = ctx->nocc_a, ob = ctx->nocc_b, omax = std::max(oa, ob);
  const size_t n2 = (size_t)n * n, n4 = n2 * n2;
  if (nao != n) return fail(ctx, NW_ERR_UNSUPPORTED, "this build requires nao == nmo");
  if (subset && subset->size() != (size_t)npair) return fail(ctx, NW_ERR_INVALID, "reference-pair subset size");
  const cudaStream_t h = 0;  // the build runs on the legacy default stream
  // a rebuild replaces the slab: nothing evaluates until it has completed
  ctx->built = false;
  ctx->partial = false;
  // the ordered reference pairs whose slab pieces this build holds (all, or a block of a
  // blocked evaluation); every per-pair scalar and the Fock basis cover all pairs
  auto resident = [&](int p) { return !subset || (*subset)[p] != 0; };

  // ---------------- workspace ----------------
  const size_t per_ps = 2 * (size_t)nao * omax + omax + 2 * n2 /*M*/ + 4 * n2 /*rowc colc cxs cws*/ +
                        8 * n2 /*mts/ms products*/ + 4 * n2 /*cx xc*/ + 2 * n2 /*MS*/ + 2 * n2 /*MtS*/ +
                        4 * n2 /*X Y*/ + 2 * n2 /*tmp*/ + 2 * n2 /*JK*/ + 2 * n2 /*Jc*/ + 4 * n2 /*Fh*/ +
                        8 * n2 /*V*/ + 8 * n2 /*vab or vba*/ + 2 * n2 /*hxc*/ + 4 * n2 /*JKxc*/ +
                        4 * n2 /*JcXc*/ + 64;
  // 40 arena pieces, each rounded up to 256 bytes
  const size_t work_doubles = per_ps * nps + 5 * n4 + 40 * 32 + 4096;
  // the workspace stays with the context, so rebuilds (blocked evaluation, transform changes)
  // do not allocate it again
  Arena ar;
  {
    nw_status st = ensure(ctx, ctx->build_work, work_doubles * sizeof(double) + 256 * 64);
    if (st != NW_OK) return fail(ctx, NW_ERR_ALLOC, "build workspace allocation failed");
    ar.base = static_cast<char*>(ctx->build_work.p);
    ar.cap = ctx->build_work.bytes;
  }

  double* ctx_t = ar.take((size_t)nps * nao * omax);
  double* ctw_t = ar.take((size_t)nps * nao * omax);
  double* sv = ar.take((size_t)nps * omax);
  PairSpinMeta* meta = reinterpret_cast<PairSpinMeta*>(ar.take((size_t)nps * 4));
  double* M = ar.take((size_t)nps * 2 * n2);
  double* rowc = ar.take((size_t)nps * n2);
  double* colc = ar.take((size_t)nps * n2);
  double* cxs = ar.take((size_t)nps * n2);
  double* cws = ar.take((size_t)nps * n2);
  double* MtS = ar.take((size_t)nps * 2 * n2);
  double* MS = ar.take((size_t)nps * 2 * n2);
  double* mtsx = ar.take((size_t)nps * 2 * n2);
  double* mtsw = ar.take((size_t)nps * 2 * n2);
  double* msx = ar.take((size_t)nps * 2 * n2);
  double* msw = ar.take((size_t)nps * 2 * n2);
  double* cx = ar.take((size_t)nps * 2 * n2);
  double* xc = ar.take((size_t)nps * 2 * n2);
  double* X = ar.take((size_t)nps * 2 * n2);
  double* Y = ar.take((size_t)nps * 2 * n2);
  double* tmp = ar.take((size_t)nps * 2 * n2);
  double* JK = ar.take((size_t)nps * 2 * n2);
  double* Jc = ar.take((size_t)nps * 2 * n2);
  double* Fh = ar.take((size_t)nps * 4 * n2);
  double* Vv = ar.take((size_t)nps * 8 * n2);
  double* Vd = ar.take((size_t)nps * 8 * n2);  // vab for alpha (ps even), vba for beta (ps odd)
  double* hxc = ar.take((size_t)nps * 2 * n2);
  double* JKxc = ar.take((size_t)nps * 4 * n2);
  double* JcXc = ar.take((size_t)nps * 4 * n2);
  double* G = ar.take(n4);
  double* tA = ar.take(n4);
  double* tB = ar.take(n4);
  double* tD = ar.take(n4);
  double* tE = ar.take(n4);
  if (!tE) return fail(ctx, NW_ERR_ALLOC, "build workspace too small");
  // Cholesky route of the four-index tensors (nw_set_transform)
  CholWork cw{};
  CholWork* cwp = nullptr;
  if (ctx->transform != NW_TRANSFORM_FP64) {
    if (!ctx->d_chol) return fail(ctx, NW_ERR_STATE, "Cholesky transform without Cholesky factors");
    nw_status st = chol_work(ctx, n, &cw);
    if (st != NW_OK) return st;
    cwp = &cw;
  }

  // ---------------- pairing ----------------
  {
    const size_t smem = ((size_t)nao * omax + 3 * (size_t)omax * omax + omax) * sizeof(double);
    if (smem > 200 * 1024) return fail(ctx, NW_ERR_UNSUPPORTED, "occupied space too large for the pairing kernel");
    NW_CUDA(ctx, cudaFuncSetAttribute(pairing_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    pairing_kernel<<<nps, 128, smem>>>(ctx->d_s, ctx->d_ca, ctx->d_cb, nref, nao, n, oa, ob, ctx->tol, omax, ctx_t,
                                       ctw_t, sv, meta);
    NW_CUDA(ctx, cudaGetLastError());
  }
  m_kernel<<<dim3(grid_for(n2) > 64 ? 64 : grid_for(n2), nps), 256>>>(ctx_t, ctw_t, sv, meta, nao, omax, ctx->tol, M);
  NW_CUDA(ctx, cudaGetLastError());
  spaces_kernel<<<dim3(grid_for(n2) > 64 ? 64 : grid_for(n2), nps), 256>>>(ctx->d_ca, ctx->d_cb, nref, nao, n, oa, ob,
                                                                         rowc, colc, cxs, cws);
  NW_CUDA(ctx, cudaGetLastError());

  std::vector<PairSpinMeta> hmeta(nps);
  NW_CUDA(ctx, cudaMemcpy(hmeta.data(), meta, sizeof(PairSpinMeta) * nps, cudaMemcpyDeviceToHost));

  // ---------------- dense products ----------------
  const int B2 = nps * 2;  // (ps, m)
  // MtS = M^T S, MS = M S
  NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, M, n, n2, ctx->d_s, n, 0, 0.0, MtS, n, n2, B2));
  NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, M, n, n2, ctx->d_s, n, 0, 0.0, MS, n, n2, B2));
  // products with the per-ps C copies, one call per m
  for (int m = 0; m < 2; ++m) {
    const size_t off = (size_t)m * n2;
    NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, MtS + off, n, 2 * n2, cxs, n, n2, 0.0, mtsx + off, n, 2 * n2, nps));
    NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, MtS + off, n, 2 * n2, cws, n, n2, 0.0, mtsw + off, n, 2 * n2, nps));
    NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, MS + off, n, 2 * n2, cxs, n, n2, 0.0, msx + off, n, 2 * n2, nps));
    NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, MS + off, n, 2 * n2, cws, n, n2, 0.0, msw + off, n, 2 * n2, nps));
  }
  cxxc_kernel<<<dim3(grid_for(n2) > 64 ? 64 : grid_for(n2), B2), 256>>>(mtsx, mtsw, msx, msw, cxs, cws, nao, n, oa, ob,
                                                                      cx, xc);
  NW_CUDA(ctx, cudaGetLastError());
  // X^(m) = rowc^T (S M S) colc: tmp = MS * S; X = rowc^T tmp colc
  NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, ctx->d_s, n, 0, MS, n, n2, 0.0, tmp, n, n2, B2));  // S M S
  for (int m = 0; m < 2; ++m) {
    const size_t off = (size_t)m * n2;
    NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, rowc, n, n2, tmp + off, n, 2 * n2, 0.0, MS + off, n, 2 * n2, nps));
    NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, MS + off, n, 2 * n2, colc, n, n2, 0.0, X + off, n, 2 * n2, nps));
  }
  // Y^(0) = X^(0) - rowc^T S colc, Y^(1) = X^(1): tmp(ps,0) = rowc^T S, tmp(ps,1) = tmp(ps,0) colc
  NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, rowc, n, n2, ctx->d_s, n, 0, 0.0, tmp, n, 2 * n2, nps));
  NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, tmp, n, 2 * n2, colc, n, n2, 0.0, tmp + n2, n, 2 * n2, nps));
  NW_CUDA(ctx, cudaMemcpyAsync(Y, X, sizeof(double) * nps * 2 * n2, cudaMemcpyDeviceToDevice));
  // Y(ps,0) -= tmp(ps,1)
  axpy_batched_kernel<<<dim3(grid_for(n2) > 64 ? 64 : grid_for(n2), nps), 256>>>(-1.0, tmp + n2, 2 * (long long)n2, Y,
                                                                              2 * (long long)n2, (long long)n2);
  NW_CUDA(ctx, cudaGetLastError());
  // JK and Coulomb-only J for all (ps, m): rows of M are vec(M)
  g_kernel<<<grid_for(n4), 256>>>(ctx->d_eri, n, G);
  NW_CUDA(ctx, cudaGetLastError());
  NW_DG(ctx, gemm(h, false, true, B2, (int)n2, (int)n2, 1.0, M, (int)n2, G, (int)n2, 0.0, JK, (int)n2));
  NW_DG(ctx, gemm(h, false, true, B2, (int)n2, (int)n2, 1.0, M, (int)n2, ctx->d_eri, (int)n2, 0.0, Jc, (int)n2));
  // hxc[ps][mj] = h xc[mj]; Fh[ps][mi][mj] = cx[mi]^T hxc[mj]
  NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, ctx->d_h, n, 0, xc, n, n2, 0.0, hxc, n, n2, B2));
  for (int mi = 0; mi < 2; ++mi)
    for (int mj = 0; mj < 2; ++mj)
      NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, cx + mi * n2, n, 2 * n2, hxc + mj * n2, n, 2 * n2, 0.0,
                          Fh + (size_t)(mi * 2 + mj) * n2, n, 4 * n2, nps));
  // JKxc[ps][mk][mj] = JK[mk] xc[mj]; V[ps][mi][mj][mk] = cx[mi]^T JKxc[mk][mj]
  for (int mk = 0; mk < 2; ++mk)
    for (int mj = 0; mj < 2; ++mj)
      NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, JK + mk * n2, n, 2 * n2, xc + mj * n2, n, 2 * n2, 0.0,
                          JKxc + (size_t)(mk * 2 + mj) * n2, n, 4 * n2, nps));
  for (int mi = 0; mi < 2; ++mi)
    for (int mj = 0; mj < 2; ++mj)
      for (int mk = 0; mk < 2; ++mk)
        NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, cx + mi * n2, n, 2 * n2, JKxc + (size_t)(mk * 2 + mj) * n2, n,
                            4 * n2, 0.0, Vv + (size_t)((mi * 2 + mj) * 2 + mk) * n2, n, 8 * n2, nps));
  // Different-spin: for alpha (ps = 2p) vab[ma0][mb0][mak] = cx_a[ma0]^T Jc_b[mb0] xc_a[mak];
  // for beta (ps = 2p+1) vba[mb0][ma0][mbk] = cx_b[mb0]^T Jc_a[ma0] xc_b[mbk].
  // JcXc[ps][mo][mk] = Jc_other[mo] xc_this[mk]
  for (int mo = 0; mo < 2; ++mo)
    for (int mk = 0; mk < 2; ++mk) {
      // alpha rows: other = beta (ps+1)
      NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, Jc + 2 * n2 + mo * n2, n, 4 * n2, xc + mk * n2, n, 4 * n2, 0.0,
                          JcXc + (size_t)(mo * 2 + mk) * n2, n, 8 * n2, npair));
      // beta rows: other = alpha (ps-1)
      NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, Jc + mo * n2, n, 4 * n2, xc + 2 * n2 + mk * n2, n, 4 * n2, 0.0,
                          JcXc + 4 * n2 + (size_t)(mo * 2 + mk) * n2, n, 8 * n2, npair));
    }
  for (int mt = 0; mt < 2; ++mt)
    for (int mo = 0; mo < 2; ++mo)
      for (int mk = 0; mk < 2; ++mk)
        NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, cx + mt * n2, n, 2 * n2, JcXc + (size_t)(mo * 2 + mk) * n2, n,
                            4 * n2, 0.0, Vd + (size_t)((mt * 2 + mo) * 2 + mk) * n2, n, 8 * n2, nps));

  // ---------------- scalars ----------------
  // per ps: f0h[2] = tr(M[m] h), v0 terms tr(JK0 M0), tr(JK0 M1), tr(JK1 M1);
  // per pair: vab0[i][j] = tr(Jc_a[i] M_b[j]), vba0[j][i] = tr(Jc_b[j] M_a[i]).
  const int nsc_ps = 5, nsc_p = 8;
  const int ntr = nps * nsc_ps + npair * nsc_p;
  std::vector<const double*> ha(ntr), hb(ntr);
  for (int ps = 0; ps < nps; ++ps) {
    const double* Mp = M + (size_t)ps * 2 * n2;
    const double* JKp = JK + (size_t)ps * 2 * n2;
    ha[ps * 5 + 0] = Mp;
    hb[ps * 5 + 0] = ctx->d_h;
    ha[ps * 5 + 1] = Mp + n2;
    hb[ps * 5 + 1] = ctx->d_h;
    ha[ps * 5 + 2] = JKp;
    hb[ps * 5 + 2] = Mp;
    ha[ps * 5 + 3] = JKp;
    hb[ps * 5 + 3] = Mp + n2;
    ha[ps * 5 + 4] = JKp + n2;
    hb[ps * 5 + 4] = Mp + n2;
  }
  for (int p = 0; p < npair; ++p) {
    const int base = nps * 5 + p * 8;
    const double* Ma = M + (size_t)(2 * p) * 2 * n2;
    const double* Mb = M + (size_t)(2 * p + 1) * 2 * n2;
    const double* Ja = Jc + (size_t)(2 * p) * 2 * n2;
    const double* Jb = Jc + (size_t)(2 * p + 1) * 2 * n2;
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        ha[base + i * 2 + j] = Ja + i * n2;  // vab0[i][j]
        hb[base + i * 2 + j] = Mb + j * n2;
        ha[base + 4 + j * 2 + i] = Jb + j * n2;  // vba0[j][i]
        hb[base + 4 + j * 2 + i] = Ma + i * n2;
      }
  }
  std::vector<double> traces(ntr);
  {
    const double** dptr = nullptr;
    double* dtr = nullptr;
    NW_CUDA(ctx, cudaMalloc(&dptr, sizeof(double*) * 2 * ntr));
    NW_CUDA(ctx, cudaMalloc(&dtr, sizeof(double) * ntr));
    NW_CUDA(ctx, cudaMemcpy(dptr, ha.data(), sizeof(double*) * ntr, cudaMemcpyHostToDevice));
    NW_CUDA(ctx, cudaMemcpy(dptr + ntr, hb.data(), sizeof(double*) * ntr, cudaMemcpyHostToDevice));
    trace_kernel<<<ntr, 256>>>(dptr, dptr + ntr, n, dtr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(traces.data(), dtr, sizeof(double) * ntr, cudaMemcpyDeviceToHost);
    cudaFree(dptr);
    cudaFree(dtr);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace kernel");
  }

  // ---------------- slab layout ----------------
  ctx->m_counts.assign(2 * npair, 0);
  std::vector<char> generic(npair, 0);
  for (int p = 0; p < npair; ++p) {
    ctx->m_counts[2 * p] = hmeta[2 * p].m;
    ctx->m_counts[2 * p + 1] = hmeta[2 * p + 1].m;
    generic[p] = (hmeta[2 * p].m + hmeta[2 * p + 1].m) > 0;
  }
  size_t slab = 0;
  auto reserve = [&](size_t ndouble) {
    const size_t off = slab;
    slab += ((ndouble + 31) / 32) * 32;  // 256-byte aligned pieces
    return off;
  };
  struct GenOff {
    size_t x[2][2], y[2][2], fh[2][4], v[2][8], j[2][10], vab[8], vba[8], ii[16];
  };
  struct FastOff {
    size_t recx[2], recy[2], jas[2], ii0;
  };
  std::vector<FastOff> fo(npair);
  std::vector<GenOff> go(npair);
  for (int p = 0; p < npair; ++p) {
    if (!resident(p)) continue;
    if (!generic[p]) {
      for (int s = 0; s < 2; ++s) {
        fo[p].recx[s] = reserve(2 * n2);
        fo[p].recy[s] = reserve(2 * n2);
        fo[p].jas[s] = reserve(n4);
      }
      fo[p].ii0 = reserve(n4);
    } else {
      GenOff& g = go[p];
      for (int s = 0; s < 2; ++s) {
        const int ms = hmeta[2 * p + s].m;
        for (int m = 0; m < 2; ++m) {
          g.x[s][m] = reserve(n2);
          g.y[s][m] = reserve(n2);
        }
        for (int k = 0; k < 4; ++k) g.fh[s][k] = reserve(n2);
        for (int k = 0; k < 8; ++k) g.v[s][k] = reserve(n2);
        static const int br[10][4] = {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {0, 1, 0, 1},
                                      {0, 1, 1, 0}, {0, 1, 1, 1}, {1, 0, 1, 0}, {1, 0, 1, 1}, {1, 1, 1, 1}};
        for (int sl = 0; sl < 10; ++sl)
          g.j[s][sl] = (br[sl][0] + br[sl][1] + br[sl][2] + br[sl][3] <= ms) ? reserve(n4) : (size_t)-1;
      }
      for (int k = 0; k < 8; ++k) {
        g.vab[k] = reserve(n2);
        g.vba[k] = reserve(n2);
      }
      const int ma = hmeta[2 * p].m, mb = hmeta[2 * p + 1].m;
      for (int k = 0; k < 16; ++k) {
        const int a0 = (k >> 3) & 1, az = (k >> 2) & 1, b0 = (k >> 1) & 1, by = k & 1;
        g.ii[k] = (a0 + az <= ma && b0 + by <= mb) ? reserve(n4) : (size_t)-1;
      }
    }
  }
  // a slab at least as large is reused (rebuilds, the blocks of a blocked evaluation)
  const size_t slab_need = std::max<size_t>(slab, 32) * sizeof(double);
  if (ctx->d_slab && ctx->slab_capacity < slab_need) {
    cudaFree(ctx->d_slab);
    ctx->d_slab = nullptr;
    ctx->slab_capacity = 0;
  }
  {
    if (!ctx->d_slab) {
      cudaError_t e = cudaMalloc(&ctx->d_slab, slab_need);
      if (e != cudaSuccess) {
        ctx->d_slab = nullptr;
        return fail(ctx, NW_ERR_ALLOC, "intermediate slab allocation failed (" +
                                           std::to_string(slab * 8 / (1 << 20)) + " MiB)");
      }
      ctx->slab_capacity = slab_need;
    }
    ctx->slab_bytes = slab * sizeof(double);
  }
  double* S0 = ctx->d_slab;

  // ---------------- fill ----------------
  const int g4 = grid_for(n4), g2 = grid_for(n2);
  std::vector<FastPair> hfast(npair);
  std::vector<GenPair> hgen(npair);
  std::memset(hfast.data(), 0, sizeof(FastPair) * npair);
  std::memset(hgen.data(), 0, sizeof(GenPair) * npair);
  for (int p = 0; p < npair; ++p) {
    if (!resident(p)) continue;
    const int psa = 2 * p, psb = 2 * p + 1;
    auto CX = [&](int ps, int m) { return cx + ((size_t)ps * 2 + m) * n2; };
    auto XC = [&](int ps, int m) { return xc + ((size_t)ps * 2 + m) * n2; };
    const double* tr_a = &traces[psa * 5];
    const double* tr_b = &traces[psb * 5];
    const double* tr_p = &traces[nps * 5 + p * 8];
    const double pref_a = hmeta[psa].phase * hmeta[psa].tsp;
    const double pref_b = hmeta[psb].phase * hmeta[psb].tsp;
    if (!generic[p]) {
      FastPair& fp = hfast[p];
      for (int s = 0; s < 2; ++s) {
        const int ps = 2 * p + s;
        double2* recx = reinterpret_cast<double2*>(S0 + fo[p].recx[s]);
        double2* recy = reinterpret_cast<double2*>(S0 + fo[p].recy[s]);
        records_kernel<<<g2, 256>>>(X + (size_t)ps * 2 * n2, Y + (size_t)ps * 2 * n2, Fh + (size_t)ps * 4 * n2,
                                    Vv + (size_t)ps * 8 * n2, Vd + (size_t)ps * 8 * n2, n, recx, recy);
        NW_CUDA(ctx, cudaGetLastError());
        {
          nw_status st = transform4(ctx, ctx->d_eri, n, CX(ps, 0), XC(ps, 0), CX(ps, 0), XC(ps, 0), tA, tD, cwp);
          if (st != NW_OK) return st;
          st = transform4(ctx, ctx->d_eri, n, CX(ps, 0), CX(ps, 0), XC(ps, 0), XC(ps, 0), tA, tE, cwp);
          if (st != NW_OK) return st;
        }
        jas_kernel<<<g4, 256>>>(tD, tE, n, S0 + fo[p].jas[s]);
        NW_CUDA(ctx, cudaGetLastError());
        FastSpin& fs = s ? fp.b : fp.a;
        fs.recx = recx;
        fs.recy = recy;
        fs.jas = S0 + fo[p].jas[s];
        const double* tr = s ? tr_b : tr_a;
        fs.pref = s ? pref_b : pref_a;
        fs.g0 = tr[0] + 0.5 * tr[2];
      }
      {
        nw_status st = transform4(ctx, ctx->d_eri, n, CX(psa, 0), XC(psa, 0), CX(psb, 0), XC(psb, 0), tA, tD, cwp);
        if (st != NW_OK) return st;
      }
      ii_kernel<<<g4, 256>>>(tD, n, S0 + fo[p].ii0);
      NW_CUDA(ctx, cudaGetLastError());
      fp.ii0 = S0 + fo[p].ii0;
      fp.vab0 = tr_p[0];
    } else {
      GenPair& gp = hgen[p];
      const GenOff& g = go[p];
      for (int s = 0; s < 2; ++s) {
        const int ps = 2 * p + s;
        const int ms = hmeta[ps].m;
        GenSpin& gs = s ? gp.b : gp.a;
        for (int m = 0; m < 2; ++m) {
          NW_CUDA(ctx, cudaMemcpyAsync(S0 + g.x[s][m], X + ((size_t)ps * 2 + m) * n2, n2 * 8, cudaMemcpyDeviceToDevice));
          NW_CUDA(ctx, cudaMemcpyAsync(S0 + g.y[s][m], Y + ((size_t)ps * 2 + m) * n2, n2 * 8, cudaMemcpyDeviceToDevice));
          gs.x[m] = S0 + g.x[s][m];
          gs.y[m] = S0 + g.y[s][m];
        }
        for (int k = 0; k < 4; ++k) {
          transpose_kernel<<<g2, 256>>>(Fh + ((size_t)ps * 4 + k) * n2, n, S0 + g.fh[s][k]);
          gs.fh_t[k >> 1][k & 1] = S0 + g.fh[s][k];
        }
        for (int k = 0; k < 8; ++k) {
          transpose_kernel<<<g2, 256>>>(Vv + ((size_t)ps * 8 + k) * n2, n, S0 + g.v[s][k]);
          gs.v_t[k >> 2][(k >> 1) & 1][k & 1] = S0 + g.v[s][k];
        }
        NW_CUDA(ctx, cudaGetLastError());
        static const int br[10][4] = {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {0, 1, 0, 1},
                                      {0, 1, 1, 0}, {0, 1, 1, 1}, {1, 0, 1, 0}, {1, 0, 1, 1}, {1, 1, 1, 1}};
        for (int sl = 0; sl < 10; ++sl) {
          if (g.j[s][sl] == (size_t)-1) {
            gs.j[sl] = nullptr;
            continue;
          }
          const int a = br[sl][0], b = br[sl][1], c = br[sl][2], d = br[sl][3];
          nw_status st = transform4(ctx, ctx->d_eri, n, CX(ps, a), XC(ps, b), CX(ps, c), XC(ps, d), tA, tD, cwp);
          if (st != NW_OK) return st;
          st = transform4(ctx, ctx->d_eri, n, CX(ps, a), CX(ps, c), XC(ps, b), XC(ps, d), tA, tE, cwp);
          if (st != NW_OK) return st;
          jstored_kernel<<<g4, 256>>>(tD, tE, n, S0 + g.j[s][sl]);
          NW_CUDA(ctx, cudaGetLastError());
          gs.j[sl] = S0 + g.j[s][sl];
        }
        const double* tr = s ? tr_b : tr_a;
        gs.pref = s ? pref_b : pref_a;
        gs.f0h[0] = tr[0];
        gs.f0h[1] = tr[1];
        gs.v0[0] = tr[2];
        gs.v0[1] = ms >= 1 ? 2.0 * tr[3] : 0.0;
        gs.v0[2] = ms >= 2 ? tr[4] : 0.0;
        gs.m = ms;
      }
      for (int k = 0; k < 8; ++k) {
        transpose_kernel<<<g2, 256>>>(Vd + ((size_t)psa * 8 + k) * n2, n, S0 + g.vab[k]);
        transpose_kernel<<<g2, 256>>>(Vd + ((size_t)psb * 8 + k) * n2, n, S0 + g.vba[k]);
        gp.vab_t[k >> 2][(k >> 1) & 1][k & 1] = S0 + g.vab[k];
        gp.vba_t[k >> 2][(k >> 1) & 1][k & 1] = S0 + g.vba[k];
      }
      NW_CUDA(ctx, cudaGetLastError());
      for (int k = 0; k < 16; ++k) {
        const int a0 = (k >> 3) & 1, az = (k >> 2) & 1, b0 = (k >> 1) & 1, by = k & 1;
        if (g.ii[k] == (size_t)-1) {
          gp.ii[a0][az][b0][by] = nullptr;
          continue;
        }
        nw_status st = transform4(ctx, ctx->d_eri, n, CX(psa, a0), XC(psa, az), CX(psb, b0), XC(psb, by), tA, tD, cwp);
        if (st != NW_OK) return st;
        ii_kernel<<<g4, 256>>>(tD, n, S0 + g.ii[k]);
        NW_CUDA(ctx, cudaGetLastError());
        gp.ii[a0][az][b0][by] = S0 + g.ii[k];
      }
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
          gp.vab0[i][j] = tr_p[i * 2 + j];
          gp.vba0[j][i] = tr_p[4 + j * 2 + i];
        }
    }
  }

  // ---------------- tables ----------------
  // sort positions: the resident m = 0 pairs, then the resident others; -1 marks a pair whose
  // slab pieces this build does not hold (its pairs are skipped by the evaluators)
  ctx->order_host.assign(npair, -1);
  int pos = 0;
  for (int p = 0; p < npair; ++p)
    if (resident(p) && !generic[p]) ctx->order_host[p] = pos++;
  ctx->nfast = pos;
  for (int p = 0; p < npair; ++p)
    if (resident(p) && generic[p]) ctx->order_host[p] = pos++;
  ctx->nresident = pos;
  if (!ctx->d_fast) NW_CUDA(ctx, cudaMalloc(&ctx->d_fast, sizeof(FastPair) * npair));
  if (!ctx->d_gen) NW_CUDA(ctx, cudaMalloc(&ctx->d_gen, sizeof(GenPair) * npair));
  if (!ctx->d_order) NW_CUDA(ctx, cudaMalloc(&ctx->d_order, sizeof(int32_t) * npair));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_fast, hfast.data(), sizeof(FastPair) * npair, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_gen, hgen.data(), sizeof(GenPair) * npair, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_order, ctx->order_host.data(), sizeof(int32_t) * npair, cudaMemcpyHostToDevice));

  // ---------------- kept for the Fock path ----------------
  // per (pair, spin): [M^(0), M^(1), cx^(0), cx^(1), xc^(0), xc^(1)]
  ctx->fock_ready = false;
  if (ctx->d_fbase) {
    cudaFree(ctx->d_fbase);
    ctx->d_fbase = nullptr;
  }
  if (cudaMalloc(&ctx->d_fbase, sizeof(double) * nps * 6 * n2) != cudaSuccess)
    return fail(ctx, NW_ERR_ALLOC, "Fock basis allocation failed");
  const double* kept[3] = {M, cx, xc};
  for (int k = 0; k < 3; ++k)
    NW_CUDA(ctx, cudaMemcpy2D(ctx->d_fbase + 2 * k * n2, 6 * n2 * sizeof(double), kept[k], 2 * n2 * sizeof(double),
                              2 * n2 * sizeof(double), nps, cudaMemcpyDeviceToDevice));
  ctx->fast_host = hfast;
  ctx->gen_host = hgen;
  ctx->generic_host = generic;
  NW_CUDA(ctx, cudaDeviceSynchronize());
  if (cwp) {
    uint32_t err = 0;
    NW_CUDA(ctx, cudaMemcpy(&err, cw.err, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (err) return fail(ctx, NW_ERR_CUDA, "tcgen05 split product gave up waiting (flags " + std::to_string(err) + ")");
  }
  ctx->built = true;
  ctx->partial = pos < npair;
  return NW_OK;
}

// Slab doubles of one ordered reference pair under the layout of build_all (the same rounding
// of every piece to 256 bytes): the fast layout, or the reference-ordered one with the J and II
// slots its zero-overlap counts (m_alpha, m_beta) need.
size_t pair_slab_doubles(int n, int ma, int mb) {
  const size_t n2 = (size_t)n * n, n4 = n2 * n2;
  auto r = [](size_t d) { return ((d + 31) / 32) * 32; };
  if (ma + mb == 0) return 2 * (2 * r(2 * n2) + r(n4)) + r(n4);
  static const int br[10][4] = {{0, 0, 0, 0}, {0, 0, 0, 1}, {0, 0, 1, 0}, {0, 0, 1, 1}, {0, 1, 0, 1},
                                {0, 1, 1, 0}, {0, 1, 1, 1}, {1, 0, 1, 0}, {1, 0, 1, 1}, {1, 1, 1, 1}};
  size_t t = 0;
  for (int ms : {ma, mb}) {
    t += 4 * r(n2) + 4 * r(n2) + 8 * r(n2);
    for (int sl = 0; sl < 10; ++sl) t += (br[sl][0] + br[sl][1] + br[sl][2] + br[sl][3] <= ms) ? r(n4) : 0;
  }
  t += 16 * r(n2);
  for (int k = 0; k < 16; ++k) {
    const int a0 = (k >> 3) & 1, az = (k >> 2) & 1, b0 = (k >> 1) & 1, by = k & 1;
    t += (a0 + az <= ma && b0 + by <= mb) ? r(n4) : 0;
  }
  return t;
}

// Fock tables for the F + S path (update_wicks_fock, src/noci/wicks.rs:290-330, with
// construct_f_scalar, build.rs:564-617): per (pair, spin) F^(mi,mj) = cx^(mi)^T F xc^(mj) and
// F_0^(m) = tr(M^(m) F) from the M, cx, xc kept by the build (the same Loewdin pairing and
// null gauge as the Hamiltonian intermediates).
nw_status update_fock(nw_ctx* ctx, const double* fa, const double* fb) {
  if (!ctx->built || !ctx->d_fbase) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  const int n = ctx->nmo, nref = ctx->nref, npair = nref * nref, nps = 2 * npair;
  const size_t n2 = (size_t)n * n;
  const cudaStream_t h = 0;  // the build runs on the legacy default stream
  ctx->fock_ready = false;
  if (!ctx->d_fock && cudaMalloc(&ctx->d_fock, sizeof(double) * 2 * n2) != cudaSuccess)
    return fail(ctx, NW_ERR_ALLOC, "Fock matrix allocation failed");
  NW_CUDA(ctx, cudaMemcpy(ctx->d_fock, fa, sizeof(double) * n2, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(ctx->d_fock + n2, fb, sizeof(double) * n2, cudaMemcpyHostToDevice));
  double* work = nullptr;
  if (cudaMalloc(&work, sizeof(double) * nps * 6 * n2) != cudaSuccess)
    return fail(ctx, NW_ERR_ALLOC, "Fock workspace allocation failed");
  struct Free {
    void* p;
    ~Free() { cudaFree(p); }
  } free_work{work};
  double* Fxc = work;                 // [ps][mj]
  double* ff = work + nps * 2 * n2;   // [ps][mi][mj]
  const double* fbase = ctx->d_fbase;
  // Fxc[2p+s][mj] = F_s xc[2p+s][mj]
  for (int s = 0; s < 2; ++s)
    for (int mj = 0; mj < 2; ++mj)
      NW_DG(ctx, gemm_b(h, false, false, n, n, n, 1.0, ctx->d_fock + s * n2, n, 0, fbase + s * 6 * n2 + (4 + mj) * n2,
                          n, 12 * n2, 0.0, Fxc + (size_t)(s * 2 + mj) * n2, n, 4 * n2, npair));
  // ff[ps][mi][mj] = cx[ps][mi]^T Fxc[ps][mj]
  for (int mi = 0; mi < 2; ++mi)
    for (int mj = 0; mj < 2; ++mj)
      NW_DG(ctx, gemm_b(h, true, false, n, n, n, 1.0, fbase + (2 + mi) * n2, n, 6 * n2, Fxc + mj * n2, n, 2 * n2, 0.0,
                          ff + (size_t)(mi * 2 + mj) * n2, n, 4 * n2, nps));
  // f0f[ps][m] = tr(M[ps][m] F_s)
  const int ntr = 2 * nps;
  std::vector<const double*> ha(ntr), hb(ntr);
  for (int ps = 0; ps < nps; ++ps)
    for (int m = 0; m < 2; ++m) {
      ha[ps * 2 + m] = fbase + (size_t)ps * 6 * n2 + m * n2;
      hb[ps * 2 + m] = ctx->d_fock + (ps & 1) * n2;
    }
  std::vector<double> f0f(ntr);
  {
    const double** dptr = nullptr;
    double* dtr = nullptr;
    NW_CUDA(ctx, cudaMalloc(&dptr, sizeof(double*) * 2 * ntr));
    NW_CUDA(ctx, cudaMalloc(&dtr, sizeof(double) * ntr));
    cudaError_t e = cudaMemcpy(dptr, ha.data(), sizeof(double*) * ntr, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dptr + ntr, hb.data(), sizeof(double*) * ntr, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      trace_kernel<<<ntr, 256>>>(dptr, dptr + ntr, n, dtr);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(f0f.data(), dtr, sizeof(double) * ntr, cudaMemcpyDeviceToHost);
    cudaFree(dptr);
    cudaFree(dtr);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "Fock trace kernel");
  }
  // slab: fast pairs {X0|Y0, F^(00)} records per spin, other pairs F^(mi,mj) transposed
  size_t slab = 0;
  std::vector<size_t> off(npair);
  for (int p = 0; p < npair; ++p) {
    off[p] = slab;
    slab += 8 * n2;  // per spin: two records of 2 n^2 doubles (fast) or four n^2 matrices (other)
  }
  if (ctx->d_fslab) {
    cudaFree(ctx->d_fslab);
    ctx->d_fslab = nullptr;
  }
  if (cudaMalloc(&ctx->d_fslab, sizeof(double) * std::max<size_t>(slab, 32)) != cudaSuccess)
    return fail(ctx, NW_ERR_ALLOC, "Fock table allocation failed");
  std::vector<FockPair> hfock(npair);
  std::memset(hfock.data(), 0, sizeof(FockPair) * npair);
  const int g2 = grid_for(n2);
  for (int p = 0; p < npair; ++p) {
    for (int s = 0; s < 2; ++s) {
      const int ps = 2 * p + s;
      FockSpinTab& t = s ? hfock[p].b : hfock[p].a;
      double* base = ctx->d_fslab + off[p] + (size_t)s * 4 * n2;
      const double* ffps = ff + (size_t)ps * 4 * n2;
      if (!ctx->generic_host[p]) {
        const FastSpin& fs = s ? ctx->fast_host[p].b : ctx->fast_host[p].a;
        double2* frecx = reinterpret_cast<double2*>(base);
        double2* frecy = reinterpret_cast<double2*>(base + 2 * n2);
        fock_records_kernel<<<g2, 256>>>(fs.recx, fs.recy, ffps, n, frecx, frecy);
        t.recx = frecx;
        t.recy = frecy;
      } else {
        for (int k = 0; k < 4; ++k) {
          transpose_kernel<<<g2, 256>>>(ffps + k * n2, n, base + k * n2);
          t.ff_t[k >> 1][k & 1] = base + k * n2;
        }
      }
      NW_CUDA(ctx, cudaGetLastError());
      t.f0f[0] = f0f[ps * 2];
      t.f0f[1] = f0f[ps * 2 + 1];
    }
  }
  if (!ctx->d_fockp && cudaMalloc(&ctx->d_fockp, sizeof(FockPair) * npair) != cudaSuccess)
    return fail(ctx, NW_ERR_ALLOC, "Fock table allocation failed");
  NW_CUDA(ctx, cudaMemcpy(ctx->d_fockp, hfock.data(), sizeof(FockPair) * npair, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaDeviceSynchronize());
  ctx->fock_ready = true;
  return NW_OK;
}

}  // namespace nw
