// Dense NOCI matrices over the resident basis and the generalised eigenproblem, on the GPU.
//
//   build_matrix  : (H, S) or (F, S) for every pair of a left x right block of determinants
//                   (upper triangle mirrored when symmetric), as calculate_matrix_elements +
//                   scatter_matrix_elements do (src/noci/matrix.rs:39-110) for build_noci_hs /
//                   build_noci_fock.  Pairs are generated on the device row block by row block
//                   and evaluated by the sorted pair pipeline of eval.cu.
//   general_evp   : H C = S C e by Loewdin orthogonalisation on the positive subspace of S,
//                   FP64 (src/maths/linalg.rs:180-256, positive_subspace / loewdin_x /
//                   general_evp), with cuSOLVER's symmetric eigensolver and cuBLAS products.
#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "internal.cuh"

namespace nw {
namespace {

// Pairs (left[r0 + i], right[j]) of rows [r0, r0 + nrow), j >= r0 + i when symmetric; row i of
// the block starts at row_off[i] in the pair list.
__global__ void matrix_pairs_kernel(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                                    uint64_t r0, uint64_t nr, int symmetric, const uint64_t* __restrict__ row_off,
                                    uint2* __restrict__ pairs) {
  const uint64_t i = r0 + blockIdx.x;
  const uint64_t j0 = symmetric ? i : 0;
  const uint64_t base = row_off[blockIdx.x];
  const uint32_t a = left[i];
  for (uint64_t j = j0 + threadIdx.x; j < nr; j += blockDim.x) pairs[base + (j - j0)] = make_uint2(a, right[j]);
}

// Scatter the evaluated (A, S) of the block into the dense nl x nr matrices; mirrored when
// symmetric (real symmetric matrices: the mirror is the value itself).
__global__ void matrix_scatter_kernel(const double2* __restrict__ vals, uint64_t r0, uint64_t nr, int symmetric,
                                      const uint64_t* __restrict__ row_off, double* __restrict__ a,
                                      double* __restrict__ s) {
  const uint64_t i = r0 + blockIdx.x;
  const uint64_t j0 = symmetric ? i : 0;
  const uint64_t base = row_off[blockIdx.x];
  for (uint64_t j = j0 + threadIdx.x; j < nr; j += blockDim.x) {
    const double2 v = vals[base + (j - j0)];
    a[i * nr + j] = v.x;
    s[i * nr + j] = v.y;
    if (symmetric && j != i) {
      a[j * nr + i] = v.x;
      s[j * nr + i] = v.y;
    }
  }
}

// x[:, c] *= 1 / sqrt(lam[c]) for a column-major n x k block.
__global__ void scale_columns_kernel(double* __restrict__ x, const double* __restrict__ lam, int n, int k) {
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < (int64_t)n * k;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(idx / n);
    x[idx] *= 1.0 / sqrt(lam[c]);
  }
}

struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

nw_status dev_alloc(nw_ctx* ctx, DevMem& m, size_t bytes, const char* what) {
  if (cudaMalloc(&m.p, std::max<size_t>(bytes, 256)) != cudaSuccess) {
    m.p = nullptr;
    return fail(ctx, NW_ERR_ALLOC, std::string(what) + ": device allocation failed");
  }
  return NW_OK;
}

#define NW_SOLVER(ctx, call)                                                                 \
  do {                                                                                       \
    const cusolverStatus_t s_ = (call);                                                      \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                                       \
      return fail(ctx, NW_ERR_CUDA, std::string(#call) + " failed: status " + std::to_string((int)s_)); \
  } while (0)

// Symmetric eigen-decomposition in place (column-major a, n x n, triangle `uplo`): eigenvalues
// ascending into lam, eigenvectors as the columns of a.
nw_status syevd(nw_ctx* ctx, cublasFillMode_t uplo, int n, double* a, double* lam) {
  int lwork = 0;
  NW_SOLVER(ctx, cusolverDnDsyevd_bufferSize(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, uplo, n, a, n, lam, &lwork));
  DevMem work, info;
  nw_status st = dev_alloc(ctx, work, sizeof(double) * (size_t)std::max(lwork, 1), "eigensolver workspace");
  if (st != NW_OK) return st;
  if ((st = dev_alloc(ctx, info, sizeof(int), "eigensolver status")) != NW_OK) return st;
  NW_SOLVER(ctx, cusolverDnDsyevd(ctx->solver, CUSOLVER_EIG_MODE_VECTOR, uplo, n, a, n, lam, work.as<double>(), lwork,
                                  info.as<int>()));
  int hinfo = 0;
  NW_CUDA(ctx, cudaMemcpy(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (hinfo != 0) return fail(ctx, NW_ERR_CUDA, "symmetric eigensolver did not converge (info " + std::to_string(hinfo) + ")");
  return NW_OK;
}

}  // namespace

nw_status build_matrix(nw_ctx* ctx, EvalMode mode, const uint32_t* left, uint64_t nl, const uint32_t* right,
                       uint64_t nr, bool symmetric, double* a_host, double* s_host) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (!ctx->d_dets) return fail(ctx, NW_ERR_STATE, "no determinant basis set");
  if (symmetric && nl != nr) return fail(ctx, NW_ERR_INVALID, "a symmetric block needs as many rows as columns");
  for (uint64_t i = 0; i < nl; ++i)
    if (left[i] >= ctx->ndet) return fail(ctx, NW_ERR_INVALID, "left determinant index out of range");
  for (uint64_t j = 0; j < nr; ++j)
    if (right[j] >= ctx->ndet) return fail(ctx, NW_ERR_INVALID, "right determinant index out of range");
  if (nl == 0 || nr == 0) return NW_OK;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t nmat = (size_t)nl * nr;
  DevMem dl, dr, da, ds, dpairs, dvals, doff;
  nw_status st;
  if ((st = dev_alloc(ctx, dl, nl * 4, "left indices")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dr, nr * 4, "right indices")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, da, nmat * 8, "matrix")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, ds, nmat * 8, "overlap matrix")) != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpy(dl.p, left, nl * 4, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(dr.p, right, nr * 4, cudaMemcpyHostToDevice));
  // row blocks of at most kChunk pairs (one row may exceed it: it is then a block of its own)
  constexpr uint64_t kChunk = 1ull << 24;
  const uint64_t max_row = nr;
  const uint64_t cap = std::max(kChunk, max_row);
  if ((st = dev_alloc(ctx, dpairs, cap * sizeof(uint2), "pair block")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dvals, cap * 2 * sizeof(double), "pair values")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, doff, std::min<uint64_t>(nl, cap) * sizeof(uint64_t), "row offsets")) != NW_OK) return st;
  std::vector<uint64_t> off;
  uint64_t r0 = 0;
  while (r0 < nl) {
    off.clear();
    uint64_t total = 0, r1 = r0;
    while (r1 < nl) {
      const uint64_t len = symmetric ? nr - r1 : nr;
      if (total + len > cap && r1 > r0) break;
      off.push_back(total);
      total += len;
      ++r1;
    }
    const uint64_t nrow = r1 - r0;
    NW_CUDA(ctx, cudaMemcpy(doff.p, off.data(), nrow * sizeof(uint64_t), cudaMemcpyHostToDevice));
    matrix_pairs_kernel<<<(unsigned)nrow, 256>>>(dl.as<uint32_t>(), dr.as<uint32_t>(), r0, nr, symmetric ? 1 : 0,
                                                 doff.as<uint64_t>(), dpairs.as<uint2>());
    NW_CUDA(ctx, cudaGetLastError());
    if ((st = eval_pairs(ctx, dpairs.as<uint32_t>(), total, dvals.as<double>(), mode, nullptr)) != NW_OK) return st;
    matrix_scatter_kernel<<<(unsigned)nrow, 256>>>(dvals.as<double2>(), r0, nr, symmetric ? 1 : 0,
                                                   doff.as<uint64_t>(), da.as<double>(), ds.as<double>());
    NW_CUDA(ctx, cudaGetLastError());
    NW_CUDA(ctx, cudaStreamSynchronize(nullptr));
    r0 = r1;
  }
  NW_CUDA(ctx, cudaMemcpy(a_host, da.p, nmat * 8, cudaMemcpyDeviceToHost));
  NW_CUDA(ctx, cudaMemcpy(s_host, ds.p, nmat * 8, cudaMemcpyDeviceToHost));
  return NW_OK;
}

nw_status general_evp(nw_ctx* ctx, int n, const double* h, const double* s, bool project, double tol, double* evals,
                      double* c, int* nkept) {
  if (n <= 0) return fail(ctx, NW_ERR_INVALID, "matrix dimension must be positive");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!ctx->solver) NW_SOLVER(ctx, cusolverDnCreate(&ctx->solver));
  const size_t n2 = (size_t)n * n;
  DevMem dS, dH, dlam, dX, dT, dHt, deps, dC;
  nw_status st;
  if ((st = dev_alloc(ctx, dS, n2 * 8, "overlap")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dH, n2 * 8, "Hamiltonian")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dlam, (size_t)n * 8, "overlap eigenvalues")) != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpy(dS.p, s, n2 * 8, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(dH.p, h, n2 * 8, cudaMemcpyHostToDevice));
  // The row-major input read column-major is the transpose: its lower triangle (the one the
  // reference diagonalises, UPLO::Lower) is the upper triangle of the column-major view.
  if ((st = syevd(ctx, CUBLAS_FILL_MODE_UPPER, n, dS.as<double>(), dlam.as<double>())) != NW_OK) return st;
  std::vector<double> lam(n);
  NW_CUDA(ctx, cudaMemcpy(lam.data(), dlam.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
  // the products below read the column-major (cuSOLVER) results as row-major transposes
  int k = n;
  double* X = nullptr;
  if (project) {
    // positive_subspace: eigenvalues > tol, ascending, are the last k columns
    k = 0;
    for (int i = 0; i < n; ++i) k += lam[i] > tol ? 1 : 0;
    for (int i = 0; i < n - k; ++i)
      if (lam[i] > tol) return fail(ctx, NW_ERR_CUDA, "eigenvalues not ascending");
    if (k == 0) {
      *nkept = 0;
      return NW_OK;
    }
    X = dS.as<double>() + (size_t)(n - k) * n;
    scale_columns_kernel<<<148 * 4, 256>>>(X, dlam.as<double>() + (n - k), n, k);
    NW_CUDA(ctx, cudaGetLastError());
  } else {
    // X = U diag(lam^-1/2) U^T
    if ((st = dev_alloc(ctx, dX, n2 * 8, "orthogonaliser")) != NW_OK) return st;
    if ((st = dev_alloc(ctx, dT, n2 * 8, "orthogonaliser work")) != NW_OK) return st;
    NW_CUDA(ctx, cudaMemcpy(dT.p, dS.p, n2 * 8, cudaMemcpyDeviceToDevice));
    scale_columns_kernel<<<148 * 4, 256>>>(dT.as<double>(), dlam.as<double>(), n, n);
    NW_CUDA(ctx, cudaGetLastError());
    NW_CUDA(ctx, dgemm_strided(0, true, false, n, n, n, 1.0, dS.as<double>(), n, 0, dT.as<double>(), n, 0, 0.0,
                               dX.as<double>(), n, 0, 1));
    X = dX.as<double>();
  }
  // Ht = X^T H X with the full H (the column-major view of the row-major H is H^T)
  DevMem dHX;
  if ((st = dev_alloc(ctx, dHX, (size_t)n * k * 8, "H X")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dHt, (size_t)k * k * 8, "projected Hamiltonian")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, deps, (size_t)k * 8, "eigenvalues")) != NW_OK) return st;
  if ((st = dev_alloc(ctx, dC, (size_t)n * k * 8, "eigenvectors")) != NW_OK) return st;
  NW_CUDA(ctx, dgemm_strided(0, false, true, k, n, n, 1.0, X, n, 0, dH.as<double>(), n, 0, 0.0, dHX.as<double>(), n,
                             0, 1));
  NW_CUDA(ctx, dgemm_strided(0, false, true, k, k, n, 1.0, dHX.as<double>(), n, 0, X, n, 0, 0.0, dHt.as<double>(), k,
                             0, 1));
  // column-major Ht holds the matrix itself: its lower triangle is UPLO::Lower
  if ((st = syevd(ctx, CUBLAS_FILL_MODE_LOWER, k, dHt.as<double>(), deps.as<double>())) != NW_OK) return st;
  // C = X U2 (n x k); computed as C^T = U2^T X^T column-major (k x n) = row-major n x k
  NW_CUDA(ctx, dgemm_strided(0, true, true, n, k, k, 1.0, X, n, 0, dHt.as<double>(), k, 0, 0.0, dC.as<double>(), k,
                             0, 1));
  NW_CUDA(ctx, cudaMemcpy(evals, deps.p, (size_t)k * 8, cudaMemcpyDeviceToHost));
  NW_CUDA(ctx, cudaMemcpy(c, dC.p, (size_t)n * k * 8, cudaMemcpyDeviceToHost));
  *nkept = k;
  return NW_OK;
}

}  // namespace nw
