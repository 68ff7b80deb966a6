// NOCI-PT2 / SNOCI linear solve on the GPU (nw_pt2_*): the candidate-candidate shifted Fock
// matrix M = F - E0 S stored packed on the device, its symmetric mat-vec, the projected
// operator M^Omega, the diagonal / Woodbury preconditioners and restarted right-preconditioned
// GMRES, all in FP64.
//
//   build     : build_candidate_m / fill_candidate_m (src/snoci/operators.rs:205-296): the upper
//               triangle of M in packed rows (row a holds M[a][a..n)), from the (F, S) pair
//               pipeline; the pairs of consecutive rows are exactly consecutive packed entries.
//   mat-vec   : apply_candidate_m (operators.rs:375-488) with the stored matrix: one pass over
//               the packed triangle in 256 x 256 tiles; a tile adds its row sums to y[rows] and,
//               off the diagonal, its column sums to y[cols] (FP64 atomics, 512 per tile).  The
//               triangle is streamed from HBM once per product.  Without a stored matrix
//               (nw_pt2_create_matrix_free, operators.rs:424-471) every product evaluates the
//               upper-triangle (F, S) pairs again through the sorted pair pipeline, block by
//               block, and accumulates them into y directly: no n^2 storage.
//   projected : apply_omega_m / apply_projection_correction (operators.rs:696-955):
//               y = M x - f_a0 (s_0a.x) - s_a0 (f_0a.x) + 2 E0 s_a0 (s_0a.x).
//   GMRES     : gmres / run_arnoldi_cycle (src/snoci/gmres.rs:268-544): zero start, Arnoldi on
//               A P^-1 with two Gram-Schmidt passes (here classical, as two matrix-vector
//               products per pass, in place of the reference's two modified passes), Givens
//               rotations, back substitution, restart from the true residual; convergence on
//               |r| / sqrt(n) <= res_tol.
//   precond   : Preconditioner::new / apply (src/snoci/types.rs:161-288): diagonal inverse with
//               the reference's floor, and the Woodbury rank-2 correction for the projection.
#include <cuda_runtime.h>
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "internal.cuh"

namespace {

constexpr int kTile = 256;
constexpr int kTileWarps = 8;
constexpr int kRowsPerWarp = kTile / kTileWarps;  // 32
constexpr int kColsPerLane = kTile / 32;          // 8

__host__ __device__ inline uint64_t row_start(uint64_t a, uint64_t n) { return a * (2 * n - a + 1) / 2; }

// Tile (I, J), I <= J, of the upper triangle for linear tile index t (row-major over I).
__device__ inline void tile_of(uint64_t t, uint64_t nb, uint64_t* I, uint64_t* J) {
  // start(I) = I nb - I (I - 1) / 2; solve start(I) <= t with a float guess and exact fix-up
  const double b = 2.0 * (double)nb + 1.0;
  const double g = floor((b - sqrt(b * b - 8.0 * (double)t)) / 2.0);
  uint64_t i = g < 0 ? 0 : (uint64_t)g;
  if (i >= nb) i = nb - 1;
  auto start = [nb](uint64_t r) { return r * nb - r * (r - 1) / 2; };
  while (i > 0 && start(i) > t) --i;
  while (i + 1 < nb && start(i + 1) <= t) ++i;
  *I = i;
  *J = i + (t - start(i));
}

// One 256 x 256 tile per block, 8 warps x 32 rows; a lane holds 8 columns (stride 32, so each
// load instruction of a warp reads 256 contiguous bytes of one packed row).  A warp issues the
// loads of kSymvRows rows before it reduces any of them, so 8 x kSymvRows x 256 bytes per warp
// are in flight; the row sums go to y[rows] and, off the diagonal, the per-lane column sums
// to y[cols].
constexpr int kSymvRows = 2;

__global__ void __launch_bounds__(kTile, 2) packed_symv_kernel(const double* __restrict__ m, uint64_t n, uint64_t nb,
                                                               const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double xrow[kTile];
  __shared__ double rowsum[kTile];
  __shared__ double colsum[kTileWarps][kTile];
  uint64_t I, J;
  tile_of(blockIdx.x, nb, &I, &J);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t r0 = I * kTile, c0 = J * kTile;
  xrow[threadIdx.x] = r0 + threadIdx.x < n ? x[r0 + threadIdx.x] : 0.0;
  double xc[kColsPerLane], cacc[kColsPerLane];
#pragma unroll
  for (int k = 0; k < kColsPerLane; ++k) {
    const uint64_t b = c0 + lane + 32 * k;
    xc[k] = b < n ? x[b] : 0.0;
    cacc[k] = 0.0;
  }
  __syncthreads();
  for (int rr = 0; rr < kRowsPerWarp; rr += kSymvRows) {
    double v[kSymvRows][kColsPerLane];
#pragma unroll
    for (int g = 0; g < kSymvRows; ++g) {
      const uint64_t a = r0 + warp * kRowsPerWarp + rr + g;
      const double* row = m + (a < n ? row_start(a, n) - a : 0);  // row[b] = M[a][b] for b >= a
#pragma unroll
      for (int k = 0; k < kColsPerLane; ++k) {
        const uint64_t b = c0 + lane + 32 * k;
        v[g][k] = (a < n && b < n && b >= a) ? __ldcs(row + b) : 0.0;
      }
    }
#pragma unroll
    for (int g = 0; g < kSymvRows; ++g) {
      const int rl = warp * kRowsPerWarp + rr + g;
      const uint64_t a = r0 + rl;
      const double xa = xrow[rl];
      double rs = 0.0;
#pragma unroll
      for (int k = 0; k < kColsPerLane; ++k) {
        rs = fma(v[g][k], xc[k], rs);
        if (c0 + lane + 32 * k != a) cacc[k] = fma(v[g][k], xa, cacc[k]);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) rs += __shfl_xor_sync(0xFFFFFFFFu, rs, off);
      if (lane == 0) rowsum[rl] = rs;
    }
  }
#pragma unroll
  for (int k = 0; k < kColsPerLane; ++k) colsum[warp][lane + 32 * k] = cacc[k];
  __syncthreads();
  const int t = threadIdx.x;
  if (r0 + t < n && rowsum[t] != 0.0) atomicAdd(y + r0 + t, rowsum[t]);
  double cs = 0.0;
#pragma unroll
  for (int w = 0; w < kTileWarps; ++w) cs += colsum[w][t];
  // column sums of the strictly upper part (entries with b < a were loaded as zero)
  if (c0 + t < n && cs != 0.0) atomicAdd(y + c0 + t, cs);
}

// M[row_start(r0) + k] = F_k - e0 S_k for the (F, S) pairs of consecutive rows.
__global__ void packed_fill_kernel(const double2* __restrict__ fs, uint64_t count, double e0, double* __restrict__ m) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = fs[k];
    m[k] = v.x - e0 * v.y;
  }
}

__global__ void packed_diag_kernel(const double* __restrict__ m, uint64_t n, double* __restrict__ d) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n; a += (uint64_t)gridDim.x * blockDim.x)
    d[a] = m[row_start(a, n)];
}

// Pair k of a block is packed entry base + k; its (row, col) by a search over the rows >= r0.
__global__ void upper_pairs_kernel(const uint32_t* __restrict__ cand, uint64_t n, uint64_t r0, uint64_t base,
                                   uint64_t count, uint2* __restrict__ pairs) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = base + k;
    uint64_t lo = r0, hi = n;  // largest a with row_start(a) <= p
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (row_start(mid, n) <= p)
        lo = mid;
      else
        hi = mid;
    }
    const uint64_t b = lo + (p - row_start(lo, n));
    pairs[k] = make_uint2(cand[lo], cand[b]);
  }
}

// Matrix-free product of one block of upper-triangle entries base .. base + count (rows from
// r0): M_ab = F_ab - e0 S_ab, y[a] += M_ab x[b] and, off the diagonal, y[b] += M_ab x[a]
// (apply_candidate_m without a cached matrix, src/snoci/operators.rs:424-471).  Each thread
// takes kMfRun consecutive entries, which lie in one row except at row ends, and adds its row
// sum with one atomic per row it touches; the column terms go out one atomic each.
constexpr int kMfRun = 8;

__global__ void mf_apply_kernel(const double2* __restrict__ fs, uint64_t n, uint64_t r0, uint64_t base,
                                uint64_t count, double e0, const double* __restrict__ x, double* __restrict__ y) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t k0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * kMfRun; k0 < count; k0 += nthreads * kMfRun) {
    const uint64_t p0 = base + k0;
    uint64_t lo = r0, hi = n;  // row of entry p0: largest a with row_start(a) <= p0
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (row_start(mid, n) <= p0)
        lo = mid;
      else
        hi = mid;
    }
    uint64_t a = lo, b = lo + (p0 - row_start(lo, n));
    double xa = x[a], rowsum = 0.0;
    const uint64_t kend = k0 + kMfRun < count ? k0 + kMfRun : count;
    for (uint64_t k = k0; k < kend; ++k) {
      if (b >= n) {  // next row
        if (rowsum != 0.0) atomicAdd(y + a, rowsum);
        ++a;
        b = a;
        xa = x[a];
        rowsum = 0.0;
      }
      const double2 v = fs[k];
      const double m = v.x - e0 * v.y;
      rowsum = fma(m, x[b], rowsum);
      if (b != a) {
        const double cy = m * xa;
        if (cy != 0.0) atomicAdd(y + b, cy);
      }
      ++b;
    }
    if (rowsum != 0.0) atomicAdd(y + a, rowsum);
  }
}

// diagonal pairs (cand[a], cand[a])
__global__ void diag_pairs_kernel(const uint32_t* __restrict__ cand, uint64_t n, uint2* __restrict__ pairs) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n; a += (uint64_t)gridDim.x * blockDim.x)
    pairs[a] = make_uint2(cand[a], cand[a]);
}

__global__ void diag_fill_kernel(const double2* __restrict__ fs, uint64_t n, double e0, double* __restrict__ d) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < n; a += (uint64_t)gridDim.x * blockDim.x)
    d[a] = fs[a].x - e0 * fs[a].y;
}

__global__ void mul_kernel(const double* __restrict__ a, const double* __restrict__ b, uint64_t n,
                           double* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = a[i] * b[i];
}

inline int grid_n(uint64_t n) { return (int)std::min<uint64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

struct nw_pt2 {
  nw_ctx* ctx = nullptr;
  uint64_t n = 0;
  double e0 = 0.0;
  double* m = nullptr;      // packed upper triangle, n (n + 1) / 2 (null when matrix-free)
  double* mdiag = nullptr;  // diagonal of M
  float last_symv_ms = 0.0f;
  // matrix-free mode: candidates, and one block of upper-triangle pairs and their (F, S)
  uint32_t* dcand = nullptr;
  uint2* pairs = nullptr;
  double2* fs = nullptr;
  uint64_t blk = 0;
};

namespace {

nw_status pfail(nw_pt2* p, nw_status s, const std::string& m) { return nw::fail(p->ctx, s, m); }

#define PT_BLAS(p, call)                                                                           \
  do {                                                                                             \
    const cublasStatus_t s_ = (call);                                                              \
    if (s_ != CUBLAS_STATUS_SUCCESS) return pfail(p, NW_ERR_CUDA, std::string(#call) + " failed"); \
  } while (0)

// First row of the packed entry `base`: largest r with row_start(r) <= base.
uint64_t first_row(uint64_t base, uint64_t n) {
  uint64_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint64_t mid = (lo + hi) >> 1;
    if (row_start(mid, n) <= base)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// y = M x (device vectors, legacy stream): one pass over the packed triangle, or, matrix-free,
// every upper-triangle pair evaluated again through the (F, S) pipeline block by block.
nw_status symv(nw_pt2* p, const double* x, double* y) {
  const uint64_t n = p->n, nb = (n + kTile - 1) / kTile;
  NW_CUDA(p->ctx, cudaMemsetAsync(y, 0, sizeof(double) * n, nullptr));
  if (p->m) {
    const uint64_t ntiles = nb * (nb + 1) / 2;
    packed_symv_kernel<<<(unsigned)ntiles, kTile>>>(p->m, n, nb, x, y);
    NW_CUDA(p->ctx, cudaGetLastError());
    return NW_OK;
  }
  const uint64_t len = n * (n + 1) / 2;
  for (uint64_t base = 0; base < len; base += p->blk) {
    const uint64_t count = std::min(p->blk, len - base);
    const uint64_t r0 = first_row(base, n);
    upper_pairs_kernel<<<grid_n(count), 256>>>(p->dcand, n, r0, base, count, p->pairs);
    nw_status st = nw::eval_pairs(p->ctx, reinterpret_cast<const uint32_t*>(p->pairs), count,
                                  reinterpret_cast<double*>(p->fs), nw::EvalMode::kFS, nullptr);
    if (st != NW_OK) return st;
    mf_apply_kernel<<<grid_n((count + kMfRun - 1) / kMfRun), 256>>>(p->fs, n, r0, base, count, p->e0, x, y);
    NW_CUDA(p->ctx, cudaGetLastError());
  }
  return NW_OK;
}

struct Projection {
  double e0;
  const double *s_a0, *s_0a, *f_a0, *f_0a;  // device
};

// y = M^Omega x.
nw_status apply_omega(nw_pt2* p, const Projection& pr, const double* x, double* y) {
  nw_status st = symv(p, x, y);
  if (st != NW_OK) return st;
  cublasHandle_t h = p->ctx->blas;
  double sx = 0.0, fx = 0.0;
  PT_BLAS(p, cublasDdot(h, (int)p->n, pr.s_0a, 1, x, 1, &sx));
  PT_BLAS(p, cublasDdot(h, (int)p->n, pr.f_0a, 1, x, 1, &fx));
  const double cf = -sx, cs = 2.0 * pr.e0 * sx - fx;
  PT_BLAS(p, cublasDaxpy(h, (int)p->n, &cf, pr.f_a0, 1, y, 1));
  PT_BLAS(p, cublasDaxpy(h, (int)p->n, &cs, pr.s_a0, 1, y, 1));
  return NW_OK;
}

struct Precond {
  double* dinv;
  double *z0, *z1;
  const double *v0, *v1;
  double w00, w01, w10, w11;
  bool active;
};

nw_status apply_precond(nw_pt2* p, const Precond& P, const double* v, double* y) {
  mul_kernel<<<grid_n(p->n), 256>>>(v, P.dinv, p->n, y);
  NW_CUDA(p->ctx, cudaGetLastError());
  if (!P.active) return NW_OK;
  cublasHandle_t h = p->ctx->blas;
  double t0 = 0.0, t1 = 0.0;
  PT_BLAS(p, cublasDdot(h, (int)p->n, P.v0, 1, y, 1, &t0));
  PT_BLAS(p, cublasDdot(h, (int)p->n, P.v1, 1, y, 1, &t1));
  const double c0 = -(P.w00 * t0 + P.w01 * t1), c1 = -(P.w10 * t0 + P.w11 * t1);
  PT_BLAS(p, cublasDaxpy(h, (int)p->n, &c0, P.z0, 1, y, 1));
  PT_BLAS(p, cublasDaxpy(h, (int)p->n, &c1, P.z1, 1, y, 1));
  return NW_OK;
}

}  // namespace

extern "C" {

nw_status nw_pt2_create(nw_ctx* ctx, const uint32_t* cand, uint64_t n, double e0, nw_pt2** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!ctx || !cand || n == 0 || !std::isfinite(e0)) return NW_ERR_INVALID;
  if (!ctx->fock_ready) return nw::fail(ctx, NW_ERR_STATE, "Fock tables not set (nw_update_fock)");
  if (!ctx->d_dets) return nw::fail(ctx, NW_ERR_STATE, "no determinant basis set");
  if (n > 0x7FFFFFFFull) return nw::fail(ctx, NW_ERR_UNSUPPORTED, "too many candidates");
  for (uint64_t i = 0; i < n; ++i)
    if (cand[i] >= ctx->ndet) return nw::fail(ctx, NW_ERR_INVALID, "candidate index out of range");
  const uint64_t nb = (n + kTile - 1) / kTile;
  if (nb * (nb + 1) / 2 > 0x7FFFFFFFull) return nw::fail(ctx, NW_ERR_UNSUPPORTED, "too many candidates");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw_pt2* p = new (std::nothrow) nw_pt2;
  if (!p) return NW_ERR_ALLOC;
  p->ctx = ctx;
  p->n = n;
  p->e0 = e0;
  const uint64_t len = n * (n + 1) / 2;
  uint32_t* dcand = nullptr;
  uint2* pairs = nullptr;
  double2* fs = nullptr;
  auto cleanup = [&](nw_status st) {
    if (dcand) cudaFree(dcand);
    if (pairs) cudaFree(pairs);
    if (fs) cudaFree(fs);
    if (st != NW_OK) {
      if (p->m) cudaFree(p->m);
      if (p->mdiag) cudaFree(p->mdiag);
      delete p;
    }
    return st;
  };
  if (cudaMalloc(&p->m, sizeof(double) * len) != cudaSuccess || cudaMalloc(&p->mdiag, sizeof(double) * n) != cudaSuccess)
    return cleanup(nw::fail(ctx, NW_ERR_ALLOC, "packed candidate matrix allocation failed (" +
                                                   std::to_string(len * 8 >> 20) + " MiB)"));
  constexpr uint64_t kBlock = 1ull << 24;  // pairs per evaluation block
  const uint64_t blk = std::min(kBlock, len);
  if (cudaMalloc(&dcand, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&pairs, sizeof(uint2) * blk) != cudaSuccess ||
      cudaMalloc(&fs, sizeof(double2) * blk) != cudaSuccess)
    return cleanup(nw::fail(ctx, NW_ERR_ALLOC, "candidate pair buffers"));
  if (cudaMemcpy(dcand, cand, sizeof(uint32_t) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(nw::fail(ctx, NW_ERR_CUDA, "candidate upload"));
  for (uint64_t base = 0; base < len; base += blk) {
    const uint64_t count = std::min(blk, len - base);
    // first row of the block: largest r with row_start(r) <= base
    uint64_t lo = 0, hi = n;
    while (hi - lo > 1) {
      const uint64_t mid = (lo + hi) >> 1;
      if (row_start(mid, n) <= base)
        lo = mid;
      else
        hi = mid;
    }
    upper_pairs_kernel<<<grid_n(count), 256>>>(dcand, n, lo, base, count, pairs);
    nw_status st = nw::eval_pairs(ctx, reinterpret_cast<const uint32_t*>(pairs), count, reinterpret_cast<double*>(fs),
                                  nw::EvalMode::kFS, nullptr);
    if (st != NW_OK) return cleanup(st);
    packed_fill_kernel<<<grid_n(count), 256>>>(fs, count, e0, p->m + base);
    if (cudaGetLastError() != cudaSuccess) return cleanup(nw::fail(ctx, NW_ERR_CUDA, "packed fill"));
  }
  packed_diag_kernel<<<grid_n(n), 256>>>(p->m, n, p->mdiag);
  if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(nw::fail(ctx, NW_ERR_CUDA, "candidate matrix build"));
  *out = p;
  return cleanup(NW_OK);
}

nw_status nw_pt2_create_matrix_free(nw_ctx* ctx, const uint32_t* cand, uint64_t n, double e0, nw_pt2** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!ctx || !cand || n == 0 || !std::isfinite(e0)) return NW_ERR_INVALID;
  if (!ctx->fock_ready) return nw::fail(ctx, NW_ERR_STATE, "Fock tables not set (nw_update_fock)");
  if (!ctx->d_dets) return nw::fail(ctx, NW_ERR_STATE, "no determinant basis set");
  if (n > 0x7FFFFFFFull) return nw::fail(ctx, NW_ERR_UNSUPPORTED, "too many candidates");
  for (uint64_t i = 0; i < n; ++i)
    if (cand[i] >= ctx->ndet) return nw::fail(ctx, NW_ERR_INVALID, "candidate index out of range");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw_pt2* p = new (std::nothrow) nw_pt2;
  if (!p) return NW_ERR_ALLOC;
  p->ctx = ctx;
  p->n = n;
  p->e0 = e0;
  constexpr uint64_t kBlock = 1ull << 24;  // pairs per evaluation block
  p->blk = std::max(std::min(kBlock, n * (n + 1) / 2), n);  // a block also holds the n diagonal pairs
  auto cleanup = [&](nw_status st) {
    if (st != NW_OK) nw_pt2_destroy(p);
    return st;
  };
  if (cudaMalloc(&p->dcand, sizeof(uint32_t) * n) != cudaSuccess || cudaMalloc(&p->mdiag, sizeof(double) * n) != cudaSuccess ||
      cudaMalloc(&p->pairs, sizeof(uint2) * p->blk) != cudaSuccess ||
      cudaMalloc(&p->fs, sizeof(double2) * p->blk) != cudaSuccess)
    return cleanup(nw::fail(ctx, NW_ERR_ALLOC, "matrix-free candidate buffers"));
  if (cudaMemcpy(p->dcand, cand, sizeof(uint32_t) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(nw::fail(ctx, NW_ERR_CUDA, "candidate upload"));
  // the diagonal for the preconditioners
  diag_pairs_kernel<<<grid_n(n), 256>>>(p->dcand, n, p->pairs);
  nw_status st = nw::eval_pairs(ctx, reinterpret_cast<const uint32_t*>(p->pairs), n, reinterpret_cast<double*>(p->fs),
                                nw::EvalMode::kFS, nullptr);
  if (st != NW_OK) return cleanup(st);
  diag_fill_kernel<<<grid_n(n), 256>>>(p->fs, n, e0, p->mdiag);
  if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(nw::fail(ctx, NW_ERR_CUDA, "matrix-free set-up"));
  *out = p;
  return NW_OK;
}

nw_status nw_pt2_apply_m(nw_pt2* p, const double* x, double* y) {
  if (!p || !x || !y) return NW_ERR_INVALID;
  nw_ctx* ctx = p->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  double *dx = nullptr, *dy = nullptr;
  if (cudaMalloc(&dx, sizeof(double) * p->n) != cudaSuccess || cudaMalloc(&dy, sizeof(double) * p->n) != cudaSuccess) {
    if (dx) cudaFree(dx);
    return pfail(p, NW_ERR_ALLOC, "vector allocation");
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = cudaMemcpy(dx, x, sizeof(double) * p->n, cudaMemcpyHostToDevice);
  nw_status st = NW_OK;
  if (e == cudaSuccess) {
    cudaEventRecord(e0, nullptr);
    st = symv(p, dx, dy);
    cudaEventRecord(e1, nullptr);
    if (st == NW_OK) e = cudaMemcpy(y, dy, sizeof(double) * p->n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && st == NW_OK) cudaEventElapsedTime(&p->last_symv_ms, e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dx);
  cudaFree(dy);
  if (st != NW_OK) return st;
  if (e != cudaSuccess) return nw::cuda_fail(ctx, e, "candidate mat-vec");
  return NW_OK;
}

nw_status nw_pt2_last_apply_ms(const nw_pt2* p, float* ms) {
  if (!p || !ms) return NW_ERR_INVALID;
  *ms = p->last_symv_ms;
  return NW_OK;
}

nw_status nw_pt2_solve(nw_pt2* p, const nw_pt2_projection* proj, const double* rhs, const nw_gmres_opts* opts,
                       double* x_out, nw_gmres_info* info) {
  if (!p || !proj || !rhs || !opts || !x_out || !info) return NW_ERR_INVALID;
  if (!proj->s_a0 || !proj->s_0a || !proj->f_a0 || !proj->f_0a) return NW_ERR_INVALID;
  if (opts->max_iter < 0 || opts->restart < 1 || !(opts->res_tol >= 0.0)) return NW_ERR_INVALID;
  nw_ctx* ctx = p->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  const uint64_t n = p->n;
  const int kmax = opts->restart;
  // device vectors: 4 projection, dinv, z0, z1, b, x, r, w, z, Krylov basis (kmax + 1)
  const uint64_t nvec = 12 + (uint64_t)kmax + 1;
  double* base = nullptr;
  if (cudaMalloc(&base, sizeof(double) * n * nvec) != cudaSuccess) return pfail(p, NW_ERR_ALLOC, "GMRES vectors");
  struct Free {
    double* q;
    ~Free() { cudaFree(q); }
  } free_base{base};
  auto vec = [&](int i) { return base + (uint64_t)i * n; };
  double *s_a0 = vec(0), *s_0a = vec(1), *f_a0 = vec(2), *f_0a = vec(3), *dinv = vec(4), *z0 = vec(5), *z1 = vec(6);
  double *b = vec(7), *x = vec(8), *r = vec(9), *w = vec(10), *z = vec(11), *Q = vec(12);
  const size_t vb = sizeof(double) * n;
  NW_CUDA(ctx, cudaMemcpy(s_a0, proj->s_a0, vb, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(s_0a, proj->s_0a, vb, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(f_a0, proj->f_a0, vb, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(f_0a, proj->f_0a, vb, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(b, rhs, vb, cudaMemcpyHostToDevice));
  const Projection pr{proj->e0, s_a0, s_0a, f_a0, f_0a};
  cublasHandle_t h = ctx->blas;

  // preconditioner (types.rs:161-251): Diag inverts the projected diagonal, Woodbury the
  // unprojected diagonal plus the rank-2 projection terms
  std::vector<double> mdiag(n);
  NW_CUDA(ctx, cudaMemcpy(mdiag.data(), p->mdiag, vb, cudaMemcpyDeviceToHost));
  const double *sa0 = proj->s_a0, *s0a = proj->s_0a, *fa0 = proj->f_a0, *f0a = proj->f_0a;
  const bool woodbury = opts->preconditioner == NW_PRECOND_WOODBURY;
  std::vector<double> d(n);
  for (uint64_t a = 0; a < n; ++a)
    d[a] = woodbury ? mdiag[a]
                    : mdiag[a] - fa0[a] * s0a[a] - sa0[a] * f0a[a] + 2.0 * proj->e0 * sa0[a] * s0a[a];
  double dmax = 0.0;
  for (double v : d) dmax = std::max(dmax, std::fabs(v));
  const double dfloor = std::max(1e-12 * dmax, 1e-14);
  std::vector<double> hd(n), hz0(n), hz1(n);
  for (uint64_t a = 0; a < n; ++a) hd[a] = std::fabs(d[a]) > dfloor ? 1.0 / d[a] : d[a] / (dfloor * dfloor);
  Precond P{dinv, z0, z1, s_0a, f_0a, 1.0, 0.0, 0.0, 1.0, false};
  if (woodbury) {
    double c00 = 1.0, c01 = 0.0, c10 = 0.0, c11 = 1.0;
    for (uint64_t a = 0; a < n; ++a) {
      const double u0 = -fa0[a] + 2.0 * proj->e0 * sa0[a], u1 = -sa0[a];
      hz0[a] = hd[a] * u0;
      hz1[a] = hd[a] * u1;
      c00 += s0a[a] * hz0[a];
      c01 += s0a[a] * hz1[a];
      c10 += f0a[a] * hz0[a];
      c11 += f0a[a] * hz1[a];
    }
    const double det = c00 * c11 - c01 * c10;
    if (std::fabs(det) > 1e-14) {
      P.active = true;
      P.w00 = c11 / det;
      P.w01 = -c01 / det;
      P.w10 = -c10 / det;
      P.w11 = c00 / det;
    }
    NW_CUDA(ctx, cudaMemcpy(z0, hz0.data(), vb, cudaMemcpyHostToDevice));
    NW_CUDA(ctx, cudaMemcpy(z1, hz1.data(), vb, cudaMemcpyHostToDevice));
  }
  NW_CUDA(ctx, cudaMemcpy(dinv, hd.data(), vb, cudaMemcpyHostToDevice));

  const double rms = std::sqrt((double)n);
  const double one = 1.0, mone = -1.0, zero = 0.0;
  constexpr double kSmall = 1e-14;
  NW_CUDA(ctx, cudaMemset(x, 0, vb));
  NW_CUDA(ctx, cudaMemcpy(r, b, vb, cudaMemcpyDeviceToDevice));  // r = b - A 0
  double beta = 0.0;
  PT_BLAS(p, cublasDnrm2(h, (int)n, r, 1, &beta));
  double res = beta / rms;
  int total = 0;
  bool converged = res <= opts->res_tol;
  std::vector<double> H((size_t)(kmax + 1) * kmax), cs(kmax), sn(kmax), g(kmax + 1), hcol(kmax + 1), c(kmax + 1);
  auto Hh = [&](int i, int j) -> double& { return H[(size_t)i * kmax + j]; };
  while (!converged && total < opts->max_iter) {
    PT_BLAS(p, cublasDnrm2(h, (int)n, r, 1, &beta));
    if (beta <= kSmall) {
      res = beta / rms;
      break;
    }
    // the Krylov dimension cannot exceed n (and r holds the k + 1 coefficients below)
    const int inner = (int)std::min<uint64_t>(std::min(kmax, opts->max_iter - total), n);
    std::fill(H.begin(), H.end(), 0.0);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    const double inv = 1.0 / beta;
    NW_CUDA(ctx, cudaMemcpy(Q, r, vb, cudaMemcpyDeviceToDevice));
    PT_BLAS(p, cublasDscal(h, (int)n, &inv, Q, 1));
    int kfinal = 0;
    for (int k = 0; k < inner; ++k) {
      const double* qk = Q + (uint64_t)k * n;
      nw_status st = apply_precond(p, P, qk, z);
      if (st == NW_OK) st = apply_omega(p, pr, z, w);
      if (st != NW_OK) return st;
      // two classical Gram-Schmidt passes against q_0..q_k; r is free during the cycle and
      // holds the k + 1 <= n coefficients
      std::fill(hcol.begin(), hcol.end(), 0.0);
      for (int pass = 0; pass < 2; ++pass) {
        PT_BLAS(p, cublasDgemv(h, CUBLAS_OP_T, (int)n, k + 1, &one, Q, (int)n, w, 1, &zero, r, 1));
        PT_BLAS(p, cublasDgemv(h, CUBLAS_OP_N, (int)n, k + 1, &mone, Q, (int)n, r, 1, &one, w, 1));
        NW_CUDA(ctx, cudaMemcpy(c.data(), r, sizeof(double) * (k + 1), cudaMemcpyDeviceToHost));
        for (int j = 0; j <= k; ++j) hcol[j] += c[j];
      }
      double hnext = 0.0;
      PT_BLAS(p, cublasDnrm2(h, (int)n, w, 1, &hnext));
      for (int j = 0; j <= k; ++j) Hh(j, k) = hcol[j];
      Hh(k + 1, k) = hnext;
      if (hnext > kSmall) {
        const double s = 1.0 / hnext;
        NW_CUDA(ctx, cudaMemcpy(Q + (uint64_t)(k + 1) * n, w, vb, cudaMemcpyDeviceToDevice));
        PT_BLAS(p, cublasDscal(h, (int)n, &s, Q + (uint64_t)(k + 1) * n, 1));
      }
      // previous rotations, then the new one (gmres.rs:197-266)
      for (int j = 0; j < k; ++j) {
        const double t = cs[j] * Hh(j, k) + sn[j] * Hh(j + 1, k);
        Hh(j + 1, k) = -sn[j] * Hh(j, k) + cs[j] * Hh(j + 1, k);
        Hh(j, k) = t;
      }
      const double a = Hh(k, k), bb = Hh(k + 1, k);
      const double den = std::hypot(a, bb);
      if (den > kSmall) {
        cs[k] = a / den;
        sn[k] = bb / den;
      } else {
        cs[k] = 1.0;
        sn[k] = 0.0;
      }
      Hh(k, k) = cs[k] * a + sn[k] * bb;
      Hh(k + 1, k) = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      kfinal = k + 1;
      if (std::fabs(g[k + 1]) / rms <= opts->res_tol || hnext <= kSmall) break;
    }
    // back substitution, then x += P^-1 Q y
    std::vector<double> yv(kfinal, 0.0);
    for (int ii = kfinal - 1; ii >= 0; --ii) {
      double s = g[ii];
      for (int j = ii + 1; j < kfinal; ++j) s -= Hh(ii, j) * yv[j];
      yv[ii] = std::fabs(Hh(ii, ii)) > kSmall ? s / Hh(ii, ii) : 0.0;
    }
    NW_CUDA(ctx, cudaMemcpy(r, yv.data(), sizeof(double) * kfinal, cudaMemcpyHostToDevice));
    PT_BLAS(p, cublasDgemv(h, CUBLAS_OP_N, (int)n, kfinal, &one, Q, (int)n, r, 1, &zero, w, 1));
    nw_status st = apply_precond(p, P, w, z);
    if (st != NW_OK) return st;
    PT_BLAS(p, cublasDaxpy(h, (int)n, &one, z, 1, x, 1));
    total += kfinal;
    // the true residual decides convergence
    st = apply_omega(p, pr, x, w);
    if (st != NW_OK) return st;
    NW_CUDA(ctx, cudaMemcpy(r, b, vb, cudaMemcpyDeviceToDevice));
    PT_BLAS(p, cublasDaxpy(h, (int)n, &mone, w, 1, r, 1));
    PT_BLAS(p, cublasDnrm2(h, (int)n, r, 1, &beta));
    res = beta / rms;
    converged = res <= opts->res_tol;
  }
  NW_CUDA(ctx, cudaMemcpy(x_out, x, vb, cudaMemcpyDeviceToHost));
  info->residual_rms = res;
  info->iterations = total;
  info->converged = converged ? 1 : 0;
  return NW_OK;
}

nw_status nw_pt2_destroy(nw_pt2* p) {
  if (!p) return NW_OK;
  cudaSetDevice(p->ctx->device);
  cudaDeviceSynchronize();
  for (void* q : {(void*)p->m, (void*)p->mdiag, (void*)p->dcand, (void*)p->pairs, (void*)p->fs})
    if (q) cudaFree(q);
  delete p;
  return NW_OK;
}

}  // extern "C"
