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
//               upper-triangle (F, S) pairs again through the sorted pair pipeline in blocks of
//               whole 256 x 256 tiles and accumulates each tile into y as the stored product
//               does (row and column sums, 512 atomics per tile): no n^2 storage.
//   projected : apply_omega_m / apply_projection_correction (operators.rs:696-955):
//               y = M x - f_a0 (s_0a.x) - s_a0 (f_0a.x) + 2 E0 s_a0 (s_0a.x).
//   GMRES     : gmres / run_arnoldi_cycle (src/snoci/gmres.rs:268-544): zero start, Arnoldi on
//               A P^-1 with two Gram-Schmidt passes (here classical, as two matrix-vector
//               products per pass, in place of the reference's two modified passes), Givens
//               rotations, back substitution, restart from the true residual; convergence on
//               |r| / sqrt(n) <= res_tol.  Each Arnoldi step runs on the device (own two-pass
//               reduction kernels; the Hessenberg matrix, rotations and stopping rule in device
//               memory); on the packed path the step is one CUDA graph, replayed for every step
//               of a cycle without host synchronisation (one per restart cycle).
//   precond   : Preconditioner::new / apply (src/snoci/types.rs:161-288): diagonal inverse with
//               the reference's floor, and the Woodbury rank-2 correction for the projection.
#include <cuda_runtime.h>
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
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
                                                               const double* __restrict__ x, double* __restrict__ y,
                                                               const int* __restrict__ skip) {
  if (skip && *skip) return;  // a finished Arnoldi cycle (device-side GMRES)
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

// Row of packed entry p: the largest a with row_start(a) <= p, from the root of the quadratic
// row_start(a) = p (FP64, within one of the answer) and an exact integer fix-up.
__device__ inline uint64_t row_of(uint64_t p, uint64_t n) {
  const double b = 2.0 * (double)n + 1.0;
  const double g = floor((b - sqrt(b * b - 8.0 * (double)p)) / 2.0);
  uint64_t a = g < 0.0 ? 0 : (uint64_t)g;
  if (a >= n) a = n - 1;
  while (a > 0 && row_start(a, n) > p) --a;
  while (a + 1 < n && row_start(a + 1, n) <= p) ++a;
  return a;
}

// Pair k of a block is packed entry base + k (the packed build's row-major order).
__global__ void upper_pairs_kernel(const uint32_t* __restrict__ cand, uint64_t n, uint64_t base, uint64_t count,
                                   uint2* __restrict__ pairs) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = base + k;
    const uint64_t a = row_of(p, n);
    const uint64_t b = a + (p - row_start(a, n));
    pairs[k] = make_uint2(cand[a], cand[b]);
  }
}

// Matrix-free products go over the upper triangle in 256 x 256 tiles (I <= J), 65536 pair slots
// per tile in row-major (i, j) order; slots outside the triangle (b < a on a diagonal tile, or
// past the last candidate) get the pair (cand[0], cand[0]) and are ignored by the product.
constexpr uint64_t kTileSlots = (uint64_t)kTile * kTile;

__global__ void tile_pairs_kernel(const uint32_t* __restrict__ cand, uint64_t n, uint64_t nb, uint64_t t0,
                                  uint64_t nslots, uint2* __restrict__ pairs) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < nslots; s += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t I, J;
    tile_of(t0 + s / kTileSlots, nb, &I, &J);
    const uint64_t k = s % kTileSlots;
    const uint64_t a = I * kTile + k / kTile, b = J * kTile + k % kTile;
    const bool live = a < n && b < n && b >= a;
    pairs[s] = live ? make_uint2(cand[a], cand[b]) : make_uint2(cand[0], cand[0]);
  }
}

// y += M x over the tiles t0 .. t0 + gridDim.x of a block of evaluated (F, S) slots, M = F - e0 S:
// the structure of packed_symv_kernel (8 warps x 32 rows, a lane holds 8 columns; row sums to
// y[rows], strictly-upper column sums to y[cols], 512 atomics per tile) with the tile's entries
// read from its 65536 contiguous (F, S) slots.
__global__ void __launch_bounds__(kTile, 2) mf_tile_apply_kernel(const double2* __restrict__ fs, uint64_t n,
                                                                 uint64_t nb, uint64_t t0, double e0,
                                                                 const double* __restrict__ x,
                                                                 double* __restrict__ y) {
  __shared__ double xrow[kTile];
  __shared__ double rowsum[kTile];
  __shared__ double colsum[kTileWarps][kTile];
  uint64_t I, J;
  tile_of(t0 + blockIdx.x, nb, &I, &J);
  const double2* tile = fs + (uint64_t)blockIdx.x * kTileSlots;
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
      const int rl = warp * kRowsPerWarp + rr + g;
      const uint64_t a = r0 + rl;
#pragma unroll
      for (int k = 0; k < kColsPerLane; ++k) {
        const int cl = lane + 32 * k;
        const uint64_t b = c0 + cl;
        double m = 0.0;
        if (a < n && b < n && b >= a) {
          const double2 e = __ldcs(tile + rl * kTile + cl);
          m = e.x - e0 * e.y;
        }
        v[g][k] = m;
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
  if (c0 + t < n && cs != 0.0) atomicAdd(y + c0 + t, cs);
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

// ---------------------------------------------------------------------------------------
// Device-side Arnoldi step of GMRES (one CUDA graph per solve on the packed path).  The
// scalars of the cycle live on the device (ArnoldiState, the Hessenberg matrix, the Givens
// rotations and the rotated right-hand side g); every reduction is two-pass and in a fixed
// order (per-block partial sums, then one ordered sum), and every kernel returns at once when
// the cycle is done, so the host can queue the `inner` steps of a cycle back to back and
// synchronise once per cycle (gmres.rs:197-266 for the rotations and the stopping rule).
// ---------------------------------------------------------------------------------------
constexpr int kVB = 256;            // threads of the vector kernels
constexpr int kVBlocks = 148 * 4;   // blocks of the vector kernels = partial sums per reduction

struct ArnoldiState {
  int k;        // current column
  int inner;    // columns of this cycle
  int done;     // the cycle has finished (converged, breakdown or k == inner)
  int kfinal;   // columns completed
  int col;      // column that receives w / h_{k+1,k}
  int pad;
  double tol;   // res_tol sqrt(n): the stopping bound on |g[k+1]|
  double inv;   // 1 / h_{k+1,k} (0 on breakdown)
};

constexpr double kArnoldiSmall = 1e-14;

// Sum over the block of v (thread 0 gets the total); sh holds 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
  }
  return t;
}

// Ordered sum of the kVBlocks partials part[b * stride + j] (every thread gets it).
__device__ __forceinline__ double sum_partials(const double* __restrict__ part, int stride, int j, double* sh) {
  double v = 0.0;
  for (int b = threadIdx.x; b < kVBlocks; b += blockDim.x) v += part[(size_t)b * stride + j];
  v = block_sum(v, sh);
  if (threadIdx.x == 0) sh[32] = v;
  __syncthreads();
  v = sh[32];
  __syncthreads();
  return v;
}

// z = P^-1 q_k, diagonal part: z = dinv (.) q_k, with partial sums of (v0.z, v1.z) when the
// Woodbury correction follows, else of (s_0a.z, f_0a.z) for the projection.
__global__ void __launch_bounds__(kVB) arn_precond_kernel(const ArnoldiState* __restrict__ st, const double* __restrict__ Q,
                                                          const double* __restrict__ dinv, const double* __restrict__ u0,
                                                          const double* __restrict__ u1, uint64_t n, double* __restrict__ z,
                                                          double* __restrict__ part) {
  __shared__ double sh[33];
  if (st->done) return;
  const double* q = Q + (uint64_t)st->k * n;
  double a0 = 0.0, a1 = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) {
    const double v = q[i] * dinv[i];
    z[i] = v;
    a0 = fma(u0[i], v, a0);
    a1 = fma(u1[i], v, a1);
  }
  a0 = block_sum(a0, sh);
  a1 = block_sum(a1, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a0;
    part[2 * blockIdx.x + 1] = a1;
  }
}

// Woodbury correction z += c0 z0 + c1 z1, c = -W (v0.z, v1.z), then partial sums of
// (s_0a.z, f_0a.z) into part_out.
__global__ void __launch_bounds__(kVB) arn_woodbury_kernel(const ArnoldiState* __restrict__ st,
                                                           const double* __restrict__ part_in, double w00, double w01,
                                                           double w10, double w11, const double* __restrict__ z0,
                                                           const double* __restrict__ z1, const double* __restrict__ s_0a,
                                                           const double* __restrict__ f_0a, uint64_t n,
                                                           double* __restrict__ z, double* __restrict__ part_out) {
  __shared__ double sh[33];
  if (st->done) return;
  const double t0 = sum_partials(part_in, 2, 0, sh), t1 = sum_partials(part_in, 2, 1, sh);
  const double c0 = -(w00 * t0 + w01 * t1), c1 = -(w10 * t0 + w11 * t1);
  double a0 = 0.0, a1 = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) {
    const double v = z[i] + c0 * z0[i] + c1 * z1[i];
    z[i] = v;
    a0 = fma(s_0a[i], v, a0);
    a1 = fma(f_0a[i], v, a1);
  }
  a0 = block_sum(a0, sh);
  a1 = block_sum(a1, sh);
  if (threadIdx.x == 0) {
    part_out[2 * blockIdx.x] = a0;
    part_out[2 * blockIdx.x + 1] = a1;
  }
}

__global__ void __launch_bounds__(kVB) arn_zero_kernel(const ArnoldiState* __restrict__ st, uint64_t n,
                                                       double* __restrict__ w) {
  if (st->done) return;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) w[i] = 0.0;
}

// Projection of the product (apply_projection_correction): w += -sx f_a0 + (2 e0 sx - fx) s_a0
// with (sx, fx) = (s_0a.z, f_0a.z); then partial sums of q_j.w for j <= k (first Gram-Schmidt
// pass) into part[b * ld + j].
__global__ void __launch_bounds__(kVB) arn_project_kernel(const ArnoldiState* __restrict__ st,
                                                          const double* __restrict__ part_sf, double e0,
                                                          const double* __restrict__ f_a0, const double* __restrict__ s_a0,
                                                          const double* __restrict__ Q, uint64_t n, int ld,
                                                          double* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[33];
  if (st->done) return;
  const double sx = sum_partials(part_sf, 2, 0, sh), fx = sum_partials(part_sf, 2, 1, sh);
  const double cf = -sx, cs = 2.0 * e0 * sx - fx;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB)
    w[i] = w[i] + cf * f_a0[i] + cs * s_a0[i];
  __syncthreads();
  const int k = st->k;
  for (int j = 0; j <= k; ++j) {
    const double* q = Q + (uint64_t)j * n;
    double a = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) a = fma(q[i], w[i], a);
    a = block_sum(a, sh);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * ld + j] = a;
  }
}

// Gram-Schmidt coefficients c_j = sum of the partials (j <= k); hcol = c (first pass) or
// hcol += c (second pass).  One block.
__global__ void __launch_bounds__(kVB) arn_coef_kernel(const ArnoldiState* __restrict__ st, const double* __restrict__ part,
                                                       int ld, int accumulate, double* __restrict__ coef,
                                                       double* __restrict__ hcol) {
  if (st->done) return;
  const int k = st->k, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int j = wid; j <= k; j += kVB / 32) {
    double v = 0.0;
    for (int b = lane; b < kVBlocks; b += 32) v += part[(size_t)b * ld + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) {
      coef[j] = v;
      hcol[j] = accumulate ? hcol[j] + v : v;
    }
  }
}

// w -= sum_{j <= k} q_j c_j; then the partial sums of the second pass (q_j.w into part) or,
// after it, of |w|^2 (part[b * ld]).
__global__ void __launch_bounds__(kVB) arn_orth_kernel(const ArnoldiState* __restrict__ st, const double* __restrict__ Q,
                                                       const double* __restrict__ coef, uint64_t n, int ld, int norm,
                                                       double* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[33];
  if (st->done) return;
  const int k = st->k;
  double a2 = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) {
    double v = w[i];
    for (int j = 0; j <= k; ++j) v -= Q[(uint64_t)j * n + i] * coef[j];
    w[i] = v;
    a2 = fma(v, v, a2);
  }
  if (norm) {
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * ld] = a2;
    return;
  }
  __syncthreads();
  for (int j = 0; j <= k; ++j) {
    const double* q = Q + (uint64_t)j * n;
    double a = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) a = fma(q[i], w[i], a);
    a = block_sum(a, sh);
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * ld + j] = a;
  }
}

// h_{k+1,k} = |w|, column k of the Hessenberg matrix, the earlier rotations and the new one,
// the rotated right-hand side and the stopping rule (gmres.rs:197-266).  One block.
__global__ void __launch_bounds__(kVB) arn_givens_kernel(ArnoldiState* __restrict__ st, const double* __restrict__ part,
                                                         int ld, const double* __restrict__ hcol, int kmax,
                                                         double* __restrict__ H, double* __restrict__ cs,
                                                         double* __restrict__ sn, double* __restrict__ g) {
  __shared__ double sh[33];
  if (st->done) return;
  double v = 0.0;
  for (int b = threadIdx.x; b < kVBlocks; b += kVB) v += part[(size_t)b * ld];
  v = block_sum(v, sh);
  if (threadIdx.x != 0) return;
  const int k = st->k;
  const double hnext = sqrt(v);
  auto Hh = [&](int i, int j) -> double& { return H[(size_t)i * kmax + j]; };
  for (int j = 0; j <= k; ++j) Hh(j, k) = hcol[j];
  Hh(k + 1, k) = hnext;
  for (int j = 0; j < k; ++j) {
    const double t = cs[j] * Hh(j, k) + sn[j] * Hh(j + 1, k);
    Hh(j + 1, k) = -sn[j] * Hh(j, k) + cs[j] * Hh(j + 1, k);
    Hh(j, k) = t;
  }
  const double a = Hh(k, k), bb = Hh(k + 1, k);
  const double den = hypot(a, bb);
  if (den > kArnoldiSmall) {
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
  st->kfinal = k + 1;
  st->col = k + 1;
  st->inv = hnext > kArnoldiSmall ? 1.0 / hnext : 0.0;
  st->k = k + 1;
  if (fabs(g[k + 1]) <= st->tol || hnext <= kArnoldiSmall || k + 1 >= st->inner) st->done = 1;
}

// q_{k+1} = w / h_{k+1,k} (skipped once the cycle is done: no later step reads it).
__global__ void __launch_bounds__(kVB) arn_next_kernel(const ArnoldiState* __restrict__ st, const double* __restrict__ w,
                                                       uint64_t n, double* __restrict__ Q) {
  if (st->done) return;
  double* q = Q + (uint64_t)st->col * n;
  const double inv = st->inv;
  for (uint64_t i = blockIdx.x * (uint64_t)kVB + threadIdx.x; i < n; i += (uint64_t)kVBlocks * kVB) q[i] = w[i] * inv;
}

__global__ void arn_init_kernel(ArnoldiState* __restrict__ st, int inner, double tol, double beta, int kmax,
                                double* __restrict__ H, double* __restrict__ g) {
  for (int i = threadIdx.x; i < (kmax + 1) * kmax; i += blockDim.x) H[i] = 0.0;
  for (int i = threadIdx.x; i <= kmax; i += blockDim.x) g[i] = i == 0 ? beta : 0.0;
  if (threadIdx.x == 0) {
    st->k = 0;
    st->inner = inner;
    st->done = inner <= 0;
    st->kfinal = 0;
    st->col = 0;
    st->tol = tol;
    st->inv = 0.0;
  }
}

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


// y = M x (device vectors, legacy stream): one pass over the packed triangle, or, matrix-free,
// every upper-triangle pair evaluated again through the (F, S) pipeline block by block.
nw_status symv(nw_pt2* p, const double* x, double* y) {
  const uint64_t n = p->n, nb = (n + kTile - 1) / kTile;
  NW_CUDA(p->ctx, cudaMemsetAsync(y, 0, sizeof(double) * n, nullptr));
  if (p->m) {
    const uint64_t ntiles = nb * (nb + 1) / 2;
    packed_symv_kernel<<<(unsigned)ntiles, kTile>>>(p->m, n, nb, x, y, nullptr);
    NW_CUDA(p->ctx, cudaGetLastError());
    return NW_OK;
  }
  const uint64_t ntiles = nb * (nb + 1) / 2, per_block = p->blk / kTileSlots;
  for (uint64_t t0 = 0; t0 < ntiles; t0 += per_block) {
    const uint64_t nt = std::min(per_block, ntiles - t0), nslots = nt * kTileSlots;
    tile_pairs_kernel<<<grid_n(nslots), 256>>>(p->dcand, n, nb, t0, nslots, p->pairs);
    nw_status st = nw::eval_pairs(p->ctx, reinterpret_cast<const uint32_t*>(p->pairs), nslots,
                                  reinterpret_cast<double*>(p->fs), nw::EvalMode::kFS, nullptr);
    if (st != NW_OK) return st;
    mf_tile_apply_kernel<<<(unsigned)nt, kTile>>>(p->fs, n, nb, t0, p->e0, x, y);
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
  nw::CtxGuard guard(ctx, nullptr);
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
    upper_pairs_kernel<<<grid_n(count), 256>>>(dcand, n, base, count, pairs);
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
  nw::CtxGuard guard(ctx, nullptr);
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
  // pairs per evaluation block: 2^26 (1.6 GB of pairs and (F, S)) keeps the per-block cost of
  // the sort (counter clear and scan) small next to the evaluation
  constexpr uint64_t kBlock = 1ull << 26;
  const uint64_t nb = (n + kTile - 1) / kTile;
  p->blk = std::min(kBlock, nb * (nb + 1) / 2 * kTileSlots);  // whole tiles
  p->blk = std::max(p->blk, ((n + kTileSlots - 1) / kTileSlots) * kTileSlots);  // it also holds the n diagonal pairs
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
  nw::CtxGuard guard(p->ctx, nullptr);
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
  nw::CtxGuard guard(p->ctx, nullptr);
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
  std::vector<double> H((size_t)(kmax + 1) * kmax), g(kmax + 1);
  auto Hh = [&](int i, int j) -> double& { return H[(size_t)i * kmax + j]; };

  // device-side Arnoldi scratch: the cycle state, per-block partial sums, Gram-Schmidt
  // coefficients, the Hessenberg matrix, rotations and g
  const int ld = kmax + 1;
  const size_t nscr = (size_t)kVBlocks * ld + 4 * (size_t)kVBlocks + 2 * (size_t)ld + (size_t)(kmax + 1) * kmax +
                      2 * (size_t)kmax + (size_t)ld;
  struct ArnoldiRes {
    void* mem = nullptr;
    cudaStream_t q = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~ArnoldiRes() {
      if (exec) cudaGraphExecDestroy(exec);
      if (q) cudaStreamDestroy(q);
      if (mem) cudaFree(mem);
    }
  } ar;
  if (cudaMalloc(&ar.mem, sizeof(ArnoldiState) + sizeof(double) * nscr) != cudaSuccess)
    return pfail(p, NW_ERR_ALLOC, "GMRES Arnoldi scratch");
  // a blocking stream: ordered with the legacy-stream work (products, cuBLAS) around it
  NW_CUDA(ctx, cudaStreamCreate(&ar.q));
  ArnoldiState* dst = static_cast<ArnoldiState*>(ar.mem);
  double* part = reinterpret_cast<double*>(static_cast<char*>(ar.mem) + sizeof(ArnoldiState));
  double* part_a = part + (size_t)kVBlocks * ld;      // 2 per block
  double* part_b = part_a + 2 * (size_t)kVBlocks;     // 2 per block
  double* coef = part_b + 2 * (size_t)kVBlocks;
  double* hcol = coef + ld;
  double* dH = hcol + ld;
  double* dcs = dH + (size_t)(kmax + 1) * kmax;
  double* dsn = dcs + kmax;
  double* dg = dsn + kmax;
  const int* done_flag = reinterpret_cast<const int*>(reinterpret_cast<const char*>(dst) + offsetof(ArnoldiState, done));
  const uint64_t nb = (n + kTile - 1) / kTile;
  // One Arnoldi step: z = P^-1 q_k, w = M^Omega z, two classical Gram-Schmidt passes, |w|, the
  // Givens update and q_{k+1}; every kernel is a no-op once the cycle is done.
  auto enqueue_step = [&](cudaStream_t q) -> nw_status {
    arn_precond_kernel<<<kVBlocks, kVB, 0, q>>>(dst, Q, dinv, s_0a, f_0a, n, z, P.active ? part_a : part_b);
    if (P.active)
      arn_woodbury_kernel<<<kVBlocks, kVB, 0, q>>>(dst, part_a, P.w00, P.w01, P.w10, P.w11, z0, z1, s_0a, f_0a, n, z,
                                                   part_b);
    if (p->m) {
      arn_zero_kernel<<<kVBlocks, kVB, 0, q>>>(dst, n, w);
      packed_symv_kernel<<<(unsigned)(nb * (nb + 1) / 2), kTile, 0, q>>>(p->m, n, nb, z, w, done_flag);
      NW_CUDA(ctx, cudaGetLastError());
    } else {
      // matrix-free: the (F, S) pair pipeline on the legacy stream (the host checks `done`
      // before every step, so this runs only inside a live cycle)
      nw_status st = symv(p, z, w);
      if (st != NW_OK) return st;
    }
    arn_project_kernel<<<kVBlocks, kVB, 0, q>>>(dst, part_b, pr.e0, f_a0, s_a0, Q, n, ld, w, part);
    arn_coef_kernel<<<1, kVB, 0, q>>>(dst, part, ld, 0, coef, hcol);
    arn_orth_kernel<<<kVBlocks, kVB, 0, q>>>(dst, Q, coef, n, ld, 0, w, part);
    arn_coef_kernel<<<1, kVB, 0, q>>>(dst, part, ld, 1, coef, hcol);
    arn_orth_kernel<<<kVBlocks, kVB, 0, q>>>(dst, Q, coef, n, ld, 1, w, part);
    arn_givens_kernel<<<1, kVB, 0, q>>>(dst, part, ld, hcol, kmax, dH, dcs, dsn, dg);
    arn_next_kernel<<<kVBlocks, kVB, 0, q>>>(dst, w, n, Q);
    NW_CUDA(ctx, cudaGetLastError());
    return NW_OK;
  };
  if (p->m) {
    // the packed path's step is one CUDA graph, captured once per solve and replayed per step
    cudaGraph_t graph = nullptr;
    NW_CUDA(ctx, cudaStreamBeginCapture(ar.q, cudaStreamCaptureModeThreadLocal));
    const nw_status cst = enqueue_step(ar.q);
    const cudaError_t ce = cudaStreamEndCapture(ar.q, &graph);
    if (cst != NW_OK) {
      if (graph) cudaGraphDestroy(graph);
      return cst;
    }
    NW_CUDA(ctx, ce);
    const cudaError_t ie = cudaGraphInstantiate(&ar.exec, graph, 0);
    cudaGraphDestroy(graph);
    NW_CUDA(ctx, ie);
  }
  while (!converged && total < opts->max_iter) {
    PT_BLAS(p, cublasDnrm2(h, (int)n, r, 1, &beta));
    if (beta <= kSmall) {
      res = beta / rms;
      break;
    }
    // the Krylov dimension cannot exceed n
    const int inner = (int)std::min<uint64_t>(std::min(kmax, opts->max_iter - total), n);
    const double inv = 1.0 / beta;
    NW_CUDA(ctx, cudaMemcpy(Q, r, vb, cudaMemcpyDeviceToDevice));
    PT_BLAS(p, cublasDscal(h, (int)n, &inv, Q, 1));
    arn_init_kernel<<<1, kVB, 0, ar.q>>>(dst, inner, opts->res_tol * rms, beta, kmax, dH, dg);
    NW_CUDA(ctx, cudaGetLastError());
    if (ar.exec) {
      // every step of the cycle queued at once; the steps after the stopping point are no-ops
      for (int k = 0; k < inner; ++k) NW_CUDA(ctx, cudaGraphLaunch(ar.exec, ar.q));
    } else {
      for (int k = 0; k < inner; ++k) {
        nw_status st = enqueue_step(ar.q);
        if (st != NW_OK) return st;
        int done = 0;
        NW_CUDA(ctx, cudaMemcpyAsync(&done, done_flag, sizeof(int), cudaMemcpyDeviceToHost, ar.q));
        NW_CUDA(ctx, cudaStreamSynchronize(ar.q));
        if (done) break;
      }
    }
    NW_CUDA(ctx, cudaStreamSynchronize(ar.q));
    ArnoldiState hst;
    NW_CUDA(ctx, cudaMemcpy(&hst, dst, sizeof(hst), cudaMemcpyDeviceToHost));
    const int kfinal = hst.kfinal;
    NW_CUDA(ctx, cudaMemcpy(H.data(), dH, sizeof(double) * H.size(), cudaMemcpyDeviceToHost));
    NW_CUDA(ctx, cudaMemcpy(g.data(), dg, sizeof(double) * g.size(), cudaMemcpyDeviceToHost));
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
