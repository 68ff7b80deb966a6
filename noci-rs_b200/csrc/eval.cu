// Batched (H, S) evaluation of determinant pairs on the B200.
//
// Pipeline for one request batch (all on one stream, no host synchronisation):
//   1. classify: read each pair's two 16-bit determinant descriptors (the full 32-byte records
//      only for same-parent pairs, which get exact zeros when more than a double excitation
//      apart, noci-rs hs.rs:96-101), key every other pair by (contraction-rank class, ket
//      reference, bra determinant) -- pair_sort_key -- and take its rank within the key from a
//      global per-key counter;
//   2. scan the per-key counts (two passes over tiles);
//   3. scatter each pair's request index to offsets[key] + rank;
//   4. evaluate: one thread per pair; a warp sees one (L_alpha, L_beta) class, mostly one bra
//      determinant, so the fused m = 0 evaluator runs divergence-free with its contraction
//      determinant, cofactors and gathered intermediates in registers, and the lanes share the
//      bra's rows of the gathered tables.  Reference pairs with zero-overlap orbitals (m > 0)
//      are evaluated by a separate kernel over the tail of the sorted order, keyed by
//      (reference pair, L_alpha, L_beta), whose warps take 32-pair chunks from a counter.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.cuh"
#include "sort.cuh"
#include "wick_math.cuh"

namespace nw {
namespace {

// Items per thread and loop trip in the sort kernels: independent loads and atomics of
// kSortUnroll pairs are in flight together (the chains are latency-bound otherwise).
constexpr int kSortUnroll = 4;

__global__ void __launch_bounds__(256) classify_kernel(EvalParams P, const uint32_t* __restrict__ pairs,
                                                       uint64_t npairs, const uint32_t* __restrict__ npairs_dev,
                                                       uint32_t* __restrict__ keys, uint32_t* __restrict__ ranks,
                                                       uint32_t* __restrict__ counts, double* __restrict__ out,
                                                       int out_stride, uint32_t* __restrict__ flag) {
  if (npairs_dev) npairs = min(npairs, (uint64_t)*npairs_dev);
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const uint32_t lanes_below = (1u << lane) - 1u;
  // The trip count depends only on the warp's first index, so every lane of a warp runs every
  // iteration and the full-mask warp intrinsics below are well defined.
  const uint64_t warp0 = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u);
  for (uint64_t w0 = warp0; w0 < npairs; w0 += kSortUnroll * nthreads) {
    const uint64_t i0 = w0 + lane;
    uint2 ab[kSortUnroll];
    uint32_t key[kSortUnroll], rk[kSortUnroll];
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) {
      const uint64_t i = i0 + u * nthreads;
      ab[u] = i < npairs ? __ldg(reinterpret_cast<const uint2*>(pairs) + i) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) {
      const uint64_t i = i0 + u * nthreads;
      key[u] = i < npairs ? classify_one(P, ab[u], i, out, out_stride, flag) : kSkipKey;
    }
    // Ranks inside each key's bucket: lanes holding the same key take consecutive ranks from
    // one atomic of their leader (attempts of one QMC parent share keys, so per-lane atomics
    // would serialise on a single counter).
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) {
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key[u]);
      const int leader = __ffs(peers) - 1;
      uint32_t base = 0u;
      if (lane == leader && key[u] != kSkipKey) base = atomicAdd(&counts[key[u]], (uint32_t)__popc(peers));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      rk[u] = key[u] != kSkipKey ? base + (uint32_t)__popc(peers & lanes_below) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) {
      const uint64_t i = i0 + u * nthreads;
      if (i < npairs) {
        keys[i] = key[u];
        ranks[i] = rk[u];
      }
    }
  }
}

// Exclusive scan of counts[0..n) into offsets[0..n] (offsets[n] = total), in two passes over
// tiles of kScanTile counters: tile sums, then each tile's scan from its base, the sum of the
// earlier tiles' sums that the tile's block adds up itself (at most a few thousand tiles).
constexpr int kScanThreads = 256;
constexpr int kScanTile = kScanThreads * 16;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, d);
      if (lane >= d) t += y;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = t;
    if (lane == kScanThreads / 32 - 1) *total = t;
  }
  __syncthreads();
  const uint32_t excl = x - v + (wid > 0 ? warp_tot[wid - 1] : 0u);
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(const uint32_t* __restrict__ counts, uint32_t n,
                                                                   uint32_t* __restrict__ tsum) {
  __shared__ uint32_t red[kScanThreads / 32];
  const uint32_t base = blockIdx.x * (uint32_t)kScanTile;
  uint32_t s = 0;
  for (int r = 0; r < kScanTile / kScanThreads; ++r) {
    const uint32_t k = base + r * kScanThreads + threadIdx.x;
    if (k < n) s += counts[k];
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += red[w];
    tsum[blockIdx.x] = t;
  }
}

// Each thread owns kScanPer consecutive counters of the tile, so the tile takes one block-wide
// scan (a round of block scans per kScanThreads counters left every launch as long as 16
// dependent block barriers).  Full 16-counter runs of 16-byte-aligned buffers move as uint4.
constexpr int kScanPer = kScanTile / kScanThreads;
static_assert(kScanPer == 16, "four uint4 per thread");

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const uint32_t* __restrict__ counts, uint32_t n,
                                                                  const uint32_t* __restrict__ tsum,
                                                                  uint32_t* __restrict__ offsets) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  __shared__ uint32_t total;
  const uint32_t k0 = blockIdx.x * (uint32_t)kScanTile + threadIdx.x * (uint32_t)kScanPer;
  const bool vec = (uint64_t)k0 + kScanPer <= n &&
                   ((reinterpret_cast<uintptr_t>(counts) | reinterpret_cast<uintptr_t>(offsets)) & 15) == 0;
  uint32_t v[kScanPer];
  if (vec) {
#pragma unroll
    for (int q = 0; q < kScanPer / 4; ++q) {
      const uint4 c = __ldg(reinterpret_cast<const uint4*>(counts + k0) + q);
      v[4 * q] = c.x;
      v[4 * q + 1] = c.y;
      v[4 * q + 2] = c.z;
      v[4 * q + 3] = c.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) v[j] = (uint64_t)k0 + j < n ? counts[k0 + j] : 0u;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < kScanPer; ++j) sum += v[j];
  // base of the tile: the sums of tiles 0 .. blockIdx.x - 1
  uint32_t part = 0;
  for (uint32_t t = threadIdx.x; t < blockIdx.x; t += kScanThreads) part += tsum[t];
  block_exclusive_scan(part, warp_tot, &total);
  const uint32_t base = total;  // read before the next scan rewrites it (behind its first barrier)
  uint32_t run = base + block_exclusive_scan(sum, warp_tot, &total);
  if (vec) {
#pragma unroll
    for (int q = 0; q < kScanPer / 4; ++q) {
      uint4 o;
      o.x = run;
      run += v[4 * q];
      o.y = run;
      run += v[4 * q + 1];
      o.z = run;
      run += v[4 * q + 2];
      o.w = run;
      run += v[4 * q + 3];
      reinterpret_cast<uint4*>(offsets + k0)[q] = o;
    }
  } else {
#pragma unroll
    for (int j = 0; j < kScanPer; ++j) {
      if ((uint64_t)k0 + j <= n) offsets[k0 + j] = run;  // offsets[n] = total of all counters
      run += v[j];
    }
  }
}

// Scatter each pair's position in the request to offsets[key] + rank (the evaluators read the
// pair itself through that index: one random 4-byte write here instead of 12).
__global__ void __launch_bounds__(256) scatter_kernel(const uint32_t* __restrict__ keys,
                                                      const uint32_t* __restrict__ ranks, uint64_t npairs,
                                                      const uint32_t* __restrict__ npairs_dev,
                                                      const uint32_t* __restrict__ offsets,
                                                      uint32_t* __restrict__ sidx) {
  if (npairs_dev) npairs = min(npairs, (uint64_t)*npairs_dev);
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i0 < npairs; i0 += kSortUnroll * nthreads) {
    uint32_t k[kSortUnroll], r[kSortUnroll], o[kSortUnroll];
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) {
      const uint64_t i = i0 + u * nthreads;
      k[u] = i < npairs ? keys[i] : kSkipKey;
      r[u] = i < npairs ? ranks[i] : 0u;
    }
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u) o[u] = k[u] != kSkipKey ? __ldg(offsets + k[u]) : 0u;
#pragma unroll
    for (int u = 0; u < kSortUnroll; ++u)
      if (k[u] != kSkipKey) sidx[o[u] + r[u]] = (uint32_t)(i0 + u * nthreads);
  }
}

// One contraction-rank class (L_alpha, L_beta) over its sorted range
// [offsets[c * nbucket], offsets[(c + 1) * nbucket]) of all fast reference pairs.
template <int LA, int LB>
__device__ __forceinline__ void run_class(const EvalParams& P, const uint2* __restrict__ pairs,
                                          const uint32_t* __restrict__ sidx, const uint32_t* __restrict__ offsets,
                                          double* __restrict__ out) {
  constexpr int c = LA * 5 + LB;
  const uint32_t begin = offsets[c * P.nbucket];
  const uint32_t end = offsets[(c + 1) * P.nbucket];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint32_t i = sidx[t];
    const uint2 ab = __ldg(pairs + i);
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const FastPair fp = P.fast[(int)x.parent * P.nref + (int)w.parent];
    double h, s;
    eval_m0_ct<LA, LB>(fp, x, w, P.n, P.nocc_a, P.nocc_b, P.enuc, &h, &s);
    store_hs(out, i, h, s);
  }
}

// The 25 fixed-rank classes in three kernels grouped by register demand, so the dominant
// small-rank classes keep a small register footprint (high occupancy) and the rare
// quadruple-rank classes do not force it up.
__global__ void __launch_bounds__(256) eval_light_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                         const uint32_t* __restrict__ sidx,
                                                         const uint32_t* __restrict__ offsets,
                                                         double* __restrict__ out) {
  run_class<2, 2>(P, pairs, sidx, offsets, out);
  run_class<2, 1>(P, pairs, sidx, offsets, out);
  run_class<1, 2>(P, pairs, sidx, offsets, out);
  run_class<2, 0>(P, pairs, sidx, offsets, out);
  run_class<0, 2>(P, pairs, sidx, offsets, out);
  run_class<1, 1>(P, pairs, sidx, offsets, out);
  run_class<1, 0>(P, pairs, sidx, offsets, out);
  run_class<0, 1>(P, pairs, sidx, offsets, out);
  run_class<0, 0>(P, pairs, sidx, offsets, out);
}

__global__ void __launch_bounds__(256) eval_medium_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                          const uint32_t* __restrict__ sidx,
                                                          const uint32_t* __restrict__ offsets,
                                                          double* __restrict__ out) {
  run_class<3, 1>(P, pairs, sidx, offsets, out);
  run_class<1, 3>(P, pairs, sidx, offsets, out);
  run_class<3, 0>(P, pairs, sidx, offsets, out);
  run_class<0, 3>(P, pairs, sidx, offsets, out);
  run_class<3, 2>(P, pairs, sidx, offsets, out);
  run_class<2, 3>(P, pairs, sidx, offsets, out);
  run_class<3, 3>(P, pairs, sidx, offsets, out);
}

__global__ void __launch_bounds__(256) eval_heavy_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                         const uint32_t* __restrict__ sidx,
                                                         const uint32_t* __restrict__ offsets,
                                                         double* __restrict__ out) {
  run_class<4, 0>(P, pairs, sidx, offsets, out);
  run_class<0, 4>(P, pairs, sidx, offsets, out);
  run_class<4, 1>(P, pairs, sidx, offsets, out);
  run_class<1, 4>(P, pairs, sidx, offsets, out);
  run_class<4, 2>(P, pairs, sidx, offsets, out);
  run_class<2, 4>(P, pairs, sidx, offsets, out);
  run_class<4, 3>(P, pairs, sidx, offsets, out);
  run_class<3, 4>(P, pairs, sidx, offsets, out);
  run_class<4, 4>(P, pairs, sidx, offsets, out);
}

// Contraction ranks above 4 in either spin (class 25), runtime-size arithmetic.
__global__ void __launch_bounds__(128) eval_rt_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                      const uint32_t* __restrict__ sidx,
                                                      const uint32_t* __restrict__ offsets,
                                                      double* __restrict__ out) {
  const uint32_t begin = offsets[25 * P.nbucket];
  const uint32_t end = offsets[26 * P.nbucket];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint32_t i = sidx[t];
    const uint2 ab = __ldg(pairs + i);
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const FastPair fp = P.fast[(int)x.parent * P.nref + (int)w.parent];
    double h, s;
    eval_m0_rt(fp, x, w, P.n, P.nocc_a, P.nocc_b, P.enuc, &h, &s);
    store_hs(out, i, h, s);
  }
}

// ---------------------------------------------------------------------------------------
// m > 0 reference pairs.
// ---------------------------------------------------------------------------------------
__device__ __noinline__ void eval_gen_one(const GenPair& g, const DetRec& x, const DetRec& w, const EvalParams& P,
                                          double* H, double* S) {
  eval_gen_any(g, x, w, P.n, P.nocc_a, P.nocc_b, P.enuc, P.tol, P.exact != 0, H, S);
}

// Work distribution of the m > 0 evaluators: each warp takes the next 32 key-sorted pairs from a
// counter (cleared before the launch).  The classes of one reference pair lie in one key range
// in the same order for every reference pair, so with a static grid stride a thread would meet
// the same (L_alpha, L_beta) class on every pass and the threads of the costly classes would
// set the kernel's length while most SMs idle.  Needs every lane of the warp (blockDim % 32 == 0).
template <typename F>
__device__ __forceinline__ void for_each_gen_pair(uint32_t begin, uint32_t end, uint32_t* work, F&& f) {
  const int lane = threadIdx.x & 31;
  const uint32_t nchunk = (end - begin + 31) / 32;
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(work, 1u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= nchunk) break;
    // chunks are handed out from the end of the range: within each reference pair the classes
    // are keyed in increasing (L_alpha, L_beta), so the costliest chunks go first and the last
    // ones, which set the kernel's tail, are the cheapest
    const uint32_t t = begin + (nchunk - 1 - c) * 32 + lane;
    if (t < end) f(t);
  }
}

__global__ void __launch_bounds__(128) eval_gen_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                       const uint32_t* __restrict__ sidx,
                                                       const uint32_t* __restrict__ offsets, int nkeys,
                                                       double* __restrict__ out, uint32_t* __restrict__ work) {
  for_each_gen_pair(offsets[kClasses * P.nbucket], offsets[nkeys], work, [&](uint32_t t) {
    const uint32_t i = sidx[t];
    const uint2 ab = __ldg(pairs + i);
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const GenPair& g = P.gen[(int)x.parent * P.nref + (int)w.parent];
    double h, s;
    eval_gen_one(g, x, w, P, &h, &s);
    store_hs(out, i, h, s);
  });
}

// ---------------------------------------------------------------------------------------
// Fock one-body element with the overlap, (F, S) per pair, over the same sorted order.
// ---------------------------------------------------------------------------------------
template <int LA, int LB>
__device__ __forceinline__ void run_fs_class(const EvalParams& P, const uint2* __restrict__ pairs,
                                             const uint32_t* __restrict__ sidx, const uint32_t* __restrict__ offsets,
                                             double* __restrict__ out) {
  constexpr int c = LA * 5 + LB;
  const uint32_t begin = offsets[c * P.nbucket];
  const uint32_t end = offsets[(c + 1) * P.nbucket];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint32_t i = sidx[t];
    const uint2 ab = __ldg(pairs + i);
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const int p = (int)x.parent * P.nref + (int)w.parent;
    double f, s;
    if constexpr (c == 25)
      eval_fs_m0_rt(P.fast[p], P.fock[p], x, w, P.n, P.nocc_a, P.nocc_b, &f, &s);
    else
      eval_fs_m0_ct<LA, LB>(P.fast[p], P.fock[p], x, w, P.n, P.nocc_a, P.nocc_b, &f, &s);
    store_hs(out, i, f, s);
  }
}

__global__ void __launch_bounds__(256) eval_fs_light_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                            const uint32_t* __restrict__ sidx,
                                                            const uint32_t* __restrict__ offsets,
                                                            double* __restrict__ out) {
  run_fs_class<2, 2>(P, pairs, sidx, offsets, out);
  run_fs_class<2, 1>(P, pairs, sidx, offsets, out);
  run_fs_class<1, 2>(P, pairs, sidx, offsets, out);
  run_fs_class<2, 0>(P, pairs, sidx, offsets, out);
  run_fs_class<0, 2>(P, pairs, sidx, offsets, out);
  run_fs_class<1, 1>(P, pairs, sidx, offsets, out);
  run_fs_class<1, 0>(P, pairs, sidx, offsets, out);
  run_fs_class<0, 1>(P, pairs, sidx, offsets, out);
  run_fs_class<0, 0>(P, pairs, sidx, offsets, out);
}

__global__ void __launch_bounds__(256) eval_fs_heavy_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                            const uint32_t* __restrict__ sidx,
                                                            const uint32_t* __restrict__ offsets,
                                                            double* __restrict__ out) {
  run_fs_class<3, 1>(P, pairs, sidx, offsets, out);
  run_fs_class<1, 3>(P, pairs, sidx, offsets, out);
  run_fs_class<3, 0>(P, pairs, sidx, offsets, out);
  run_fs_class<0, 3>(P, pairs, sidx, offsets, out);
  run_fs_class<3, 2>(P, pairs, sidx, offsets, out);
  run_fs_class<2, 3>(P, pairs, sidx, offsets, out);
  run_fs_class<3, 3>(P, pairs, sidx, offsets, out);
  run_fs_class<4, 0>(P, pairs, sidx, offsets, out);
  run_fs_class<0, 4>(P, pairs, sidx, offsets, out);
  run_fs_class<4, 1>(P, pairs, sidx, offsets, out);
  run_fs_class<1, 4>(P, pairs, sidx, offsets, out);
  run_fs_class<4, 2>(P, pairs, sidx, offsets, out);
  run_fs_class<2, 4>(P, pairs, sidx, offsets, out);
  run_fs_class<4, 3>(P, pairs, sidx, offsets, out);
  run_fs_class<3, 4>(P, pairs, sidx, offsets, out);
  run_fs_class<4, 4>(P, pairs, sidx, offsets, out);
  run_fs_class<5, 0>(P, pairs, sidx, offsets, out);  // class 25: runtime ranks
}

__device__ __noinline__ void eval_fs_gen_one(const GenPair& g, const FockPair& fk, const DetRec& x, const DetRec& w,
                                             const EvalParams& P, double* F, double* S) {
  eval_fs_gen_any(g, fk, x, w, P.n, P.nocc_a, P.nocc_b, P.tol, P.exact != 0, F, S);
}

__global__ void __launch_bounds__(128) eval_fs_gen_kernel(EvalParams P, const uint2* __restrict__ pairs,
                                                          const uint32_t* __restrict__ sidx,
                                                          const uint32_t* __restrict__ offsets, int nkeys,
                                                          double* __restrict__ out, uint32_t* __restrict__ work) {
  for_each_gen_pair(offsets[kClasses * P.nbucket], offsets[nkeys], work, [&](uint32_t t) {
    const uint32_t i = sidx[t];
    const uint2 ab = __ldg(pairs + i);
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const int p = (int)x.parent * P.nref + (int)w.parent;
    double f, s;
    eval_fs_gen_one(P.gen[p], P.fock[p], x, w, P, &f, &s);
    store_hs(out, i, f, s);
  });
}

// ---------------------------------------------------------------------------------------
// Overlap only (no sorting: one cheap determinant per spin).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) eval_s_kernel(EvalParams P, const uint32_t* __restrict__ pairs,
                                                     uint64_t npairs, double* __restrict__ out,
                                                     uint32_t* __restrict__ flag) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npairs; i += stride) {
    const uint2 ab = __ldg(reinterpret_cast<const uint2*>(pairs) + i);
    if (ab.x >= P.ndet || ab.y >= P.ndet) {
      atomicOr(flag, 1u);
      out[i] = __longlong_as_double(0x7FF8000000000000ll);
      continue;
    }
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    if (far_same_parent(x, w)) {
      out[i] = 0.0;
      continue;
    }
    const int p = (int)x.parent * P.nref + (int)w.parent;
    const int ord = __ldg(P.order + p);
    if (ord < 0) continue;  // reference pair outside the resident block
    const bool fast = ord < P.nfast;
    out[i] = eval_s_pair(fast ? P.fast + p : nullptr, fast ? nullptr : P.gen + p, x, w, P.n, P.nocc_a, P.nocc_b);
  }
}

inline int grid_stride_blocks(uint64_t work, int block, int per_sm) {
  uint64_t g = (work + block - 1) / block;
  const uint64_t cap = 148ull * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

EvalParams make_params(const nw_ctx* ctx) {
  EvalParams P;
  P.dets = ctx->d_dets;
  P.ndet = ctx->ndet;
  P.fast = ctx->d_fast;
  P.gen = ctx->d_gen;
  P.order = ctx->d_order;
  P.nref = ctx->nref;
  P.n = ctx->nmo;
  P.nocc_a = ctx->nocc_a;
  P.nocc_b = ctx->nocc_b;
  P.nfast = ctx->nfast;
  P.exact = ctx->convention == NW_CONVENTION_EXACT ? 1 : 0;
  P.enuc = ctx->enuc;
  P.tol = ctx->tol;
  P.desc = ctx->d_desc;
  P.fock = ctx->d_fockp;
  P.nbucket = 1;
  P.shift = 0;
  return P;
}


// Fine-key budget: at most kFineMax counters, and at most about one per pair of the request so
// the counter memset and scan stay small next to the evaluation.

// Number of sort keys for this request with at most `cap` counters for the fast classes;
// fills P.nbucket / P.shift.
uint64_t plan_keys(const nw_ctx* ctx, EvalParams& P, uint64_t cap) {
  uint32_t nb = 1;
  P.shift = sort_key_shift(P.ndet, ctx->nref, cap, &nb);
  P.nbucket = nb;
  const uint64_t ngen = (uint64_t)ctx->nresident - (uint64_t)ctx->nfast;
  return (uint64_t)kClasses * nb + (uint64_t)kGenClasses * ngen;
}

nw_status scan_exclusive(nw_ctx* ctx, const uint32_t* counts, uint64_t n, uint32_t* offsets, uint32_t* tsum,
                         cudaStream_t stream) {
  const int ntiles = (int)(n / kScanTile + 1);
  scan_tiles_kernel<<<ntiles, kScanThreads, 0, stream>>>(counts, (uint32_t)n, tsum);
  scan_down_kernel<<<ntiles, kScanThreads, 0, stream>>>(counts, (uint32_t)n, tsum, offsets);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

// classify -> scan -> scatter -> evaluate, all on `stream`.  The flag must already be cleared
// (or hold earlier calls' reports); ev (eight events or null) brackets the phases: ev[0..5] on
// `stream`, ev[6] / ev[7] around the m > 0 evaluator on its forked stream.
nw_status launch_sorted(nw_ctx* ctx, const EvalParams& P, uint64_t nkeys, const uint32_t* pairs, uint64_t npairs,
                        double* out, const SortScratch& S, cudaStream_t stream, cudaEvent_t* ev, EvalMode mode,
                        const uint32_t* npairs_dev, bool classified) {
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[0], stream));
  const int per_sm = ctx->tune_per_sm > 0 ? ctx->tune_per_sm : 8;
  if (!classified) {
    NW_CUDA(ctx, cudaMemsetAsync(S.counts, 0, sizeof(uint32_t) * nkeys, stream));
    classify_kernel<<<grid_stride_blocks(npairs, 256, per_sm), 256, 0, stream>>>(P, pairs, npairs, npairs_dev, S.keys,
                                                                                 S.ranks, S.counts, out, 2, S.flag);
    NW_CUDA(ctx, cudaGetLastError());
  }
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[1], stream));
  const int ntiles = (int)(nkeys / kScanTile + 1);
  scan_tiles_kernel<<<ntiles, kScanThreads, 0, stream>>>(S.counts, (uint32_t)nkeys, S.tsum);
  scan_down_kernel<<<ntiles, kScanThreads, 0, stream>>>(S.counts, (uint32_t)nkeys, S.tsum, S.offsets);
  NW_CUDA(ctx, cudaGetLastError());
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[2], stream));
  scatter_kernel<<<grid_stride_blocks(npairs, 256, per_sm), 256, 0, stream>>>(S.keys, S.ranks, npairs, npairs_dev,
                                                                         S.offsets, S.sidx);
  NW_CUDA(ctx, cudaGetLastError());
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[3], stream));
  const uint2* pp = reinterpret_cast<const uint2*>(pairs);
  // The class kernels write disjoint outputs and each is limited by its own occupancy, so the
  // medium, the heavy / runtime-rank and the zero-overlap generic classes run on streams forked
  // off the launching one, beside the light classes, and join before the call returns (also
  // inside a stream capture: the forked streams join the capture through the fork event).
  const bool fast = ctx->nfast > 0, gen = ctx->nfast < ctx->nresident;
  // Serial per-class timing (a profiling mode, timing enabled): every class kernel on the
  // launching stream, in the order light, medium, heavy, runtime rank, generic, each between two
  // events; the kernels and their work are the same, only their overlap is given up.
  const bool serial = ev != nullptr && ctx->serial_classes;
  cudaStream_t sq[4] = {stream, ctx->s_aux[0], ctx->s_aux[1], ctx->s_aux[2]};
  if (serial) {
    for (int i = 1; i < 4; ++i) sq[i] = stream;
    NW_CUDA(ctx, cudaEventRecord(ctx->evc[0], stream));
  } else {
    NW_CUDA(ctx, cudaEventRecord(ctx->ev_fork, stream));
    for (int i = 0; i < 3; ++i) NW_CUDA(ctx, cudaStreamWaitEvent(ctx->s_aux[i], ctx->ev_fork, 0));
  }
  auto mark = [&](int i) -> cudaError_t { return serial ? cudaEventRecord(ctx->evc[i], stream) : cudaSuccess; };
  if (fast) {
    if (mode == EvalMode::kFS) {
      eval_fs_light_kernel<<<grid_stride_blocks(npairs, 256, per_sm), 256, 0, sq[0]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(1));
      NW_CUDA(ctx, mark(2));
      eval_fs_heavy_kernel<<<148 * 2, 256, 0, sq[1]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(3));
      NW_CUDA(ctx, mark(4));
    } else {
      eval_light_kernel<<<grid_stride_blocks(npairs, 256, per_sm), 256, 0, sq[0]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(1));
      eval_medium_kernel<<<148 * 2, 256, 0, sq[1]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(2));
      eval_heavy_kernel<<<148, 256, 0, sq[2]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(3));
      eval_rt_kernel<<<148 * 2, 128, 0, sq[2]>>>(P, pp, S.sidx, S.offsets, out);
      NW_CUDA(ctx, mark(4));
    }
    NW_CUDA(ctx, cudaGetLastError());
  } else {
    for (int i = 1; i <= 4; ++i) NW_CUDA(ctx, mark(i));
  }
  if (gen) {
    NW_CUDA(ctx, cudaMemsetAsync(S.work, 0, sizeof(uint32_t), sq[3]));
    if (ev && !serial) NW_CUDA(ctx, cudaEventRecord(ev[6], sq[3]));
    if (mode == EvalMode::kFS)
      eval_fs_gen_kernel<<<148 * 4, 128, 0, sq[3]>>>(P, pp, S.sidx, S.offsets, (int)nkeys, out, S.work);
    else
      eval_gen_kernel<<<148 * 4, 128, 0, sq[3]>>>(P, pp, S.sidx, S.offsets, (int)nkeys, out, S.work);
    NW_CUDA(ctx, cudaGetLastError());
    if (ev && !serial) NW_CUDA(ctx, cudaEventRecord(ev[7], sq[3]));
  }
  NW_CUDA(ctx, mark(5));
  if (ev) {
    ctx->timed_gen = gen && !serial;
    ctx->timed_classes = serial;
  }
  if (!serial)
    for (int i = 0; i < 3; ++i) {
      NW_CUDA(ctx, cudaEventRecord(ctx->ev_join[i], ctx->s_aux[i]));
      NW_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->ev_join[i], 0));
    }
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[4], stream));
  if (ev) NW_CUDA(ctx, cudaEventRecord(ev[5], stream));
  return NW_OK;
}


nw_status eval_pairs(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* out, EvalMode mode,
                     cudaStream_t stream, bool clear_flag) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (!ctx->d_dets) return fail(ctx, NW_ERR_STATE, "no determinant basis set");
  return eval_pairs_on(ctx, make_params(ctx), pairs, npairs, out, mode, stream, clear_flag);
}

// Blocked evaluation for systems whose intermediates exceed the device memory: a build of no
// slab (the pairing, every per-pair scalar and the zero-overlap counts) sizes each ordered
// reference pair's slab pieces; the pairs are cut, in index order, into blocks whose slab fits
// `budget` bytes (0: the free device memory less 8 GB for the evaluation and the build
// workspace); each block is built and the whole request evaluated against it, every block
// writing the elements of its own reference pairs (the others are skipped by classify).  The
// results equal those of one full build bit for bit: every block computes its pairs'
// intermediates with the same products.  The context keeps the last block afterwards
// (`partial`): other evaluations refuse it until nw_build_intermediates.
nw_status eval_blocked(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* hs, uint64_t budget,
                       cudaStream_t stream, uint32_t* nblocks) {
  if (nblocks) *nblocks = 0;
  if (!ctx->d_dets) return fail(ctx, NW_ERR_STATE, "no determinant basis set");
  const int npair = ctx->nref * ctx->nref, n = ctx->nmo;
  if (budget == 0) {
    size_t fr = 0, tot = 0;
    NW_CUDA(ctx, cudaMemGetInfo(&fr, &tot));
    const size_t reserve = 8ull << 30;
    budget = fr > reserve ? fr - reserve : 0;
    if (ctx->d_slab) budget += ctx->slab_capacity;  // the current slab is reused or freed
  }
  std::vector<char> none(npair, 0);
  nw_status st = build_all(ctx, &none);
  if (st != NW_OK) return st;
  std::vector<size_t> bytes(npair);
  for (int p = 0; p < npair; ++p) {
    bytes[p] = pair_slab_doubles(n, ctx->m_counts[2 * p], ctx->m_counts[2 * p + 1]) * sizeof(double);
    if (bytes[p] > budget)
      return fail(ctx, NW_ERR_ALLOC, "one reference pair's intermediates exceed the blocked-evaluation budget");
  }
  std::vector<std::vector<char>> blocks;
  {
    std::vector<char> cur(npair, 0);
    size_t used = 0;
    bool any = false;
    for (int p = 0; p < npair; ++p) {
      if (used + bytes[p] > budget && any) {
        blocks.push_back(cur);
        std::fill(cur.begin(), cur.end(), 0);
        used = 0;
        any = false;
      }
      cur[p] = 1;
      used += bytes[p];
      any = true;
    }
    if (any) blocks.push_back(cur);
  }
  for (size_t b = 0; b < blocks.size(); ++b) {
    const bool all = blocks.size() == 1;
    if ((st = build_all(ctx, all ? nullptr : &blocks[b])) != NW_OK) return st;
    ctx->allow_partial = true;
    st = eval_pairs_on(ctx, make_params(ctx), pairs, npairs, hs, EvalMode::kHS, stream, true);
    ctx->allow_partial = false;
    if (st != NW_OK) return st;
    // the flag of out-of-range indices is read once per block: stop at the first report
    NW_CUDA(ctx, cudaMemcpyAsync(ctx->h_flag, ctx->flag.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    NW_CUDA(ctx, cudaStreamSynchronize(stream));
    if (*ctx->h_flag) return fail(ctx, NW_ERR_INVALID, "pair index out of range of the determinant basis");
  }
  if (nblocks) *nblocks = (uint32_t)blocks.size();
  return NW_OK;
}

nw_status eval_pairs_on(nw_ctx* ctx, EvalParams P, const uint32_t* pairs, uint64_t npairs, double* out, EvalMode mode,
                        cudaStream_t stream, bool clear_flag) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (ctx->partial && !ctx->allow_partial)
    return fail(ctx, NW_ERR_STATE, "the intermediates hold one block of a blocked evaluation (rebuild them)");
  if (mode == EvalMode::kFS && !ctx->fock_ready) return fail(ctx, NW_ERR_STATE, "Fock tables not set (nw_update_fock)");
  const bool overlap_only = mode == EvalMode::kS;
  if (npairs == 0) return NW_OK;
  if (npairs >= 0xFFFFFFFFull) return fail(ctx, NW_ERR_UNSUPPORTED, "at most 2^32 - 2 pairs per call");
  if ((reinterpret_cast<uintptr_t>(pairs) & 7) != 0) return fail(ctx, NW_ERR_INVALID, "pairs must be 8-byte aligned");
  if ((reinterpret_cast<uintptr_t>(out) & (overlap_only ? 7 : 15)) != 0)
    return fail(ctx, NW_ERR_INVALID, "output must be 16-byte aligned (8 for overlap only)");

  nw_status st = ensure(ctx, ctx->flag, 256);
  if (st != NW_OK) return st;
  uint32_t* flag = static_cast<uint32_t*>(ctx->flag.p);
  if (clear_flag) NW_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(uint32_t), stream));

  if (overlap_only) {
    eval_s_kernel<<<grid_stride_blocks(npairs, 128, 16), 128, 0, stream>>>(P, pairs, npairs, out, flag);
    NW_CUDA(ctx, cudaGetLastError());
    return NW_OK;
  }

  const uint64_t budget =
      ctx->tune_keys_per_pair > 0.0 ? (uint64_t)(ctx->tune_keys_per_pair * (double)npairs) : std::max(kFineMin, npairs);
  const uint64_t nkeys = plan_keys(ctx, P, std::min(kFineMax, std::max(kFineMin, budget)));
  if ((st = ensure(ctx, ctx->keys, npairs * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->ranks, npairs * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->perm, npairs * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->counts, nkeys * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->offsets, (nkeys + 1) * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->tsum, (nkeys / kScanTile + 1) * sizeof(uint32_t))) != NW_OK) return st;
  SortScratch S;
  S.keys = static_cast<uint32_t*>(ctx->keys.p);
  S.ranks = static_cast<uint32_t*>(ctx->ranks.p);
  S.sidx = static_cast<uint32_t*>(ctx->perm.p);
  S.counts = static_cast<uint32_t*>(ctx->counts.p);
  S.offsets = static_cast<uint32_t*>(ctx->offsets.p);
  S.tsum = static_cast<uint32_t*>(ctx->tsum.p);
  S.flag = flag;
  S.work = flag + 8;
  st = launch_sorted(ctx, P, nkeys, pairs, npairs, out, S, stream, ctx->timing ? ctx->ev : nullptr, mode);
  if (st == NW_OK && ctx->timing) ctx->timed_valid = true;
  return st;
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the pair evaluation (nw_eval_hs_pairs_noalloc).
//
// Some callers cannot allocate device memory when they evaluate pairs: a host that hands
// nearly all of HBM to its own memory pool (a framework's caching allocator, a solver's
// preallocated workspace), or a latency-critical loop that cannot afford cudaMalloc's implicit
// synchronisation or its failure path.  For them the per-call scratch of the evaluation (keys,
// ranks, key-sorted request indices, per-key counts and offsets, error flag)
// lives in the fixed device array below instead of buffers grown with cudaMalloc.
//
// The array is a file-scope __device__ variable, so every GPU that loads this library holds
// it (16,089,856 bytes, 15.3 MiB) until the process exits.  Host code cannot use its name as a
// device address: the address is looked up with cudaGetSymbolAddress once per device, with
// that device current, on the first call of the entry point on that device (that first call
// should therefore come before any stream capture).  Every call shares the array and it keeps
// the last call's contents: the counts and the error flag are cleared at the start of each
// call, and calls whose work overlaps on the GPU (different streams, concurrent host threads)
// race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoallocMaxPairs = 1ull << 20;                       // 1,048,576 pairs per call
constexpr int kNoallocMaxRefs = 64;                                      // reference determinants
// keys: the fast classes get at least kClasses * 64 * 64 counters, the zero-overlap reference
// pairs up to kGenClasses * 64 * 64 more
constexpr uint64_t kNoallocMaxKeys = (uint64_t)kNoallocMaxRefs * kNoallocMaxRefs * (kClasses + kGenClasses);
constexpr uint64_t kNoallocTiles = kNoallocMaxKeys / kScanTile + 1;
constexpr uint64_t kNoallocOffKeys = 0;
constexpr uint64_t kNoallocOffRanks = kNoallocOffKeys + 4 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffIdx = kNoallocOffRanks + 4 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffCounts = kNoallocOffIdx + 4 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffOffsets = kNoallocOffCounts + 4 * kNoallocMaxKeys;
constexpr uint64_t kNoallocOffTsum = kNoallocOffOffsets + 4 * (kNoallocMaxKeys + 1);
constexpr uint64_t kNoallocOffFlag = ((kNoallocOffTsum + 4 * kNoallocTiles + 255) / 256) * 256;
constexpr uint64_t kNoallocBytes = kNoallocOffFlag + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
nw_status noalloc_scratch(nw_ctx* ctx, unsigned char** out) {
  if (ctx->device < 0 || ctx->device >= kNoallocMaxDevices)
    return fail(ctx, NW_ERR_UNSUPPORTED, "device ordinal too large for the allocation-free entry point");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[ctx->device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(ctx, e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[ctx->device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_ptr[ctx->device]);
  return NW_OK;
}

}  // namespace

nw_status eval_pairs_noalloc(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* out, cudaStream_t stream) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (ctx->partial && !ctx->allow_partial)
    return fail(ctx, NW_ERR_STATE, "the intermediates hold one block of a blocked evaluation (rebuild them)");
  if (!ctx->d_dets) return fail(ctx, NW_ERR_STATE, "no determinant basis set");
  if (npairs > kNoallocMaxPairs)
    return fail(ctx, NW_ERR_UNSUPPORTED, "allocation-free evaluation takes at most " +
                                              std::to_string(kNoallocMaxPairs) + " pairs per call");
  if (ctx->nref > kNoallocMaxRefs)
    return fail(ctx, NW_ERR_UNSUPPORTED, "allocation-free evaluation supports at most " +
                                              std::to_string(kNoallocMaxRefs) + " references");
  if ((reinterpret_cast<uintptr_t>(pairs) & 7) != 0) return fail(ctx, NW_ERR_INVALID, "pairs must be 8-byte aligned");
  if ((reinterpret_cast<uintptr_t>(out) & 15) != 0) return fail(ctx, NW_ERR_INVALID, "output must be 16-byte aligned");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  unsigned char* base = nullptr;
  nw_status st = noalloc_scratch(ctx, &base);
  if (st != NW_OK) return st;
  if (npairs == 0) return NW_OK;
  EvalParams P = make_params(ctx);
  const uint64_t ngen = (uint64_t)ctx->nresident - (uint64_t)ctx->nfast;
  // the same fine-key budget as the allocating path (nw_autotune's choice when there is one),
  // clamped to the keys the fixed array holds
  const uint64_t budget =
      ctx->tune_keys_per_pair > 0.0 ? (uint64_t)(ctx->tune_keys_per_pair * (double)npairs) : std::max(kFineMin, npairs);
  const uint64_t fast_cap = std::min(kNoallocMaxKeys - (uint64_t)kGenClasses * ngen,
                                     std::min(kFineMax, std::max(kFineMin, budget)));
  const uint64_t nkeys = plan_keys(ctx, P, fast_cap);
  if (nkeys > kNoallocMaxKeys) return fail(ctx, NW_ERR_UNSUPPORTED, "sort keys exceed the allocation-free scratch");
  SortScratch S;
  S.keys = reinterpret_cast<uint32_t*>(base + kNoallocOffKeys);
  S.ranks = reinterpret_cast<uint32_t*>(base + kNoallocOffRanks);
  S.sidx = reinterpret_cast<uint32_t*>(base + kNoallocOffIdx);
  S.counts = reinterpret_cast<uint32_t*>(base + kNoallocOffCounts);
  S.offsets = reinterpret_cast<uint32_t*>(base + kNoallocOffOffsets);
  S.tsum = reinterpret_cast<uint32_t*>(base + kNoallocOffTsum);
  S.flag = reinterpret_cast<uint32_t*>(base + kNoallocOffFlag);
  S.work = S.flag + 8;
  NW_CUDA(ctx, cudaMemsetAsync(S.flag, 0, sizeof(uint32_t), stream));
  return launch_sorted(ctx, P, nkeys, pairs, npairs, out, S, stream, nullptr);
}

}  // namespace nw

// ---------------------------------------------------------------------------------------
// Autotuner: the fine sort-key budget (how finely pairs are bucketed by bra determinant; kept
// per pair so that it scales with the size of later calls
// before evaluation: locality of the intermediates against the cost of clearing and scanning
// the counters) and the blocks per SM of the grid-stride kernels, timed on the caller's pairs.
// ---------------------------------------------------------------------------------------
extern "C" nw_status nw_autotune(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* hs, void* stream,
                                 nw_tune_report* rep) {
  if (!ctx || !pairs || !hs || !rep || npairs == 0) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, static_cast<cudaStream_t>(stream));
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  static const uint64_t kBudgets[] = {1ull << 14, 1ull << 16, 1ull << 18, 1ull << 20, 1ull << 22, 1ull << 23};
  static const int kPerSm[] = {4, 8, 16};
  const double saved_ratio = ctx->tune_keys_per_pair;
  const int saved_per_sm = ctx->tune_per_sm;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return nw::fail(ctx, NW_ERR_CUDA, "autotune events");
  }
  std::memset(rep, 0, sizeof(*rep));
  float best = 0.0f, dflt = 0.0f;
  uint64_t best_budget = 0;
  int best_per_sm = 0, trials = 0;
  nw_status st = NW_OK;
  // (0, 0) first: the untuned defaults
  for (int b = -1; b < (int)(sizeof(kBudgets) / sizeof(kBudgets[0])) && st == NW_OK; ++b) {
    for (int g = 0; g < (int)(sizeof(kPerSm) / sizeof(kPerSm[0])) && st == NW_OK; ++g) {
      if (b < 0 && g > 0) break;
      ctx->tune_keys_per_pair = b < 0 ? 0.0 : (double)kBudgets[b] / (double)npairs;
      ctx->tune_per_sm = b < 0 ? 0 : kPerSm[g];
      float ms = 0.0f;
      for (int rep_i = 0; rep_i < 4 && st == NW_OK; ++rep_i) {
        if (rep_i == 1 && cudaEventRecord(e0, s) != cudaSuccess) st = NW_ERR_CUDA;
        if (st == NW_OK) st = nw::eval_pairs(ctx, pairs, npairs, hs, nw::EvalMode::kHS, s);
      }
      if (st == NW_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        st = nw::fail(ctx, NW_ERR_CUDA, "autotune timing");
      if (st != NW_OK) break;
      ms /= 3.0f;
      ++trials;
      if (b < 0) dflt = ms;
      if (best_budget == 0 && best_per_sm == 0 && b < 0) best = ms;
      if (b >= 0 && ms < best) {
        best = ms;
        best_budget = kBudgets[b];
        best_per_sm = kPerSm[g];
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != NW_OK) {
    ctx->tune_keys_per_pair = saved_ratio;
    ctx->tune_per_sm = saved_per_sm;
    return st;
  }
  // kept as keys per pair, so later calls of other sizes (e.g. the chunks of the host-buffer
  // pipeline) scale it; 0 / 0 keeps the defaults when they were fastest
  ctx->tune_keys_per_pair = (double)best_budget / (double)npairs;
  ctx->tune_per_sm = best_per_sm;
  rep->key_budget = best_budget;
  rep->blocks_per_sm = best_per_sm;
  rep->trials = trials;
  rep->best_ms = best;
  rep->default_ms = dflt;
  return NW_OK;
}
