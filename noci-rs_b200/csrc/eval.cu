// Batched (H, S) evaluation of determinant pairs on the B200.
//
// Pipeline for one request batch (all on one stream, no host synchronisation):
//   1. classify: read each pair's two 32-byte determinant records, give exact zeros to
//      same-parent pairs more than a double excitation apart (noci-rs hs.rs:96-101), and key
//      every other pair by (ordered reference pair, contraction ranks) in a block-local
//      shared-memory histogram;
//   2. scan the per-key counts (one block);
//   3. scatter pair indices into key order, reserving each block's run with one global atomic
//      per key;
//   4. evaluate: one thread per pair; a warp sees one (reference pair, L_alpha, L_beta) bin,
//      so the fused m = 0 evaluator runs divergence-free with its contraction determinant,
//      cofactors and gathered intermediates in registers.  Reference pairs with zero-overlap
//      orbitals (m > 0) are evaluated by a separate kernel over the tail of the sorted order.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "internal.cuh"
#include "wick_math.cuh"

namespace nw {
namespace {

__device__ __forceinline__ DetRec load_det(const nw_det* dets, uint32_t i) {
  const ulonglong2* p = reinterpret_cast<const ulonglong2*>(dets + i);
  const ulonglong2 lo = __ldg(p);
  const ulonglong2 hi = __ldg(p + 1);
  return unpack_det(lo.x, lo.y, hi.x, hi.y);
}

__device__ __forceinline__ void store_hs(double* out, uint64_t i, double h, double s) {
  reinterpret_cast<double2*>(out)[i] = make_double2(h, s);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Keys of every pair, and per-key counts.  Lanes of a warp holding the same key add their count
// with one atomic (warp-aggregated through __match_any_sync).
template <bool kShared>
__global__ void __launch_bounds__(256) classify_kernel(EvalParams P, const uint32_t* __restrict__ pairs,
                                                       uint64_t npairs, uint32_t* __restrict__ keys,
                                                       uint32_t* __restrict__ counts, int nkeys,
                                                       double* __restrict__ out, int out_stride,
                                                       uint32_t* __restrict__ flag) {
  extern __shared__ uint32_t hist[];
  if (kShared) {
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) hist[k] = 0;
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npairs; i += stride) {
    const uint2 ab = __ldg(reinterpret_cast<const uint2*>(pairs) + i);
    uint32_t key = kSkipKey;
    if (ab.x >= P.ndet || ab.y >= P.ndet) {
      atomicOr(flag, 1u);
      const double nan = __longlong_as_double(0x7FF8000000000000ll);
      if (out_stride == 2)
        store_hs(out, i, nan, nan);
      else
        out[i] = nan;
    } else {
      const DetRec x = load_det(P.dets, ab.x);
      const DetRec w = load_det(P.dets, ab.y);
      if (far_same_parent(x, w)) {
        if (out_stride == 2)
          store_hs(out, i, 0.0, 0.0);
        else
          out[i] = 0.0;
      } else {
        const int p = (int)x.parent * P.nref + (int)w.parent;
        const int ord = __ldg(P.order + p);
        const int cls = rank_class(x.ra + w.ra, x.rb + w.rb);
        // fast pairs: class-major keys [0, kClasses * nfast); m > 0 pairs after them
        key = (uint32_t)(ord < P.nfast ? cls * P.nfast + ord : kClasses * P.nfast + (ord - P.nfast) * kClasses + cls);
      }
    }
    keys[i] = key;
    const unsigned grp = __match_any_sync(__activemask(), key);
    if (key != kSkipKey && lane == __ffs(grp) - 1) {
      if (kShared)
        atomicAdd(&hist[key], (uint32_t)__popc(grp));
      else
        atomicAdd(&counts[key], (uint32_t)__popc(grp));
    }
  }
  if (kShared) {
    __syncthreads();
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x)
      if (hist[k]) atomicAdd(&counts[k], hist[k]);
  }
}

// Exclusive scan of counts into offsets[0..nkeys]; cursor gets a copy for the scatter.
__global__ void scan_kernel(const uint32_t* __restrict__ counts, int nkeys, uint32_t* __restrict__ offsets,
                            uint32_t* __restrict__ cursor) {
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (nkeys + nt - 1) / nt;
  const int k0 = t * per, k1 = min(nkeys, k0 + per);
  uint32_t s = 0;
  for (int k = k0; k < k1; ++k) s += counts[k];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    uint32_t run = 0;
    for (int i = 0; i < nt; ++i) {
      const uint32_t v = part[i];
      part[i] = run;
      run += v;
    }
    offsets[nkeys] = run;
  }
  __syncthreads();
  uint32_t run = part[t];
  for (int k = k0; k < k1; ++k) {
    offsets[k] = run;
    cursor[k] = run;
    run += counts[k];
  }
}

// Scatter each pair (and its position in the request) into key order.  A block owns a
// contiguous chunk: it counts its keys, reserves one run per key with a single global atomic,
// then places each pair at run base + rank (warp-aggregated ranks).
template <bool kShared>
__global__ void __launch_bounds__(256) scatter_kernel(const uint32_t* __restrict__ keys,
                                                      const uint32_t* __restrict__ pairs, uint64_t npairs,
                                                      uint32_t* __restrict__ cursor, int nkeys, uint64_t chunk,
                                                      uint2* __restrict__ spairs, uint32_t* __restrict__ sidx) {
  extern __shared__ uint32_t base[];
  const uint64_t c0 = blockIdx.x * chunk;
  const uint64_t c1 = min(npairs, c0 + chunk);
  if (c0 >= npairs) return;
  const int lane = threadIdx.x & 31;
  uint32_t* slot = kShared ? base : cursor;
  if (kShared) {
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) base[k] = 0;
    __syncthreads();
    for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
      const uint32_t k = keys[i];
      const unsigned grp = __match_any_sync(__activemask(), k);
      if (k != kSkipKey && lane == __ffs(grp) - 1) atomicAdd(&base[k], (uint32_t)__popc(grp));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nkeys; k += blockDim.x) {
      const uint32_t c = base[k];
      base[k] = c ? atomicAdd(&cursor[k], c) : 0u;
    }
    __syncthreads();
  }
  for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    const uint32_t k = keys[i];
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, k);
    const int leader = __ffs(grp) - 1;
    uint32_t b = 0;
    if (k != kSkipKey && lane == leader) b = atomicAdd(&slot[k], (uint32_t)__popc(grp));
    b = __shfl_sync(grp, b, leader);
    if (k != kSkipKey) {
      const uint32_t pos = b + (uint32_t)__popc(grp & lanemask_lt());
      spairs[pos] = __ldg(reinterpret_cast<const uint2*>(pairs) + i);
      sidx[pos] = (uint32_t)i;
    }
  }
}

// One contraction-rank class (L_alpha, L_beta) over its sorted range
// [offsets[c * nfast], offsets[(c + 1) * nfast]) of all fast reference pairs.
template <int LA, int LB>
__device__ __forceinline__ void run_class(const EvalParams& P, const uint2* __restrict__ spairs,
                                          const uint32_t* __restrict__ sidx, const uint32_t* __restrict__ offsets,
                                          double* __restrict__ out) {
  constexpr int c = LA * 5 + LB;
  const uint32_t begin = offsets[c * P.nfast];
  const uint32_t end = offsets[(c + 1) * P.nfast];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint2 ab = spairs[t];
    const uint32_t i = sidx[t];
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
__global__ void __launch_bounds__(256) eval_light_kernel(EvalParams P, const uint2* __restrict__ spairs,
                                                         const uint32_t* __restrict__ sidx,
                                                         const uint32_t* __restrict__ offsets,
                                                         double* __restrict__ out) {
  run_class<2, 2>(P, spairs, sidx, offsets, out);
  run_class<2, 1>(P, spairs, sidx, offsets, out);
  run_class<1, 2>(P, spairs, sidx, offsets, out);
  run_class<2, 0>(P, spairs, sidx, offsets, out);
  run_class<0, 2>(P, spairs, sidx, offsets, out);
  run_class<1, 1>(P, spairs, sidx, offsets, out);
  run_class<1, 0>(P, spairs, sidx, offsets, out);
  run_class<0, 1>(P, spairs, sidx, offsets, out);
  run_class<0, 0>(P, spairs, sidx, offsets, out);
}

__global__ void __launch_bounds__(256) eval_medium_kernel(EvalParams P, const uint2* __restrict__ spairs,
                                                          const uint32_t* __restrict__ sidx,
                                                          const uint32_t* __restrict__ offsets,
                                                          double* __restrict__ out) {
  run_class<3, 1>(P, spairs, sidx, offsets, out);
  run_class<1, 3>(P, spairs, sidx, offsets, out);
  run_class<3, 0>(P, spairs, sidx, offsets, out);
  run_class<0, 3>(P, spairs, sidx, offsets, out);
  run_class<3, 2>(P, spairs, sidx, offsets, out);
  run_class<2, 3>(P, spairs, sidx, offsets, out);
  run_class<3, 3>(P, spairs, sidx, offsets, out);
}

__global__ void __launch_bounds__(256) eval_heavy_kernel(EvalParams P, const uint2* __restrict__ spairs,
                                                         const uint32_t* __restrict__ sidx,
                                                         const uint32_t* __restrict__ offsets,
                                                         double* __restrict__ out) {
  run_class<4, 0>(P, spairs, sidx, offsets, out);
  run_class<0, 4>(P, spairs, sidx, offsets, out);
  run_class<4, 1>(P, spairs, sidx, offsets, out);
  run_class<1, 4>(P, spairs, sidx, offsets, out);
  run_class<4, 2>(P, spairs, sidx, offsets, out);
  run_class<2, 4>(P, spairs, sidx, offsets, out);
  run_class<4, 3>(P, spairs, sidx, offsets, out);
  run_class<3, 4>(P, spairs, sidx, offsets, out);
  run_class<4, 4>(P, spairs, sidx, offsets, out);
}

// Contraction ranks above 4 in either spin (class 25), runtime-size arithmetic.
__global__ void __launch_bounds__(128) eval_rt_kernel(EvalParams P, const uint2* __restrict__ spairs,
                                                      const uint32_t* __restrict__ sidx,
                                                      const uint32_t* __restrict__ offsets,
                                                      double* __restrict__ out) {
  const uint32_t begin = offsets[25 * P.nfast];
  const uint32_t end = offsets[26 * P.nfast];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint2 ab = spairs[t];
    const uint32_t i = sidx[t];
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
  eval_gen_pair(g, x, w, P.n, P.nocc_a, P.nocc_b, P.enuc, P.tol, P.exact != 0, H, S);
}

__global__ void __launch_bounds__(128) eval_gen_kernel(EvalParams P, const uint2* __restrict__ spairs,
                                                       const uint32_t* __restrict__ sidx,
                                                       const uint32_t* __restrict__ offsets, int nkeys,
                                                       double* __restrict__ out) {
  const uint32_t begin = offsets[kClasses * P.nfast];
  const uint32_t end = offsets[nkeys];
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t t = begin + blockIdx.x * blockDim.x + threadIdx.x; t < end; t += stride) {
    const uint2 ab = spairs[t];
    const uint32_t i = sidx[t];
    const DetRec x = load_det(P.dets, ab.x);
    const DetRec w = load_det(P.dets, ab.y);
    const GenPair& g = P.gen[(int)x.parent * P.nref + (int)w.parent];
    double h, s;
    eval_gen_one(g, x, w, P, &h, &s);
    store_hs(out, i, h, s);
  }
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
    const bool fast = __ldg(P.order + p) < P.nfast;
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

nw_status eval_pairs(nw_ctx* ctx, const uint32_t* pairs, uint64_t npairs, double* out, bool overlap_only,
                     cudaStream_t stream) {
  if (!ctx->built) return fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (!ctx->d_dets) return fail(ctx, NW_ERR_STATE, "no determinant basis set");
  if (npairs == 0) return NW_OK;
  if (npairs >= 0xFFFFFFFFull) return fail(ctx, NW_ERR_UNSUPPORTED, "at most 2^32 - 2 pairs per call");
  if ((reinterpret_cast<uintptr_t>(pairs) & 7) != 0) return fail(ctx, NW_ERR_INVALID, "pairs must be 8-byte aligned");
  if ((reinterpret_cast<uintptr_t>(out) & (overlap_only ? 7 : 15)) != 0)
    return fail(ctx, NW_ERR_INVALID, "output must be 16-byte aligned (8 for overlap only)");
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

  nw_status st = ensure(ctx, ctx->flag, 256);
  if (st != NW_OK) return st;
  uint32_t* flag = static_cast<uint32_t*>(ctx->flag.p);
  NW_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(uint32_t), stream));

  if (overlap_only) {
    eval_s_kernel<<<grid_stride_blocks(npairs, 128, 16), 128, 0, stream>>>(P, pairs, npairs, out, flag);
    NW_CUDA(ctx, cudaGetLastError());
    return NW_OK;
  }

  const int nkeys = ctx->nref * ctx->nref * kClasses;
  if ((st = ensure(ctx, ctx->keys, npairs * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->perm, npairs * sizeof(uint32_t))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->spairs, npairs * sizeof(uint2))) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->counts, (size_t)(nkeys + 1) * sizeof(uint32_t) * 2)) != NW_OK) return st;
  if ((st = ensure(ctx, ctx->offsets, (size_t)(nkeys + 1) * sizeof(uint32_t))) != NW_OK) return st;
  uint32_t* keys = static_cast<uint32_t*>(ctx->keys.p);
  uint32_t* sidx = static_cast<uint32_t*>(ctx->perm.p);
  uint2* spairs = static_cast<uint2*>(ctx->spairs.p);
  uint32_t* counts = static_cast<uint32_t*>(ctx->counts.p);
  uint32_t* cursor = counts + (nkeys + 1);
  uint32_t* offsets = static_cast<uint32_t*>(ctx->offsets.p);
  NW_CUDA(ctx, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (nkeys + 1), stream));

  const bool tm = ctx->timing;
  if (tm) NW_CUDA(ctx, cudaEventRecord(ctx->ev[0], stream));
  const size_t hist_bytes = (size_t)nkeys * sizeof(uint32_t);
  const bool shared_hist = hist_bytes <= 48 * 1024;
  const int cblocks = grid_stride_blocks(npairs, 256, 8);
  if (shared_hist)
    classify_kernel<true><<<cblocks, 256, hist_bytes, stream>>>(P, pairs, npairs, keys, counts, nkeys, out, 2, flag);
  else
    classify_kernel<false><<<cblocks, 256, 0, stream>>>(P, pairs, npairs, keys, counts, nkeys, out, 2, flag);
  NW_CUDA(ctx, cudaGetLastError());
  if (tm) NW_CUDA(ctx, cudaEventRecord(ctx->ev[1], stream));
  scan_kernel<<<1, 1024, 0, stream>>>(counts, nkeys, offsets, cursor);
  NW_CUDA(ctx, cudaGetLastError());
  if (tm) NW_CUDA(ctx, cudaEventRecord(ctx->ev[2], stream));
  const uint64_t chunk = std::max<uint64_t>(4096, (npairs + 148 * 8 - 1) / (148 * 8));
  const int sblocks = (int)((npairs + chunk - 1) / chunk);
  if (shared_hist)
    scatter_kernel<true><<<sblocks, 256, hist_bytes, stream>>>(keys, pairs, npairs, cursor, nkeys, chunk, spairs, sidx);
  else
    scatter_kernel<false><<<sblocks, 256, 0, stream>>>(keys, pairs, npairs, cursor, nkeys, chunk, spairs, sidx);
  NW_CUDA(ctx, cudaGetLastError());
  if (tm) NW_CUDA(ctx, cudaEventRecord(ctx->ev[3], stream));
  if (ctx->nfast > 0) {
    const int g = grid_stride_blocks(npairs, 256, 8);
    eval_light_kernel<<<g, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_medium_kernel<<<148 * 2, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_heavy_kernel<<<148, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_rt_kernel<<<148 * 2, 128, 0, stream>>>(P, spairs, sidx, offsets, out);
    NW_CUDA(ctx, cudaGetLastError());
  }
  if (tm) NW_CUDA(ctx, cudaEventRecord(ctx->ev[4], stream));
  if (ctx->nfast < ctx->nref * ctx->nref) {
    eval_gen_kernel<<<148 * 4, 128, 0, stream>>>(P, spairs, sidx, offsets, nkeys, out);
    NW_CUDA(ctx, cudaGetLastError());
  }
  if (tm) {
    NW_CUDA(ctx, cudaEventRecord(ctx->ev[5], stream));
    ctx->timed_valid = true;
  }
  return NW_OK;
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the pair evaluation (nw_eval_hs_pairs_noalloc).
//
// Some callers cannot allocate device memory when they evaluate pairs: a host that hands
// nearly all of HBM to its own memory pool (a framework's caching allocator, a solver's
// preallocated workspace), or a latency-critical loop that cannot afford cudaMalloc's implicit
// synchronisation or its failure path.  For them the per-call scratch of the evaluation (keys,
// key-sorted pair payload, request indices, per-key counts and offsets, error flag) lives in
// the fixed device array below instead of buffers grown with cudaMalloc.
//
// The array is a file-scope __device__ variable, so every GPU that loads this library holds
// it (18,055,680 bytes, 17.2 MiB) until the process exits.  Host code cannot use its name as a device
// address: the address is looked up with cudaGetSymbolAddress once per device, with that
// device current, on the first call of the entry point on that device (that first call
// should therefore come before any stream capture).  Every call shares the array and it keeps
// the last call's contents: the counts and the error flag are cleared at the start of each
// call, and calls whose work overlaps on the GPU (different streams, concurrent host threads)
// race on it and must be serialised by the caller.
// ---------------------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoallocMaxPairs = 1ull << 20;                       // 1,048,576 pairs per call
constexpr int kNoallocMaxRefs = 64;                                      // reference determinants
constexpr uint64_t kNoallocMaxKeys = (uint64_t)kNoallocMaxRefs * kNoallocMaxRefs * kClasses;
constexpr uint64_t kNoallocOffKeys = 0;
constexpr uint64_t kNoallocOffPairs = kNoallocOffKeys + 4 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffIdx = kNoallocOffPairs + 8 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffCounts = kNoallocOffIdx + 4 * kNoallocMaxPairs;
constexpr uint64_t kNoallocOffOffsets = kNoallocOffCounts + 8 * (kNoallocMaxKeys + 1);
constexpr uint64_t kNoallocOffFlag = ((kNoallocOffOffsets + 4 * (kNoallocMaxKeys + 1) + 255) / 256) * 256;
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
  const int nkeys = ctx->nref * ctx->nref * kClasses;
  uint32_t* keys = reinterpret_cast<uint32_t*>(base + kNoallocOffKeys);
  uint2* spairs = reinterpret_cast<uint2*>(base + kNoallocOffPairs);
  uint32_t* sidx = reinterpret_cast<uint32_t*>(base + kNoallocOffIdx);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + kNoallocOffCounts);
  uint32_t* cursor = counts + (nkeys + 1);
  uint32_t* offsets = reinterpret_cast<uint32_t*>(base + kNoallocOffOffsets);
  uint32_t* flag = reinterpret_cast<uint32_t*>(base + kNoallocOffFlag);
  NW_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(uint32_t), stream));
  NW_CUDA(ctx, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (nkeys + 1), stream));
  const size_t hist_bytes = (size_t)nkeys * sizeof(uint32_t);
  const bool shared_hist = hist_bytes <= 48 * 1024;
  const int cblocks = grid_stride_blocks(npairs, 256, 8);
  if (shared_hist)
    classify_kernel<true><<<cblocks, 256, hist_bytes, stream>>>(P, pairs, npairs, keys, counts, nkeys, out, 2, flag);
  else
    classify_kernel<false><<<cblocks, 256, 0, stream>>>(P, pairs, npairs, keys, counts, nkeys, out, 2, flag);
  NW_CUDA(ctx, cudaGetLastError());
  scan_kernel<<<1, 1024, 0, stream>>>(counts, nkeys, offsets, cursor);
  NW_CUDA(ctx, cudaGetLastError());
  const uint64_t chunk = std::max<uint64_t>(4096, (npairs + 148 * 8 - 1) / (148 * 8));
  const int sblocks = (int)((npairs + chunk - 1) / chunk);
  if (shared_hist)
    scatter_kernel<true><<<sblocks, 256, hist_bytes, stream>>>(keys, pairs, npairs, cursor, nkeys, chunk, spairs, sidx);
  else
    scatter_kernel<false><<<sblocks, 256, 0, stream>>>(keys, pairs, npairs, cursor, nkeys, chunk, spairs, sidx);
  NW_CUDA(ctx, cudaGetLastError());
  if (ctx->nfast > 0) {
    const int g = grid_stride_blocks(npairs, 256, 8);
    eval_light_kernel<<<g, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_medium_kernel<<<148 * 2, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_heavy_kernel<<<148, 256, 0, stream>>>(P, spairs, sidx, offsets, out);
    eval_rt_kernel<<<148 * 2, 128, 0, stream>>>(P, spairs, sidx, offsets, out);
    NW_CUDA(ctx, cudaGetLastError());
  }
  if (ctx->nfast < ctx->nref * ctx->nref) {
    eval_gen_kernel<<<148 * 4, 128, 0, stream>>>(P, spairs, sidx, offsets, nkeys, out);
    NW_CUDA(ctx, cudaGetLastError());
  }
  return NW_OK;
}

}  // namespace nw
