// NOCI-QMC with signed real walkers on the GPU (nw_qmc_*).
//
// One cycle (propagate_iteration, src/stochastic/metric.rs:378-473, for the uniform generator):
//   1. qmc_sample_kernel   per determinant: sampled population n~ = Phi_c1(N) (FRI), the
//                          diagonal change -dt (H_gg - E^S S_gg - E^I) n~ into delta, the
//                          number of spawning attempts max(1, ceil|n~|) and n~ / attempts;
//   2. scan of the attempts -> the attempt slots of every determinant; qmc_owners_kernel: the
//      cycle's totals and the owner of every 256th attempt slot;
//   3. qmc_spawn_kernel    per attempt: its parent (search inside its 256-slot chunk), a
//                          child != parent from the uniform or learned generator, the
//                          canonical pair (min, max) with its sort key;
//   4. (H, S) of all attempts through the engine's sorted pair pipeline, with the number of
//      attempts read on the device;
//   5. qmc_apply_kernel    per attempt: -dt (H - E^S S) (n~ / attempts) (N - 1), FRI-rounded
//                          with the spawn cutoff, added to delta[child] (FP64 atomics).
// After ncycles: qmc_block_kernel adds delta to the populations (annihilation happens in the
// dense accumulation) and reduces the statistics per block; qmc_finalize_kernel sums them in a
// fixed order, updates the shift (update_shift, metric.rs:729-751) and writes the report.
// The direct-overlap propagator (qmc_step, metric.rs:766-1087) keeps the real metric population
// N instead: its report FRI-compresses delta with the update cutoff (fri_population_updates,
// metric.rs:701-718), adds S delta through the overlap action (overlap.cu), and only then reduces
// the statistics; its populations start from S c_0 (initialise_populations, init.rs:32-83).
// Every per-run quantity (shift, cycle counter, attempt count) lives in device memory, so a
// report block is captured once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "internal.cuh"
#include "mlp.cuh"
#include "qmc_math.cuh"
#include "sort.cuh"

namespace {

constexpr int kReportRing = 4096;   // device report slots between host copies
constexpr int kBlockThreads = 256;
constexpr int kStatBlocks = 296;     // 2 x 148 SMs
constexpr int kStats = 6;            // nw, nref, num, den, sampled norm, nocc
constexpr uint32_t kRankBins = 25;   // (rank_a, rank_b) classes per child reference
constexpr int kLearnMaxRefs = 8;     // learned proposal: at most 8 x 25 bins
constexpr uint64_t kHarvestCap = 1ull << 22;
constexpr int kTrainBatchCap = 4096;

struct QmcState {
  double shift;
  double nw_prev;
  uint64_t cycle;
  uint64_t report;
  uint64_t attempts;   // attempts of the current block
  uint32_t npairs;     // attempts of the current cycle held in the buffers
  uint32_t overflow;   // a cycle needed more attempts than the buffers hold
  int32_t reached;
  int32_t pad;
  // 64-bit sum of the current cycle's attempts, added up by the sample kernel (the 32-bit
  // per-determinant counts and their scan would wrap beyond 2^32 - 1), read and cleared by the
  // owners kernel
  unsigned long long cycle_total;
  // the cycle whose attempts are being spawned and applied: the sample kernel draws with
  // `cycle`, the owners kernel copies it here and advances `cycle` for the next cycle
  uint64_t cycle_cur;
};

struct QmcParams {
  uint64_t ndet;
  uint64_t cap;
  uint64_t seed;
  double dt, target, c_sample, c_spawn, damping;
  int32_t ncycles, prop;
  int32_t gen;      // 0: uniform generator, 1: learned proposal mixed with the uniform one
  int32_t harvest;  // record the attempts for training the proposal
  double mix;       // weight of the uniform generator in the learned mixture
  uint32_t nbin;    // proposal bins (child reference x rank class)
  uint32_t pad;
  uint64_t hcap;    // harvest buffer capacity
  double hkeep;     // probability of recording an attempt while harvesting
  double c_update;  // direct overlap: FRI cutoff of a report's accumulated change
};

// One harvested attempt: parent, the child's bin and the weight |H - E^S S| / ((N - 1) pgen),
// an unbiased sample of the per-bin coupling mass sum_{child in bin} |H - E^S S|.
struct HarvestSample {
  uint32_t parent;
  uint32_t bin;
  float w;
  uint32_t pad;
};

// Learned proposal: bins and the cumulative bin probabilities of every parent.
struct Proposal {
  const float* cdf;          // [ndet][nbin] cumulative p(bin | parent)
  const uint32_t* det_bin;   // [ndet] bin of each determinant
  const uint32_t* bin_off;   // [nbin + 1] offsets into bin_mem
  const uint32_t* bin_mem;   // [ndet] determinants grouped by bin
  const uint32_t* pos;       // [ndet] position of a determinant inside its bin
  HarvestSample* samples;    // [hcap]
  unsigned long long* nsamples;
};

// Determinants of bin b other than the parent g.
__host__ __device__ __forceinline__ uint32_t bin_size_without(const Proposal& pr, uint32_t b, uint32_t g) {
  return pr.bin_off[b + 1] - pr.bin_off[b] - (pr.det_bin[g] == b ? 1u : 0u);
}

// pgen(child | parent) of the learned mixture.
__device__ __forceinline__ double learned_pgen(const QmcParams& q, const Proposal& pr, uint32_t g, uint32_t lam) {
  const uint32_t b = pr.det_bin[lam];
  const float* c = pr.cdf + (uint64_t)g * q.nbin;
  const double pb = (double)c[b] - (b > 0 ? (double)c[b - 1] : 0.0);
  return q.mix / (double)(q.ndet - 1) + (1.0 - q.mix) * pb / (double)bin_size_without(pr, b, g);
}

template <class T>
T* dalloc(size_t count, bool* ok) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 256)) != cudaSuccess) {
    *ok = false;
    return nullptr;
  }
  return static_cast<T*>(p);
}

// Per determinant: the sampled population, its attempt count and the amplitude n~ / attempts
// that each of its attempts carries (one division per determinant, read by the apply kernel
// through the attempt's parent).
__global__ void qmc_sample_kernel(QmcParams q, QmcState* __restrict__ st, const double* __restrict__ pop,
                                  const double2* __restrict__ diag, double* __restrict__ sampled,
                                  uint32_t* __restrict__ na, double* __restrict__ amp, double* __restrict__ delta) {
  const uint64_t cycle = st->cycle;
  const double es = st->shift;
  unsigned long long sum = 0ull;
  for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < q.ndet; d += (uint64_t)gridDim.x * blockDim.x) {
    const double p = pop[d];
    double n = 0.0;
    if (p != 0.0) n = nwq::fri(p, q.c_sample, nwq::uniform1(q.seed, cycle, d, nwq::kDrawSample));
    sampled[d] = n;
    const uint64_t a = nwq::attempts(n);
    const uint32_t a32 = a > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)a;
    na[d] = a32;
    amp[d] = n != 0.0 ? n / (double)a32 : 0.0;
    sum += a;
    if (n != 0.0) {
      const double2 hs = diag[d];
      delta[d] += nwq::diagonal_change(q.prop, q.dt, es, hs.x, hs.y, n);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
  if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&st->cycle_total, sum);
}

// Attempts are grouped in chunks of 2^kChunkShift; cown[c] = owner of the chunk's first attempt.
constexpr int kChunkShift = 8;

// After the scan of the attempt counts: every determinant with attempts writes itself as the
// owner of the chunks whose first attempt it holds (off[d] <= c 2^kChunkShift < off[d + 1]);
// thread 0 also settles the cycle's totals -- the 32-bit offsets are valid only while the
// cycle's 64-bit total fits the buffers (cap < 2^32), otherwise the cycle is flagged and the run
// fails on the host -- and moves the cycle counter on (spawn and apply use cycle_cur).
__global__ void qmc_owners_kernel(QmcParams q, QmcState* __restrict__ st, const uint32_t* __restrict__ off,
                                  uint32_t* __restrict__ cown) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long total64 = st->cycle_total;
    st->cycle_total = 0ull;
    const uint64_t total = total64 <= q.cap ? (uint64_t)off[q.ndet] : (uint64_t)total64;
    const uint64_t held = total < q.cap ? total : q.cap;
    if (total64 > q.cap) st->overflow = 1;
    st->npairs = (uint32_t)held;
    st->attempts += total;
    st->cycle_cur = st->cycle;
    st->cycle += 1;
  }
  // a warp takes 32 determinants and writes each one's chunk range with all its lanes, so a
  // determinant holding many chunks (a heavily populated reference) is not one thread's loop
  const uint64_t last = q.cap >> kChunkShift;  // cown holds chunks 0 .. last (+1 spare)
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t base = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) << 5; base < q.ndet;
       base += nwarps << 5) {
    const uint64_t d = base + lane;
    uint64_t c0 = 0, c1 = 0;  // chunks c with off[d] <= c 2^kChunkShift < off[d + 1]
    if (d < q.ndet) {
      c0 = ((uint64_t)off[d] + (1u << kChunkShift) - 1) >> kChunkShift;
      c1 = ((uint64_t)off[d + 1] + (1u << kChunkShift) - 1) >> kChunkShift;
      if (c1 > last + 1) c1 = last + 1;
    }
    for (int j = 0; j < 32; ++j) {
      const uint64_t a = __shfl_sync(0xFFFFFFFFu, c0, j), b = __shfl_sync(0xFFFFFFFFu, c1, j);
      for (uint64_t c = a + lane; c < b; c += 32) cown[c] = (uint32_t)(base + j);
    }
  }
}

// Spawn attempts and classify their pairs for the sorted evaluation in one pass: the child
// of every attempt, its pair, parent and generation probability, then the pair's sort key
// (nw::classify_one) and its rank within the key, taken warp-aggregated from the per-key
// counters (attempts of one parent share keys).  The loop is warp-uniform (its trip count
// depends on the warp's first attempt only), so every lane reaches the full-mask intrinsics.
__global__ void qmc_spawn_kernel(QmcParams q, Proposal pr, nw::EvalParams P, const QmcState* __restrict__ st,
                                 const uint32_t* __restrict__ off, const uint32_t* __restrict__ cown,
                                 uint2* __restrict__ pairs, uint32_t* __restrict__ child,
                                 uint32_t* __restrict__ parent, double* __restrict__ pg,
                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ ranks,
                                 uint32_t* __restrict__ counts, double* __restrict__ hs, uint32_t* __restrict__ flag) {
  const uint32_t n = st->npairs;
  const uint64_t cycle = st->cycle_cur;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lanes_below = (1u << lane) - 1u;
  for (uint32_t w0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); w0 < n; w0 += gridDim.x * blockDim.x) {
    const uint32_t t = w0 + lane;
    uint32_t key = nw::kSkipKey;
    // Owner of attempt t: the largest determinant a with off[a] <= t.  The owners of this
    // chunk's first attempt and of the next chunk's bound it (a warp's 32 attempts lie in one
    // chunk, so the bounds are warp-uniform); when they are fewer than 32 apart the warp loads
    // their offsets once and each lane counts those <= t, else each lane bisects.
    const uint32_t c = w0 >> kChunkShift;
    const uint64_t lo = cown[c];
    const uint64_t hi = ((uint64_t)(c + 1) << kChunkShift) < n ? cown[c + 1] : q.ndet - 1;
    uint64_t owner = lo;
    if (hi - lo < 32) {
      const uint32_t o = lo + lane <= hi ? off[lo + lane] : 0xFFFFFFFFu;
      uint32_t cnt = 0;
#pragma unroll
      for (int j = 0; j < 32; ++j) cnt += __shfl_sync(0xFFFFFFFFu, o, j) <= t ? 1u : 0u;
      owner = lo + (cnt > 0 ? cnt - 1 : 0);
    } else if (t < n) {
      uint64_t a = lo, b = hi + 1;  // off[a] <= t < off[b]
      while (b - a > 1) {
        const uint64_t mid = (a + b) >> 1;
        if (off[mid] <= t)
          a = mid;
        else
          b = mid;
      }
      owner = a;
    }
    if (t < n) {
      const uint64_t g = owner;
      double u0, u1;
      nwq::uniform2(q.seed, cycle, t, nwq::kDrawChild, &u0, &u1);
      uint64_t lam;
      if (q.gen == 0) {
        lam = nwq::uniform_child(g, q.ndet, u0);
      } else {
        double u2, u3;
        nwq::uniform2(q.seed, cycle, t, nwq::kDrawChildBin, &u2, &u3);
        if (u1 < q.mix) {
          lam = nwq::uniform_child(g, q.ndet, u2);
        } else {
          // bin from the parent's cumulative probabilities, then uniformly inside the bin
          // first bin with u2 < cdf (the last valid bin and those after it hold 1.0 > u2)
          const float* c = pr.cdf + g * q.nbin;
          uint32_t b = 0, hi = q.nbin - 1;
          while (b < hi) {
            const uint32_t mid = (b + hi) >> 1;
            if (u2 < (double)c[mid])
              hi = mid;
            else
              b = mid + 1;
          }
          const uint32_t size = bin_size_without(pr, b, (uint32_t)g);
          uint32_t idx = (uint32_t)(u3 * (double)size);
          if (idx >= size) idx = size - 1;
          if (pr.det_bin[g] == b && idx >= pr.pos[g]) ++idx;
          lam = pr.bin_mem[pr.bin_off[b] + idx];
        }
        pg[t] = learned_pgen(q, pr, (uint32_t)g, (uint32_t)lam);
      }
      const uint2 ab = lam <= g ? make_uint2((uint32_t)lam, (uint32_t)g) : make_uint2((uint32_t)g, (uint32_t)lam);
      pairs[t] = ab;
      child[t] = (uint32_t)lam;
      parent[t] = (uint32_t)g;
      key = nw::classify_one(P, ab, t, hs, 2, flag);
    }
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0u;
    if ((int)lane == leader && key != nw::kSkipKey) base = atomicAdd(&counts[key], (uint32_t)__popc(peers));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (t < n) {
      keys[t] = key;
      ranks[t] = key != nw::kSkipKey ? base + (uint32_t)__popc(peers & lanes_below) : 0u;
    }
  }
}

__global__ void qmc_apply_kernel(QmcParams q, Proposal pr, const QmcState* __restrict__ st,
                                 const double2* __restrict__ hs, const uint32_t* __restrict__ child,
                                 const uint32_t* __restrict__ parent, const double* __restrict__ amp,
                                 const double* __restrict__ pg, double* __restrict__ delta) {
  const uint32_t n = st->npairs;
  const uint64_t cycle = st->cycle_cur;
  const double es = st->shift;
  const double pu = 1.0 / (double)(q.ndet - 1);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const double2 v = hs[t];
    const double pgen = q.gen == 0 ? pu : pg[t];
    const double raw = nwq::spawn_amplitude(q.prop, q.dt, es, v.x, v.y, amp[parent[t]], pgen);
    const double dn = nwq::fri(raw, q.c_spawn, nwq::uniform1(q.seed, cycle, t, nwq::kDrawSpawn));
    if (dn != 0.0) atomicAdd(delta + child[t], dn);
    if (q.harvest && (q.hkeep >= 1.0 || nwq::uniform1(q.seed, cycle, t, nwq::kDrawHarvest) < q.hkeep)) {
      const unsigned long long k = atomicAdd(pr.nsamples, 1ull);
      if (k < q.hcap) {
        HarvestSample hsmp;
        hsmp.parent = parent[t];
        hsmp.bin = pr.det_bin[child[t]];
        hsmp.w = (float)(fabs(v.x - nwq::overlap_shift(q.prop, es) * v.y) * pu / pgen);
        hsmp.pad = 0;
        pr.samples[k] = hsmp;
      }
    }
  }
}

// Direct overlap: Phi_c(delta) of the report's accumulated change, one stream per (seed, report).
__global__ void qmc_update_fri_kernel(QmcParams q, const QmcState* __restrict__ st, double* __restrict__ delta) {
  const uint64_t report = st->report;
  for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < q.ndet; d += (uint64_t)gridDim.x * blockDim.x) {
    const double x = delta[d];
    if (x != 0.0) delta[d] = nwq::fri(x, q.c_update, nwq::uniform1(q.seed, report, d, nwq::kDrawUpdate));
  }
}

// N += delta, delta = 0; per-block partial statistics in a fixed order.
__global__ void __launch_bounds__(kBlockThreads) qmc_block_kernel(QmcParams q, double* __restrict__ pop,
                                                                  double* __restrict__ delta,
                                                                  const double* __restrict__ sampled,
                                                                  const double2* __restrict__ refhs,
                                                                  const uint8_t* __restrict__ isref, int apply,
                                                                  double* __restrict__ partial) {
  double acc[kStats] = {0, 0, 0, 0, 0, 0};
  for (uint64_t d = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d < q.ndet; d += (uint64_t)gridDim.x * blockDim.x) {
    double p = pop[d];
    if (apply) {
      p += delta[d];
      pop[d] = p;
      delta[d] = 0.0;
    }
    const double a = fabs(p);
    const double2 r = refhs[d];
    const double sn = sampled[d];
    acc[0] += a;
    acc[1] += isref[d] ? a : 0.0;
    acc[2] += p * r.x;
    acc[3] += p * r.y;
    acc[4] += fabs(sn);
    acc[5] += sn != 0.0 ? 1.0 : 0.0;
  }
  __shared__ double red[kStats][kBlockThreads];
#pragma unroll
  for (int k = 0; k < kStats; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = kBlockThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < kStats; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < kStats) partial[blockIdx.x * kStats + threadIdx.x] = red[threadIdx.x][0];
}

// Sum the partials (fixed order), update the shift and write the report of this block.
__global__ void qmc_finalize_kernel(QmcParams q, QmcState* __restrict__ st, const double* __restrict__ partial,
                                    int nblocks, nw_qmc_report* __restrict__ ring, int write_report) {
  if (blockIdx.x != 0) return;
  // one warp: lane l sums blocks l, l + 32, ...; then a fixed butterfly over the lanes
  double tot[kStats] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += 32)
#pragma unroll
    for (int k = 0; k < kStats; ++k) tot[k] += partial[b * kStats + k];
#pragma unroll
  for (int k = 0; k < kStats; ++k)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) tot[k] += __shfl_xor_sync(0xFFFFFFFFu, tot[k], off);
  if (threadIdx.x != 0) return;
  if (!write_report) {
    st->nw_prev = tot[0];
    return;
  }
  const double nw = tot[0];
  if (!st->reached && nw >= q.target) st->reached = 1;
  if (st->reached) st->shift = nwq::updated_shift(st->shift, q.damping, q.dt * (double)q.ncycles, nw, st->nw_prev);
  st->nw_prev = nw;
  nw_qmc_report& r = ring[st->report % kReportRing];
  r.shift = st->shift;
  r.eproj_num = tot[2];
  r.eproj_den = tot[3];
  r.nw = nw;
  r.nref = tot[1];
  r.sampled_norm = tot[4];
  r.nocc = (uint64_t)tot[5];
  r.nattempts = st->attempts;
  st->attempts = 0;
  st->report += 1;
}

__global__ void qmc_axpy2_kernel(uint64_t n, double c, const double2* __restrict__ x, double2* __restrict__ y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 v = x[i];
    y[i].x += c * v.x;
    y[i].y += c * v.y;
  }
}

__global__ void qmc_pairs_kernel(uint64_t n, uint32_t bra, uint2* __restrict__ pairs, int diagonal) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    pairs[i] = diagonal ? make_uint2((uint32_t)i, (uint32_t)i) : make_uint2(bra, (uint32_t)i);
}

// ---------------------------------------------------------------------------------------
// Learned proposal: training batches, weighted cross entropy, proposal table (the
// determinant descriptors are nw::mlp_features).
// ---------------------------------------------------------------------------------------
// Random minibatch of harvested samples (with replacement).
__global__ void gather_batch_kernel(const HarvestSample* __restrict__ samples, uint64_t ns, uint64_t seed,
                                    uint64_t step, int B, uint32_t* __restrict__ rows, uint32_t* __restrict__ tbin,
                                    float* __restrict__ w) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  uint64_t k = (uint64_t)(nwq::uniform1(seed, step, (uint64_t)r, nwq::kDrawTrain) * (double)ns);
  if (k >= ns) k = ns - 1;
  const HarvestSample h = samples[k];
  rows[r] = h.parent;
  tbin[r] = h.bin;
  w[r] = h.w;
}

__global__ void __launch_bounds__(1024) sum_kernel(const float* __restrict__ w, int B, float* __restrict__ out) {
  __shared__ float red[1024];
  float a = 0.0f;
  for (int r = threadIdx.x; r < B; r += blockDim.x) a += w[r];
  red[threadIdx.x] = a;
  __syncthreads();
  for (int k = 512; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Softmax over the bins that hold a child of the row's parent; in place, z becomes
// dL/dz of L = -sum_r w_r log p(bin_r | parent_r) / sum_r w_r.  One warp per row (lanes over the
// bins, coalesced row access, shuffle reductions); the rows' loss terms are added per block and
// reach `loss` with one atomic per block.
constexpr int kCeRowsPerBlock = 32;  // 8 warps x 4 rows

__global__ void __launch_bounds__(256) ce_kernel(float* __restrict__ z, int B, int K, const uint32_t* __restrict__ rows,
                                                 const uint32_t* __restrict__ tbin, const float* __restrict__ w,
                                                 const float* __restrict__ wsum, Proposal pr,
                                                 double* __restrict__ loss) {
  __shared__ double part[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double acc = 0.0;
  for (int j = 0; j < kCeRowsPerBlock / 8; ++j) {
    const int r = blockIdx.x * kCeRowsPerBlock + j * 8 + warp;
    if (r >= B) break;  // warp-uniform
    float* zr = z + (size_t)r * K;
    const uint32_t g = rows[r];
    float mx = -INFINITY;
    for (int k = lane; k < K; k += 32)
      if (bin_size_without(pr, (uint32_t)k, g) > 0) mx = fmaxf(mx, zr[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    float se = 0.0f;
    for (int k = lane; k < K; k += 32)
      if (bin_size_without(pr, (uint32_t)k, g) > 0) se += __expf(zr[k] - mx);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xFFFFFFFFu, se, o);
    const float scale = w[r] / *wsum;
    const uint32_t t = tbin[r];
    if (lane == 0) acc += -(double)scale * (double)(zr[t] - mx - __logf(se));
    for (int k = lane; k < K; k += 32) {
      const bool valid = bin_size_without(pr, (uint32_t)k, g) > 0;
      const float p = valid ? __expf(zr[k] - mx) / se : 0.0f;
      zr[k] = valid ? scale * (p - (k == (int)t ? 1.0f : 0.0f)) : 0.0f;
    }
  }
  if (lane == 0) part[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < 8; ++i) s += part[i];
    atomicAdd(loss, s);
  }
}

// Cumulative bin probabilities of determinants row0 .. row0 + B - 1 from their logits.
__global__ void table_kernel(const float* __restrict__ z, int B, int K, uint32_t row0, Proposal pr,
                             float* __restrict__ cdf) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  const float* zr = z + (size_t)r * K;
  const uint32_t g = row0 + (uint32_t)r;
  float mx = -INFINITY;
  int last = -1;
  for (int k = 0; k < K; ++k)
    if (bin_size_without(pr, (uint32_t)k, g) > 0) {
      mx = fmaxf(mx, zr[k]);
      last = k;
    }
  double se = 0.0;
  for (int k = 0; k < K; ++k)
    if (bin_size_without(pr, (uint32_t)k, g) > 0) se += exp((double)(zr[k] - mx));
  float* c = cdf + (uint64_t)g * K;
  double acc = 0.0;
  for (int k = 0; k < K; ++k) {
    if (bin_size_without(pr, (uint32_t)k, g) > 0) acc += exp((double)(zr[k] - mx)) / se;
    c[k] = k >= last ? 1.0f : (float)acc;
  }
}

inline int grid_for(uint64_t work, int per_sm = 8) {
  uint64_t g = (work + kBlockThreads - 1) / kBlockThreads;
  g = std::min<uint64_t>(g, 148ull * per_sm);
  return (int)std::max<uint64_t>(g, 1);
}

}  // namespace

struct nw_qmc {
  nw_ctx* ctx = nullptr;
  nw_qmc_opts opts{};
  QmcParams q{};
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // bracket the graph launches of the last run
  float last_ms = 0.0f;
  // device state
  QmcState* st = nullptr;
  double* pop = nullptr;
  double* sampled = nullptr;
  double* delta = nullptr;
  uint32_t* na = nullptr;
  uint32_t* off = nullptr;
  uint32_t* cown = nullptr;  // owner of the first attempt of each chunk
  uint32_t* tsum = nullptr;
  double2* diag = nullptr;
  double2* refhs = nullptr;
  uint8_t* isref = nullptr;
  uint2* pairs = nullptr;
  uint32_t* child = nullptr;
  double* amp = nullptr;     // per determinant: n~ / attempts of the current cycle
  uint32_t* parent = nullptr;
  double* pg = nullptr;
  double2* hs = nullptr;
  double* partial = nullptr;
  nw_qmc_report* ring = nullptr;
  nw::OverlapPlan* ovl = nullptr;  // direct overlap: the context's overlap action
  // sort scratch for the attempts
  nw::EvalParams P{};
  uint64_t nkeys = 0;
  nw::SortScratch S{};
  std::vector<void*> owned;
  // learned proposal
  Proposal pr{};
  float* cdf = nullptr;
  bool learnable = false;    // nref small enough for the bin output layer
  bool table_ready = false;  // cdf built by a training run
  std::vector<uint32_t> h_det_bin, h_bin_off;  // host copies of the bins (argument checks)
  bool counted = false;  // holds one of ctx->live_qmc
  nw::Mlp mlp{};
  uint32_t* trows = nullptr;  // training batch: parents, target bins, weights, weight sum
  uint32_t* tbin = nullptr;
  float* tw = nullptr;
  float* twsum = nullptr;
  double* tloss = nullptr;
};

namespace {

nw_status qmc_fail(nw_qmc* q, nw_status s, const std::string& m) { return nw::fail(q->ctx, s, m); }

// One cycle's launches (steps 1-5 of the file comment), then the cycle counter.
nw_status enqueue_cycle(nw_qmc* q) {
  nw_ctx* ctx = q->ctx;
  const cudaStream_t s = q->stream;
  const uint64_t nd = q->q.ndet;
  qmc_sample_kernel<<<grid_for(nd), kBlockThreads, 0, s>>>(q->q, q->st, q->pop, q->diag, q->sampled, q->na, q->amp,
                                                          q->delta);
  NW_CUDA(ctx, cudaGetLastError());
  nw_status st = nw::scan_exclusive(ctx, q->na, nd, q->off, q->tsum, s);
  if (st != NW_OK) return st;
  qmc_owners_kernel<<<grid_for(nd), kBlockThreads, 0, s>>>(q->q, q->st, q->off, q->cown);
  NW_CUDA(ctx, cudaMemsetAsync(q->S.counts, 0, sizeof(uint32_t) * q->nkeys, s));
  qmc_spawn_kernel<<<grid_for(q->q.cap), kBlockThreads, 0, s>>>(
      q->q, q->pr, q->P, q->st, q->off, q->cown, q->pairs, q->child, q->parent, q->pg,
      q->S.keys, q->S.ranks, q->S.counts, reinterpret_cast<double*>(q->hs), q->S.flag);
  NW_CUDA(ctx, cudaGetLastError());
  st = nw::launch_sorted(ctx, q->P, q->nkeys, reinterpret_cast<const uint32_t*>(q->pairs), q->q.cap,
                         reinterpret_cast<double*>(q->hs), q->S, s, nullptr, nw::EvalMode::kHS, &q->st->npairs, true);
  if (st != NW_OK) return st;
  qmc_apply_kernel<<<grid_for(q->q.cap), kBlockThreads, 0, s>>>(q->q, q->pr, q->st, q->hs, q->child, q->parent,
                                                                q->amp, q->pg, q->delta);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

nw_status enqueue_block(nw_qmc* q) {
  for (int c = 0; c < q->q.ncycles; ++c) {
    const nw_status st = enqueue_cycle(q);
    if (st != NW_OK) return st;
  }
  int apply = 1;
  if (q->q.prop == nwq::kDirectOverlap) {
    // N += S Phi_c(delta), delta = 0
    if (q->q.c_update > 0.0) qmc_update_fri_kernel<<<grid_for(q->q.ndet), kBlockThreads, 0, q->stream>>>(q->q, q->st, q->delta);
    const nw_status st = nw::overlap_apply(q->ctx, q->ovl, q->delta, q->pop, q->stream);
    if (st != NW_OK) return st;
    NW_CUDA(q->ctx, cudaMemsetAsync(q->delta, 0, sizeof(double) * q->q.ndet, q->stream));
    apply = 0;
  }
  qmc_block_kernel<<<kStatBlocks, kBlockThreads, 0, q->stream>>>(q->q, q->pop, q->delta, q->sampled, q->refhs, q->isref,
                                                                 apply, q->partial);
  qmc_finalize_kernel<<<1, 32, 0, q->stream>>>(q->q, q->st, q->partial, kStatBlocks, q->ring, 1);
  NW_CUDA(q->ctx, cudaGetLastError());
  return NW_OK;
}

// Statistics of the current populations as the previous-block reference (no report written).
nw_status reset_reference_stats(nw_qmc* q) {
  NW_CUDA(q->ctx, cudaMemsetAsync(q->sampled, 0, sizeof(double) * q->q.ndet, q->stream));
  qmc_block_kernel<<<kStatBlocks, kBlockThreads, 0, q->stream>>>(q->q, q->pop, q->delta, q->sampled, q->refhs, q->isref,
                                                                 0, q->partial);
  qmc_finalize_kernel<<<1, 32, 0, q->stream>>>(q->q, q->st, q->partial, kStatBlocks, q->ring, 0);
  NW_CUDA(q->ctx, cudaGetLastError());
  NW_CUDA(q->ctx, cudaStreamSynchronize(q->stream));
  return NW_OK;
}

void release(nw_qmc* q) {
  if (q->counted) q->ctx->live_qmc -= 1;
  nw::mlp_destroy(&q->mlp);
  if (q->graph) cudaGraphExecDestroy(q->graph);
  if (q->ev0) cudaEventDestroy(q->ev0);
  if (q->ev1) cudaEventDestroy(q->ev1);
  for (void* p : q->owned)
    if (p) cudaFree(p);
  if (q->stream) cudaStreamDestroy(q->stream);
  delete q;
}

// Loss and parameter gradients of the weighted cross entropy for the batch held in
// trows / tbin / tw (B rows); the loss goes to *loss_out when it is not null.
nw_status batch_loss_grad(nw_qmc* q, int B, double* loss_out) {
  nw_ctx* ctx = q->ctx;
  const cudaStream_t s = q->stream;
  nw::Mlp& m = q->mlp;
  nw_status st = nw::mlp_features(ctx, &m, ctx->d_dets, q->trows, 0, B, s);
  if (st != NW_OK) return st;
  st = nw::mlp_forward(ctx, &m, B, s);
  if (st != NW_OK) return st;
  sum_kernel<<<1, 1024, 0, s>>>(q->tw, B, q->twsum);
  NW_CUDA(ctx, cudaMemsetAsync(q->tloss, 0, sizeof(double), s));
  ce_kernel<<<(B + kCeRowsPerBlock - 1) / kCeRowsPerBlock, 256, 0, s>>>(m.z, B, m.nout, q->trows, q->tbin, q->tw,
                                                                         q->twsum, q->pr, q->tloss);
  NW_CUDA(ctx, cudaGetLastError());
  if ((st = nw::mlp_backward(ctx, &m, B, s)) != NW_OK) return st;
  if (loss_out) {
    NW_CUDA(ctx, cudaMemcpyAsync(loss_out, q->tloss, sizeof(double), cudaMemcpyDeviceToHost, s));
    NW_CUDA(ctx, cudaStreamSynchronize(s));
  }
  return NW_OK;
}

// Cumulative bin probabilities of every determinant from the current network.
nw_status build_table(nw_qmc* q) {
  nw_ctx* ctx = q->ctx;
  const cudaStream_t s = q->stream;
  nw::Mlp& m = q->mlp;
  for (uint64_t r0 = 0; r0 < q->q.ndet; r0 += (uint64_t)m.bcap) {
    const int B = (int)std::min<uint64_t>((uint64_t)m.bcap, q->q.ndet - r0);
    nw_status st = nw::mlp_features(ctx, &m, ctx->d_dets, nullptr, (uint32_t)r0, B, s);
    if (st == NW_OK) st = nw::mlp_forward(ctx, &m, B, s);
    if (st != NW_OK) return st;
    table_kernel<<<(B + 127) / 128, 128, 0, s>>>(m.z, B, m.nout, (uint32_t)r0, q->pr, q->cdf);
    NW_CUDA(ctx, cudaGetLastError());
  }
  NW_CUDA(ctx, cudaStreamSynchronize(s));
  q->table_ready = true;
  return NW_OK;
}

void invalidate_graph(nw_qmc* q) {
  if (q->graph) cudaGraphExecDestroy(q->graph);
  q->graph = nullptr;
}

}  // namespace

extern "C" {

nw_status nw_qmc_harvest(nw_qmc* q, int32_t enable, double keep_probability) {
  if (!q || !(keep_probability > 0.0) || !(keep_probability <= 1.0)) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  if (enable) NW_CUDA(q->ctx, cudaMemsetAsync(q->pr.nsamples, 0, sizeof(unsigned long long), q->stream));
  NW_CUDA(q->ctx, cudaStreamSynchronize(q->stream));
  q->q.harvest = enable ? 1 : 0;
  q->q.hkeep = keep_probability;
  invalidate_graph(q);
  return NW_OK;
}

nw_status nw_qmc_train_proposal(nw_qmc* q, const nw_mlp_opts* opts, nw_mlp_report* rep) {
  if (!q || !opts || !rep) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  if (opts->epochs < 0 || opts->batch < 1 || opts->batch > kTrainBatchCap || !(opts->lr > 0.0))
    return qmc_fail(q, NW_ERR_INVALID, "invalid training options (batch <= 4096)");
  nw_ctx* ctx = q->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  unsigned long long count = 0;
  NW_CUDA(ctx, cudaMemcpy(&count, q->pr.nsamples, sizeof(count), cudaMemcpyDeviceToHost));
  const uint64_t ns = std::min<uint64_t>(count, kHarvestCap);
  std::memset(rep, 0, sizeof(*rep));
  rep->samples = ns;
  if (ns == 0) return qmc_fail(q, NW_ERR_STATE, "no harvested attempts to train on (nw_qmc_harvest)");
  const int B = opts->batch;
  const uint64_t per_epoch = (ns + (uint64_t)B - 1) / (uint64_t)B;
  const uint64_t steps = (uint64_t)opts->epochs * per_epoch;
  for (uint64_t step = 0; step < steps; ++step) {
    gather_batch_kernel<<<(B + 127) / 128, 128, 0, q->stream>>>(q->pr.samples, ns, opts->seed, step, B, q->trows,
                                                                q->tbin, q->tw);
    NW_CUDA(ctx, cudaGetLastError());
    const bool report = step == 0 || step + 1 == steps;
    double loss = 0.0;
    nw_status st = batch_loss_grad(q, B, report ? &loss : nullptr);
    if (st != NW_OK) return st;
    if (step == 0) rep->loss_first = loss;
    if (step + 1 == steps) rep->loss_last = loss;
    if ((st = nw::mlp_adam(ctx, &q->mlp, (float)opts->lr, q->stream)) != NW_OK) return st;
  }
  rep->steps = (int32_t)steps;
  return build_table(q);
}

nw_status nw_qmc_set_generator(nw_qmc* q, int32_t learned, double mix) {
  if (!q || !(mix > 0.0) || !(mix <= 1.0)) return NW_ERR_INVALID;
  if (learned && !q->table_ready) return qmc_fail(q, NW_ERR_STATE, "no trained proposal (nw_qmc_train_proposal)");
  q->q.gen = learned ? 1 : 0;
  q->q.mix = mix;
  invalidate_graph(q);
  return NW_OK;
}

nw_status nw_qmc_proposal_dims(nw_qmc* q, int32_t* din, int32_t* nbin, uint64_t* nparams) {
  if (!q || !din || !nbin || !nparams) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  *din = q->mlp.din;
  *nbin = q->mlp.nout;
  *nparams = q->mlp.nparams;
  return NW_OK;
}

nw_status nw_qmc_mlp_params(nw_qmc* q, float* params) {
  if (!q || !params) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  NW_CUDA(q->ctx, cudaMemcpy(params, q->mlp.params, sizeof(float) * q->mlp.nparams, cudaMemcpyDeviceToHost));
  return NW_OK;
}

nw_status nw_qmc_set_mlp_params(nw_qmc* q, const float* params) {
  if (!q || !params) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  for (size_t i = 0; i < q->mlp.nparams; ++i)
    if (!std::isfinite(params[i])) return qmc_fail(q, NW_ERR_INVALID, "non-finite parameter");
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  NW_CUDA(q->ctx, cudaMemcpy(q->mlp.params, params, sizeof(float) * q->mlp.nparams, cudaMemcpyHostToDevice));
  nw_status st = nw::mlp_sync_bf16(q->ctx, &q->mlp, nullptr);
  if (st != NW_OK) return st;
  NW_CUDA(q->ctx, cudaDeviceSynchronize());
  return build_table(q);
}

nw_status nw_qmc_mlp_loss_grad(nw_qmc* q, const uint32_t* parents, const uint32_t* bins, const float* w, int32_t n,
                               double* loss, float* grads) {
  if (!q || !parents || !bins || !w || !loss || !grads || n < 1) return NW_ERR_INVALID;
  if (!q->learnable) return qmc_fail(q, NW_ERR_UNSUPPORTED, "learned proposal needs at most 8 references");
  if (n > kTrainBatchCap) return qmc_fail(q, NW_ERR_UNSUPPORTED, "at most 4096 rows");
  for (int32_t r = 0; r < n; ++r) {
    if (parents[r] >= q->q.ndet || bins[r] >= q->q.nbin || !std::isfinite(w[r]) || w[r] < 0.0f)
      return qmc_fail(q, NW_ERR_INVALID, "invalid training row");
    const uint32_t b = bins[r];
    if (q->h_bin_off[b + 1] - q->h_bin_off[b] - (q->h_det_bin[parents[r]] == b ? 1u : 0u) == 0)
      return qmc_fail(q, NW_ERR_INVALID, "training row targets a bin without a child of its parent");
  }
  nw_ctx* ctx = q->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  NW_CUDA(ctx, cudaMemcpy(q->trows, parents, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(q->tbin, bins, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
  NW_CUDA(ctx, cudaMemcpy(q->tw, w, sizeof(float) * n, cudaMemcpyHostToDevice));
  nw_status st = batch_loss_grad(q, n, loss);
  if (st != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpy(grads, q->mlp.grads, sizeof(float) * q->mlp.nparams, cudaMemcpyDeviceToHost));
  return NW_OK;
}

nw_status nw_qmc_proposal_probs(nw_qmc* q, uint32_t det, double* probs) {
  if (!q || !probs) return NW_ERR_INVALID;
  if (!q->table_ready) return qmc_fail(q, NW_ERR_STATE, "no trained proposal");
  if (det >= q->q.ndet) return qmc_fail(q, NW_ERR_INVALID, "determinant index out of range");
  std::vector<float> c(q->q.nbin);
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  NW_CUDA(q->ctx, cudaMemcpy(c.data(), q->cdf + (uint64_t)det * q->q.nbin, sizeof(float) * q->q.nbin,
                             cudaMemcpyDeviceToHost));
  for (uint32_t b = 0; b < q->q.nbin; ++b) probs[b] = (double)c[b] - (b > 0 ? (double)c[b - 1] : 0.0);
  return NW_OK;
}

nw_status nw_qmc_create(nw_ctx* ctx, const nw_qmc_opts* opts, const double* c0, const uint32_t* ref_idx,
                        uint64_t nref_idx, nw_qmc** out) {
  if (!out) return NW_ERR_INVALID;
  *out = nullptr;
  if (!ctx || !opts || !c0 || (nref_idx && !ref_idx)) return NW_ERR_INVALID;
  nw::CtxGuard guard(ctx, nullptr);
  if (!ctx->built) return nw::fail(ctx, NW_ERR_STATE, "intermediates not built");
  if (ctx->partial)
    return nw::fail(ctx, NW_ERR_STATE, "the intermediates hold one block of a blocked evaluation (rebuild them)");
  if (!ctx->d_dets || ctx->ndet < 2) return nw::fail(ctx, NW_ERR_STATE, "QMC needs a resident basis of >= 2 determinants");
  if (!(opts->dt > 0.0) || opts->ncycles < 1 || opts->propagator < 0 || opts->propagator > 5 ||
      !(opts->initial_population > 0.0) || !(opts->sampling_cutoff >= 0.0) || !(opts->spawn_cutoff >= 0.0) ||
      !(opts->update_cutoff >= 0.0) || !std::isfinite(opts->update_cutoff) ||
      !std::isfinite(opts->initial_shift) || !std::isfinite(opts->shift_damping))
    return nw::fail(ctx, NW_ERR_INVALID, "invalid QMC options");
  const uint64_t nd = ctx->ndet;
  double norm = 0.0;
  for (uint64_t i = 0; i < nd; ++i) {
    if (!std::isfinite(c0[i])) return nw::fail(ctx, NW_ERR_INVALID, "non-finite initial coefficient");
    norm += std::fabs(c0[i]);
  }
  if (norm == 0.0) return nw::fail(ctx, NW_ERR_INVALID, "initial coefficients are all zero");
  for (uint64_t k = 0; k < nref_idx; ++k)
    if (ref_idx[k] >= nd) return nw::fail(ctx, NW_ERR_INVALID, "reference index out of range");
  NW_CUDA(ctx, cudaSetDevice(ctx->device));

  nw_qmc* q = new (std::nothrow) nw_qmc;
  if (!q) return NW_ERR_ALLOC;
  q->ctx = ctx;
  q->counted = true;
  ctx->live_qmc += 1;
  q->opts = *opts;
  uint64_t cap = opts->max_attempts;
  // automatic: the 1-norm can overshoot the target many times before the shift holds it
  // (below the annihilation plateau it grows at the sign-incoherent rate)
  if (cap == 0) cap = (uint64_t)(16.0 * std::max(opts->target_population, opts->initial_population)) + 2 * nd + (1u << 20);
  cap = std::min<uint64_t>(cap, 0xFFFFFFF0ull);
  q->q = QmcParams{nd,
                   cap,
                   opts->seed,
                   opts->dt,
                   opts->target_population,
                   opts->sampling_cutoff,
                   opts->spawn_cutoff,
                   opts->shift_damping,
                   opts->ncycles,
                   opts->propagator,
                   0,
                   0,
                   0.1,
                   (uint32_t)ctx->nref * kRankBins,
                   0,
                   kHarvestCap,
                   1.0,
                   opts->update_cutoff};
  bool ok = true;
  auto take = [&](auto*& p, size_t count) {
    using T = std::remove_reference_t<decltype(*p)>;
    p = dalloc<T>(count, &ok);
    q->owned.push_back(p);
  };
  take(q->st, 1);
  take(q->pop, nd);
  take(q->sampled, nd);
  take(q->delta, nd);
  take(q->na, nd);
  take(q->off, nd + 1);
  take(q->cown, (cap >> kChunkShift) + 2);
  take(q->tsum, nd / 4096 + 1);
  take(q->diag, nd);
  take(q->refhs, nd);
  take(q->isref, nd);
  take(q->pairs, std::max<uint64_t>(cap, nd));
  take(q->child, cap);
  take(q->amp, nd);
  take(q->parent, cap);
  take(q->pg, cap);
  take(q->hs, std::max<uint64_t>(cap, nd));
  take(q->partial, (size_t)kStatBlocks * kStats);
  take(q->ring, kReportRing);
  q->P = nw::make_params(ctx);
  // fine sort keys sized from the walker 1-norm (a quarter of it: every cycle clears and
  // scans all keys, and finer buckets gain the evaluators less than the scan costs), not from
  // the attempt capacity
  const uint64_t typical = (uint64_t)(0.25 * std::max(opts->target_population, opts->initial_population)) + nd;
  q->nkeys = nw::plan_keys(ctx, q->P, std::min<uint64_t>(nw::kFineMax, std::max<uint64_t>(nw::kFineMin, std::min(typical, cap))));
  take(q->S.keys, cap);
  take(q->S.ranks, cap);
  take(q->S.sidx, cap);
  take(q->S.counts, q->nkeys);
  take(q->S.offsets, q->nkeys + 1);
  take(q->S.tsum, q->nkeys / 4096 + 1);
  take(q->S.flag, 64);
  q->S.work = q->S.flag ? q->S.flag + 8 : nullptr;
  // learned-proposal bins: child reference x (rank_a, rank_b) class
  q->learnable = ctx->nref <= kLearnMaxRefs;
  std::vector<uint32_t> det_bin(nd), bin_off(q->q.nbin + 1, 0), bin_mem(nd), pos(nd);
  if (q->learnable && ok) {
    std::vector<uint16_t> desc(nd);
    if (cudaMemcpy(desc.data(), ctx->d_desc, sizeof(uint16_t) * nd, cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
    for (uint64_t g = 0; g < nd; ++g) {
      const uint32_t par = desc[g] & 0xFF, ra = (desc[g] >> 8) & 15, rb = desc[g] >> 12;
      det_bin[g] = par * kRankBins + ra * 5 + rb;
      ++bin_off[det_bin[g] + 1];
    }
    for (uint32_t b = 0; b < q->q.nbin; ++b) bin_off[b + 1] += bin_off[b];
    std::vector<uint32_t> fill(bin_off.begin(), bin_off.end() - 1);
    for (uint64_t g = 0; g < nd; ++g) {
      pos[g] = fill[det_bin[g]] - bin_off[det_bin[g]];
      bin_mem[fill[det_bin[g]]++] = (uint32_t)g;
    }
    uint32_t *d_bin = nullptr, *d_off = nullptr, *d_mem = nullptr, *d_pos = nullptr;
    take(d_bin, nd);
    take(d_off, q->q.nbin + 1);
    take(d_mem, nd);
    take(d_pos, nd);
    take(q->cdf, nd * q->q.nbin);
    HarvestSample* samples = nullptr;
    unsigned long long* nsamples = nullptr;
    take(samples, kHarvestCap);
    take(nsamples, 1);
    take(q->trows, kTrainBatchCap);
    take(q->tbin, kTrainBatchCap);
    take(q->tw, kTrainBatchCap);
    take(q->twsum, 1);
    take(q->tloss, 1);
    if (ok) {
      ok = cudaMemcpy(d_bin, det_bin.data(), sizeof(uint32_t) * nd, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(d_off, bin_off.data(), sizeof(uint32_t) * (q->q.nbin + 1), cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(d_mem, bin_mem.data(), sizeof(uint32_t) * nd, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemcpy(d_pos, pos.data(), sizeof(uint32_t) * nd, cudaMemcpyHostToDevice) == cudaSuccess &&
           cudaMemset(nsamples, 0, sizeof(unsigned long long)) == cudaSuccess;
    }
    q->pr = Proposal{q->cdf, d_bin, d_off, d_mem, d_pos, samples, nsamples};
    q->h_det_bin = det_bin;
    q->h_bin_off = bin_off;
    if (ok) {
      const int din = nw::mlp_descriptor_width(ctx->nref, ctx->nmo);
      ok = nw::mlp_create(ctx, &q->mlp, din, (int)q->q.nbin, kTrainBatchCap, opts->seed ^ 0x5EEDull) == NW_OK;
    }
  }
  if (!ok) {
    release(q);
    return nw::fail(ctx, NW_ERR_ALLOC, "QMC buffer allocation failed");
  }
  if (cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&q->ev0) != cudaSuccess || cudaEventCreate(&q->ev1) != cudaSuccess) {
    release(q);
    return nw::fail(ctx, NW_ERR_CUDA, "QMC stream creation failed");
  }
  nw_status st = NW_OK;
  do {
    // diagonal (H_gg, S_gg) and projected-energy couplings sum_i c0_i (H_ig, S_ig)
    qmc_pairs_kernel<<<grid_for(nd), kBlockThreads, 0, q->stream>>>(nd, 0, q->pairs, 1);
    if ((st = nw::eval_pairs(ctx, reinterpret_cast<uint32_t*>(q->pairs), nd, reinterpret_cast<double*>(q->diag),
                             nw::EvalMode::kHS, q->stream)) != NW_OK)
      break;
    if (cudaMemsetAsync(q->refhs, 0, sizeof(double2) * nd, q->stream) != cudaSuccess) {
      st = nw::fail(ctx, NW_ERR_CUDA, "memset");
      break;
    }
    std::vector<uint8_t> isref(nd, 0);
    for (uint64_t k = 0; k < nref_idx && st == NW_OK; ++k) {
      const uint32_t i = ref_idx[k];
      isref[i] = 1;
      if (c0[i] == 0.0) continue;
      qmc_pairs_kernel<<<grid_for(nd), kBlockThreads, 0, q->stream>>>(nd, i, q->pairs, 0);
      if ((st = nw::eval_pairs(ctx, reinterpret_cast<uint32_t*>(q->pairs), nd, reinterpret_cast<double*>(q->hs),
                               nw::EvalMode::kHS, q->stream)) != NW_OK)
        break;
      qmc_axpy2_kernel<<<grid_for(nd), kBlockThreads, 0, q->stream>>>(nd, c0[i], q->hs, q->refhs);
    }
    if (st != NW_OK) break;
    std::vector<double> pop(c0, c0 + nd);
    double pnorm = norm;
    if (opts->propagator == nwq::kDirectOverlap) {
      // N_0 = S c_0 through the overlap action (delta as the source, pop as the target)
      if ((st = nw::overlap_plan_get(ctx, q->stream, &q->ovl)) != NW_OK) break;
      if (cudaMemcpyAsync(q->delta, c0, sizeof(double) * nd, cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
          cudaMemsetAsync(q->pop, 0, sizeof(double) * nd, q->stream) != cudaSuccess) {
        st = nw::fail(ctx, NW_ERR_CUDA, "QMC initialisation copies failed");
        break;
      }
      if ((st = nw::overlap_apply(ctx, q->ovl, q->delta, q->pop, q->stream)) != NW_OK) break;
      if (cudaMemcpyAsync(pop.data(), q->pop, sizeof(double) * nd, cudaMemcpyDeviceToHost, q->stream) != cudaSuccess ||
          cudaStreamSynchronize(q->stream) != cudaSuccess) {
        st = nw::fail(ctx, NW_ERR_CUDA, "QMC initialisation copies failed");
        break;
      }
      pnorm = 0.0;
      for (uint64_t i = 0; i < nd; ++i) pnorm += std::fabs(pop[i]);
      if (!(pnorm > 0.0) || !std::isfinite(pnorm)) {
        st = nw::fail(ctx, NW_ERR_INVALID, "S c0 is zero or not finite");
        break;
      }
    }
    const double scale = opts->initial_population / pnorm;
    for (uint64_t i = 0; i < nd; ++i) pop[i] *= scale;
    QmcState hst{};
    hst.shift = opts->initial_shift;
    if (cudaMemcpyAsync(q->isref, isref.data(), nd, cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
        cudaMemcpyAsync(q->pop, pop.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
        cudaMemcpyAsync(q->st, &hst, sizeof(hst), cudaMemcpyHostToDevice, q->stream) != cudaSuccess ||
        cudaMemsetAsync(q->delta, 0, sizeof(double) * nd, q->stream) != cudaSuccess ||
        cudaMemsetAsync(q->S.flag, 0, 64, q->stream) != cudaSuccess ||
        cudaStreamSynchronize(q->stream) != cudaSuccess) {
      st = nw::fail(ctx, NW_ERR_CUDA, "QMC initialisation copies failed");
      break;
    }
    st = reset_reference_stats(q);
  } while (false);
  if (st != NW_OK) {
    release(q);
    return st;
  }
  *out = q;
  return NW_OK;
}

nw_status nw_qmc_run(nw_qmc* q, int32_t nreports, nw_qmc_report* reports) {
  if (!q || nreports < 0 || (nreports && !reports)) return NW_ERR_INVALID;
  nw::CtxGuard guard(q->ctx, q->stream);
  nw_ctx* ctx = q->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!q->graph) {
    // capture one report block
    cudaGraph_t g = nullptr;
    NW_CUDA(ctx, cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
    const nw_status st = enqueue_block(q);
    const cudaError_t e = cudaStreamEndCapture(q->stream, &g);
    if (st != NW_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return nw::cuda_fail(ctx, e, "QMC graph capture");
    const cudaError_t ei = cudaGraphInstantiate(&q->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      q->graph = nullptr;
      return nw::cuda_fail(ctx, ei, "QMC graph instantiation");
    }
  }
  QmcState hst{};
  NW_CUDA(ctx, cudaMemcpyAsync(&hst, q->st, sizeof(hst), cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  uint64_t first = hst.report;
  int done = 0;
  q->last_ms = 0.0f;
  while (done < nreports) {
    const int chunk = std::min(nreports - done, kReportRing);
    NW_CUDA(ctx, cudaEventRecord(q->ev0, q->stream));
    for (int r = 0; r < chunk; ++r) NW_CUDA(ctx, cudaGraphLaunch(q->graph, q->stream));
    NW_CUDA(ctx, cudaEventRecord(q->ev1, q->stream));
    for (int r = 0; r < chunk; ++r) {
      const uint64_t slot = (first + (uint64_t)r) % kReportRing;
      NW_CUDA(ctx, cudaMemcpyAsync(&reports[done + r], q->ring + slot, sizeof(nw_qmc_report), cudaMemcpyDeviceToHost,
                                   q->stream));
    }
    NW_CUDA(ctx, cudaMemcpyAsync(&hst, q->st, sizeof(hst), cudaMemcpyDeviceToHost, q->stream));
    NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
    float ms = 0.0f;
    NW_CUDA(ctx, cudaEventElapsedTime(&ms, q->ev0, q->ev1));
    q->last_ms += ms;
    first += chunk;
    done += chunk;
    if (hst.overflow)
      return qmc_fail(q, NW_ERR_UNSUPPORTED, "a QMC cycle needed more spawning attempts than max_attempts (" +
                                                 std::to_string(q->q.cap) + ")");
  }
  return NW_OK;
}

nw_status nw_qmc_set_shift(nw_qmc* q, double shift) {
  if (!q || !std::isfinite(shift)) return NW_ERR_INVALID;
  nw_ctx* ctx = q->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  QmcState hst{};
  NW_CUDA(ctx, cudaMemcpyAsync(&hst, q->st, sizeof(hst), cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  hst.shift = shift;
  NW_CUDA(ctx, cudaMemcpyAsync(q->st, &hst, sizeof(hst), cudaMemcpyHostToDevice, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  return NW_OK;
}

nw_status nw_qmc_last_run_ms(const nw_qmc* q, float* ms) {
  if (!q || !ms) return NW_ERR_INVALID;
  *ms = q->last_ms;
  return NW_OK;
}

nw_status nw_qmc_populations(nw_qmc* q, double* populations) {
  if (!q || !populations) return NW_ERR_INVALID;
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  NW_CUDA(q->ctx, cudaMemcpyAsync(populations, q->pop, sizeof(double) * q->q.ndet, cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(q->ctx, cudaStreamSynchronize(q->stream));
  return NW_OK;
}

nw_status nw_qmc_set_populations(nw_qmc* q, const double* populations) {
  if (!q || !populations) return NW_ERR_INVALID;
  for (uint64_t i = 0; i < q->q.ndet; ++i)
    if (!std::isfinite(populations[i])) return qmc_fail(q, NW_ERR_INVALID, "non-finite population");
  NW_CUDA(q->ctx, cudaSetDevice(q->ctx->device));
  NW_CUDA(q->ctx, cudaMemcpyAsync(q->pop, populations, sizeof(double) * q->q.ndet, cudaMemcpyHostToDevice, q->stream));
  return reset_reference_stats(q);
}

nw_status nw_qmc_cycle_delta(nw_qmc* q, uint64_t cycle, double* delta) {
  if (!q || !delta) return NW_ERR_INVALID;
  nw_ctx* ctx = q->ctx;
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  QmcState hst{};
  NW_CUDA(ctx, cudaMemcpyAsync(&hst, q->st, sizeof(hst), cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  const uint64_t saved_cycle = hst.cycle, saved_attempts = hst.attempts;
  hst.cycle = cycle;
  NW_CUDA(ctx, cudaMemcpyAsync(q->st, &hst, sizeof(hst), cudaMemcpyHostToDevice, q->stream));
  NW_CUDA(ctx, cudaMemsetAsync(q->delta, 0, sizeof(double) * q->q.ndet, q->stream));
  nw_status st = enqueue_cycle(q);
  if (st != NW_OK) return st;
  NW_CUDA(ctx, cudaMemcpyAsync(delta, q->delta, sizeof(double) * q->q.ndet, cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(ctx, cudaMemsetAsync(q->delta, 0, sizeof(double) * q->q.ndet, q->stream));
  NW_CUDA(ctx, cudaMemcpyAsync(&hst, q->st, sizeof(hst), cudaMemcpyDeviceToHost, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  const bool overflow = hst.overflow != 0;
  hst.cycle = saved_cycle;
  hst.attempts = saved_attempts;
  hst.overflow = 0;
  NW_CUDA(ctx, cudaMemcpyAsync(q->st, &hst, sizeof(hst), cudaMemcpyHostToDevice, q->stream));
  NW_CUDA(ctx, cudaStreamSynchronize(q->stream));
  if (overflow) return qmc_fail(q, NW_ERR_UNSUPPORTED, "spawning attempts exceeded max_attempts");
  return NW_OK;
}

nw_status nw_qmc_destroy(nw_qmc* q) {
  if (!q) return NW_OK;
  cudaSetDevice(q->ctx->device);
  if (q->stream) cudaStreamSynchronize(q->stream);
  release(q);
  return NW_OK;
}

}  // extern "C"
