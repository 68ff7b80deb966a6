// Spin-factorised overlap action y += S x over the resident basis (nw_apply_overlap_device and
// the direct-overlap NOCI-QMC propagator).
//
// The overlap of two determinants is the product of their alpha and beta single-spin overlaps,
// and the determinants of one parent reference share single-spin components (every determinant
// with the same alpha excitation has the same alpha string).  For a target parent Q and a source
// parent P != Q
//     S_{w Omega} = r_w r_Omega A^{QP}[a_w][a_Omega] B^{QP}[b_w][b_Omega],
// A^{QP}[i][j] = det(C_Q[:, occ(i)]^T S_AO C_P[:, occ(j)]) over the ascending occupied columns of
// the two alpha strings (B the same for beta), r = the record's phase times the canonical
// excitation phase of its holes and particles (1 for canonically phased records), so S x is two
// contractions per ordered parent pair (the B-first order of apply_overlap_sparse,
// src/noci/factorise/overlap.rs:434-498, 1276-1360):
//   stage 1  U^{QP}[a][bbar] = sum_{Omega in P, a_Omega = a} r_Omega x_Omega B^{QP}[bbar][b_Omega]
//   stage 2  y_w += r_w sum_{P != Q} sum_a A^{QP}[a_w][a] U^{QP}[a][b_w]
// Determinants of one parent are orthonormal, so the same-parent block adds the sources with
// the same (a, b) pair (the determinant itself in a basis without duplicates).  Per ordered pair
// the work is nnz(x_P) nb_Q + ndet_Q na_P multiply-adds instead of ndet_Q ndet_P overlaps.
//
// Layout: the determinants sorted by (parent, alpha component, beta component); stage 1 takes
// the sorted sources of each alpha component in chunks of at most 32 (a long row, such as the
// parent's own alpha string with every beta string, is spread over many blocks that add into its
// U row) with 256 target beta components per block, reading rows of B^{QP} stored source-major
// (coalesced over bbar) with four independent loads in flight per thread; stage 2 is one thread
// per target in sorted order, reading A^{QP} stored source-major too, so for each source string a
// the lanes of a warp read equal or neighbouring a_w of A and b_w of U (broadcast or coalesced),
// with the (P, a) sum split into segments whose partial sums a finishing kernel adds in a fixed
// order.  No allocation and no host synchronisation per apply,
// so the QMC report block keeps it inside its CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "internal.cuh"
#include "wick_math.cuh"

namespace nw {

// Stage 1 works on chunks of at most kOvlChunk sources of one row (a source alpha component a of
// P for target parent Q): U^{QP}[a][.] is stored by the row's only chunk, or added atomically by
// each chunk of a longer row (whose U row is cleared first).  A block takes a group of consecutive
// chunks of one source parent (at most kOvlGroup sources), staged in shared memory.
struct OvlChunk {
  uint64_t bt;    // B^{QP} (source-major, nb_P x nb_Q) in the factor buffer
  uint64_t urow;  // row a of U^{QP} in the work buffer
  uint32_t t0, t1;  // sorted source positions
  uint32_t atomic;  // the row has several chunks
  uint32_t pad;
};
struct OvlGroup {
  uint32_t c0, c1;  // chunks
  uint32_t t0, t1;  // their sources
};

namespace {

constexpr int kOvlMaxOcc = 16;    // occupied orbitals per spin of the factor kernel
constexpr int kOvlThreads = 256;
constexpr uint64_t kOvlThreadTarget = 148ull * 2048 * 4;  // stage-2 threads to aim for (segments): 4 waves
constexpr uint32_t kOvlChunk = 32;   // sources per stage-1 chunk
constexpr uint32_t kOvlGroup = 64;   // sources per stage-1 block

// One entry of a single-spin factor table per thread; MAXO bounds nocc (the LU scratch lives in
// the thread's stack frame, MAXO^2 doubles).
template <int MAXO>
__global__ void __launch_bounds__(kOvlThreads) ovl_factor_kernel(const double* __restrict__ o, int nmo,
                                                                  const uint8_t* __restrict__ occ_t,
                                                                  const uint8_t* __restrict__ occ_s, int nocc,
                                                                  uint32_t nt, uint32_t ns, int source_major,
                                                                  uint32_t ld, double* __restrict__ out) {
  const uint64_t total = (uint64_t)nt * ns;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    // consecutive threads write consecutive entries of the output row
    const uint32_t i = source_major ? (uint32_t)(e % nt) : (uint32_t)(e / ns);
    const uint32_t j = source_major ? (uint32_t)(e / nt) : (uint32_t)(e % ns);
    const uint8_t* oi = occ_t + (uint64_t)i * nocc;
    const uint8_t* oj = occ_s + (uint64_t)j * nocc;
    double m[MAXO * MAXO];
    for (int r = 0; r < nocc; ++r)
      for (int c = 0; c < nocc; ++c) m[r * nocc + c] = o[(uint64_t)oi[r] * nmo + oj[c]];
    const double d = det_lu_inplace(m, nocc);
    out[source_major ? (uint64_t)j * ld + i : (uint64_t)i * ns + j] = d;
  }
}

__global__ void __launch_bounds__(kOvlThreads) ovl_gather_kernel(uint64_t ndet, const uint32_t* __restrict__ ord_det,
                                                                  const double* __restrict__ ord_r,
                                                                  const double* __restrict__ x,
                                                                  double* __restrict__ xs) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ndet; t += (uint64_t)gridDim.x * blockDim.x)
    xs[t] = ord_r[t] * x[ord_det[t]];
}

// Clears the U rows that several chunks add into (blockIdx.x = row, blockIdx.y = 256 columns).
__global__ void __launch_bounds__(kOvlThreads) ovl_zero_kernel(const uint64_t* __restrict__ urows, uint32_t ldb,
                                                                double* __restrict__ u) {
  const uint32_t b = blockIdx.y * blockDim.x + threadIdx.x;
  if (b < ldb) u[urows[blockIdx.x] + b] = 0.0;
}

// U^{QP}[a][bbar] for the chunks of one group (blockIdx.x) and 512 target beta components
// (blockIdx.y), two neighbouring columns per thread (16-byte loads of rows of B^{QP} padded to an
// even length ldb): every thread sums its columns over the group's staged sources; the loads of
// one chunk are independent (four in flight per step).
__global__ void __launch_bounds__(kOvlThreads) ovl_stage1_kernel(const OvlGroup* __restrict__ groups,
                                                                  const OvlChunk* __restrict__ chunks,
                                                                  const uint32_t* __restrict__ ord_b,
                                                                  const double* __restrict__ xs,
                                                                  const double* __restrict__ fac, uint32_t ldb,
                                                                  double* __restrict__ u) {
  __shared__ double sx[kOvlGroup];
  __shared__ uint32_t sb[kOvlGroup];
  const OvlGroup g = groups[blockIdx.x];
  for (uint32_t i = threadIdx.x; i < g.t1 - g.t0; i += blockDim.x) {
    sx[i] = xs[g.t0 + i];
    sb[i] = ord_b[g.t0 + i];
  }
  __syncthreads();
  const uint32_t col = 2 * (blockIdx.y * blockDim.x + threadIdx.x);
  if (col >= ldb) return;
  for (uint32_t c = g.c0; c < g.c1; ++c) {
    const OvlChunk ch = chunks[c];
    const double* bt = fac + ch.bt + col;
    auto row = [&](uint32_t k) { return __ldg(reinterpret_cast<const double2*>(bt + (uint64_t)sb[k] * ldb)); };
    const uint32_t k1 = ch.t1 - g.t0;
    uint32_t k = ch.t0 - g.t0;
    double2 a0 = make_double2(0.0, 0.0), a1 = a0, a2 = a0, a3 = a0;
    for (; k + 4 <= k1; k += 4) {
      const double2 b0 = row(k), b1 = row(k + 1), b2 = row(k + 2), b3 = row(k + 3);
      a0.x += sx[k] * b0.x;
      a0.y += sx[k] * b0.y;
      a1.x += sx[k + 1] * b1.x;
      a1.y += sx[k + 1] * b1.y;
      a2.x += sx[k + 2] * b2.x;
      a2.y += sx[k + 2] * b2.y;
      a3.x += sx[k + 3] * b3.x;
      a3.y += sx[k + 3] * b3.y;
    }
    for (; k < k1; ++k) {
      const double2 b0 = row(k);
      a0.x += sx[k] * b0.x;
      a0.y += sx[k] * b0.y;
    }
    const double s0 = (a0.x + a1.x) + (a2.x + a3.x), s1 = (a0.y + a1.y) + (a2.y + a3.y);
    double* dst = u + ch.urow + col;
    if (ch.atomic) {
      atomicAdd(dst, s0);
      atomicAdd(dst + 1, s1);
    } else {
      *reinterpret_cast<double2*>(dst) = make_double2(s0, s1);
    }
  }
}

// Partial sums over segment blockIdx.y of the (P, a) index of every target t in [t0, t1) of
// parent q: part[seg][t] = sum A^{qP}[a_t][a] U^{qP}[a][b_t].  A is stored source-major
// (row a holds the na_q targets' strings), so for a fixed a the lanes of a warp read
// neighbouring or equal a_t (one run of a string's targets, or the doubly excited strings one
// target each) as they read neighbouring or equal b_t of U: both loads coalesce or broadcast.
__global__ void __launch_bounds__(kOvlThreads) ovl_stage2_kernel(int q, int nref, uint64_t t0, uint64_t t1,
                                                                  uint64_t seglen, const uint32_t* __restrict__ ord_a,
                                                                  const uint32_t* __restrict__ ord_b,
                                                                  const uint32_t* __restrict__ na,
                                                                  const uint64_t* __restrict__ a_off,
                                                                  const uint64_t* __restrict__ u_off, uint32_t naq,
                                                                  uint32_t ldb, const double* __restrict__ fac,
                                                                  const double* __restrict__ u, uint64_t ndet,
                                                                  double* __restrict__ part) {
  const uint64_t t = t0 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= t1) return;
  const uint64_t k0 = (uint64_t)blockIdx.y * seglen, k1 = k0 + seglen;
  const uint32_t at = ord_a[t], bq = ord_b[t];
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
  uint64_t kbase = 0;
  for (int p = 0; p < nref; ++p) {
    if (p == q) continue;
    const uint64_t n = na[p];
    const uint64_t lo = k0 > kbase ? k0 : kbase;
    const uint64_t hi = k1 < kbase + n ? k1 : kbase + n;
    if (lo < hi) {
      // a = k - kbase runs over [lo - kbase, hi - kbase) of this parent's alpha components
      const double* acol = fac + a_off[(uint64_t)q * nref + p] + at;
      const double* ucol = u + u_off[(uint64_t)q * nref + p] + bq;
      const uint64_t a1 = hi - kbase;
      uint64_t a = lo - kbase;
      for (; a + 4 <= a1; a += 4) {
        const double u0 = __ldg(ucol + a * ldb), u1 = __ldg(ucol + (a + 1) * ldb);
        const double u2 = __ldg(ucol + (a + 2) * ldb), u3 = __ldg(ucol + (a + 3) * ldb);
        acc0 += __ldg(acol + a * naq) * u0;
        acc1 += __ldg(acol + (a + 1) * naq) * u1;
        acc2 += __ldg(acol + (a + 2) * naq) * u2;
        acc3 += __ldg(acol + (a + 3) * naq) * u3;
      }
      for (; a < a1; ++a) acc0 += __ldg(acol + a * naq) * __ldg(ucol + a * ldb);
    }
    kbase += n;
  }
  part[(uint64_t)blockIdx.y * ndet + t] = (acc0 + acc1) + (acc2 + acc3);
}

__global__ void __launch_bounds__(kOvlThreads) ovl_finish_kernel(uint64_t ndet, int nseg, int cross,
                                                                  const uint32_t* __restrict__ ord_det,
                                                                  const double* __restrict__ ord_r,
                                                                  const uint32_t* __restrict__ run_lo,
                                                                  const uint32_t* __restrict__ run_hi,
                                                                  const double* __restrict__ xs,
                                                                  const double* __restrict__ part,
                                                                  double* __restrict__ y) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ndet; t += (uint64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (cross)
      for (int s = 0; s < nseg; ++s) v += part[(uint64_t)s * ndet + t];
    double same = 0.0;
    if (run_lo) {
      for (uint32_t k = run_lo[t]; k < run_hi[t]; ++k) same += xs[k];
    } else {
      same = xs[t];
    }
    y[ord_det[t]] += ord_r[t] * (v + same);
  }
}

inline int grid_of(uint64_t work) {
  const uint64_t g = (work + kOvlThreads - 1) / kOvlThreads;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 16));
}

// Fermionic sign of the excitation (excitation_phase_bits, src/basis/excitation.rs:110-146):
// holes removed from the highest down, particles added from the lowest up, each contributing
// the parity of the occupied orbitals below it.
double excitation_sign(int nocc, int rank, const uint8_t* idx) {
  char occ[256] = {};  // orbital indices are bytes
  for (int i = 0; i < nocc && i < 256; ++i) occ[i] = 1;
  auto below = [&](int p) {
    int c = 0;
    for (int i = 0; i < p; ++i) c += occ[i];
    return c & 1;
  };
  int odd = 0;
  for (int k = rank - 1; k >= 0; --k) {
    odd ^= below(idx[k]);
    occ[idx[k]] = 0;
  }
  for (int k = 0; k < rank; ++k) {
    odd ^= below(idx[4 + k]);
    if (k + 1 != rank) occ[idx[4 + k]] = 1;
  }
  return odd ? -1.0 : 1.0;
}

using SpinKey = std::pair<int, uint64_t>;

SpinKey spin_key(int rank, const uint8_t* idx) {
  uint64_t v = 0;
  for (int k = 0; k < rank; ++k) {
    v |= (uint64_t)idx[k] << (8 * k);
    v |= (uint64_t)idx[4 + k] << (8 * (4 + k));
  }
  return {rank, v};
}

}  // namespace

struct OverlapPlan {
  int nref = 0, oa = 0, ob = 0;
  uint64_t ndet = 0;
  int nseg = 1;
  std::vector<uint32_t> na, nb;
  std::vector<uint32_t> ldb;            // beta strings per parent rounded up to even: row stride of B and U
  std::vector<uint64_t> pstart;         // per parent: first sorted position (nref + 1)
  std::vector<uint64_t> ngroups, groups_off;  // per target parent: stage-1 groups
  std::vector<uint64_t> nzero, zero_off;      // per target parent: U rows cleared before stage 1
  std::vector<uint64_t> seglen;         // per target parent
  void* mem = nullptr;
  uint32_t* ord_det = nullptr;
  uint32_t* ord_a = nullptr;
  uint32_t* ord_b = nullptr;
  double* ord_r = nullptr;
  uint32_t* run_lo = nullptr;  // null when every (parent, a, b) is a single determinant
  uint32_t* run_hi = nullptr;
  OvlGroup* groups = nullptr;
  OvlChunk* chunks = nullptr;
  uint64_t* zero_rows = nullptr;
  uint64_t* d_a_off = nullptr;
  uint64_t* d_u_off = nullptr;
  uint32_t* d_na = nullptr;
  double* fac = nullptr;
  double* u = nullptr;
  double* xs = nullptr;
  double* part = nullptr;
};

void overlap_plan_free(OverlapPlan* pl) {
  if (!pl) return;
  if (pl->mem) cudaFree(pl->mem);
  delete pl;
}

nw_status overlap_plan_get(nw_ctx* ctx, cudaStream_t stream, OverlapPlan** out) {
  if (ctx->ovl) {
    *out = ctx->ovl;
    return NW_OK;
  }
  if (!ctx->d_dets || ctx->ndet == 0) return fail(ctx, NW_ERR_STATE, "the overlap action needs a resident basis");
  if (ctx->nocc_a > kOvlMaxOcc || ctx->nocc_b > kOvlMaxOcc)
    return fail(ctx, NW_ERR_UNSUPPORTED, "the overlap action supports at most 16 occupied orbitals per spin");
  const int nref = ctx->nref, nmo = ctx->nmo, nao = ctx->nao;
  const uint64_t nd = ctx->ndet;
  std::vector<nw_det> dets(nd);
  NW_CUDA(ctx, cudaMemcpyAsync(dets.data(), ctx->d_dets, nd * sizeof(nw_det), cudaMemcpyDeviceToHost, stream));
  NW_CUDA(ctx, cudaStreamSynchronize(stream));

  OverlapPlan* pl = new (std::nothrow) OverlapPlan;
  if (!pl) return NW_ERR_ALLOC;
  pl->nref = nref;
  pl->oa = ctx->nocc_a;
  pl->ob = ctx->nocc_b;
  pl->ndet = nd;
  // parent-local single-spin components
  std::vector<std::map<SpinKey, uint32_t>> ca(nref), cb(nref);
  std::vector<uint32_t> aid(nd), bid(nd);
  std::vector<double> rr(nd);
  for (uint64_t d = 0; d < nd; ++d) {
    const nw_det& r = dets[d];
    const SpinKey ka = spin_key(r.rank_a, r.idx_a), kb = spin_key(r.rank_b, r.idx_b);
    auto ia = ca[r.parent].emplace(ka, (uint32_t)ca[r.parent].size()).first;
    auto ib = cb[r.parent].emplace(kb, (uint32_t)cb[r.parent].size()).first;
    aid[d] = ia->second;
    bid[d] = ib->second;
    rr[d] = r.phase * excitation_sign(ctx->nocc_a, r.rank_a, r.idx_a) * excitation_sign(ctx->nocc_b, r.rank_b, r.idx_b);
  }
  pl->na.resize(nref);
  pl->nb.resize(nref);
  pl->ldb.resize(nref);
  std::vector<uint64_t> ca_off(nref + 1, 0), cb_off(nref + 1, 0);
  for (int p = 0; p < nref; ++p) {
    pl->na[p] = (uint32_t)ca[p].size();
    pl->nb[p] = (uint32_t)cb[p].size();
    pl->ldb[p] = (pl->nb[p] + 1) & ~1u;
    ca_off[p + 1] = ca_off[p] + pl->na[p];
    cb_off[p + 1] = cb_off[p] + pl->nb[p];
  }
  // occupied orbitals of every component, ascending
  std::vector<uint8_t> occ_a(std::max<uint64_t>(1, ca_off[nref] * pl->oa)), occ_b(std::max<uint64_t>(1, cb_off[nref] * pl->ob));
  auto fill_occ = [&](const SpinKey& k, int nocc, uint8_t* dst) {
    const int rank = k.first;
    std::vector<int> o;
    for (int i = 0; i < nocc; ++i) {
      bool hole = false;
      for (int h = 0; h < rank; ++h) hole |= ((k.second >> (8 * h)) & 0xFF) == (uint64_t)i;
      if (!hole) o.push_back(i);
    }
    for (int h = 0; h < rank; ++h) o.push_back((int)((k.second >> (8 * (4 + h))) & 0xFF));
    std::sort(o.begin(), o.end());
    for (int i = 0; i < nocc; ++i) dst[i] = (uint8_t)o[i];
  };
  for (int p = 0; p < nref; ++p) {
    for (const auto& kv : ca[p]) fill_occ(kv.first, pl->oa, occ_a.data() + (ca_off[p] + kv.second) * pl->oa);
    for (const auto& kv : cb[p]) fill_occ(kv.first, pl->ob, occ_b.data() + (cb_off[p] + kv.second) * pl->ob);
  }
  // sorted order (parent, a, b)
  std::vector<uint32_t> order(nd);
  for (uint64_t d = 0; d < nd; ++d) order[d] = (uint32_t)d;
  std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
    if (dets[x].parent != dets[y].parent) return dets[x].parent < dets[y].parent;
    if (aid[x] != aid[y]) return aid[x] < aid[y];
    if (bid[x] != bid[y]) return bid[x] < bid[y];
    return x < y;
  });
  std::vector<uint32_t> o_a(nd), o_b(nd), run_lo(nd), run_hi(nd);
  std::vector<double> o_r(nd);
  std::vector<uint64_t> rowstart(ca_off[nref] + 1, 0);
  pl->pstart.assign(nref + 1, nd);
  bool dups = false;
  for (uint64_t t = 0; t < nd; ++t) {
    const uint32_t d = order[t];
    const uint32_t p = dets[d].parent;
    o_a[t] = aid[d];
    o_b[t] = bid[d];
    o_r[t] = rr[d];
    if (t == 0 || dets[order[t - 1]].parent != p) pl->pstart[p] = t;
    if (t == 0 || dets[order[t - 1]].parent != p || aid[order[t - 1]] != aid[d]) rowstart[ca_off[p] + aid[d]] = t;
  }
  rowstart[ca_off[nref]] = nd;
  for (int p = nref - 1; p >= 0; --p)
    if (pl->pstart[p] > pl->pstart[p + 1]) pl->pstart[p] = pl->pstart[p + 1];  // parents without determinants
  for (uint64_t t = 0; t < nd;) {
    uint64_t e = t + 1;
    while (e < nd && dets[order[e]].parent == dets[order[t]].parent && o_a[e] == o_a[t] && o_b[e] == o_b[t]) ++e;
    if (e - t > 1) dups = true;
    for (uint64_t k = t; k < e; ++k) {
      run_lo[k] = (uint32_t)t;
      run_hi[k] = (uint32_t)e;
    }
    t = e;
  }
  // factor tables, U offsets and stage-1 rows
  std::vector<uint64_t> a_off((size_t)nref * nref, 0), bt_off((size_t)nref * nref, 0), u_off((size_t)nref * nref, 0);
  uint64_t nfac = 0, nu = 0;
  std::vector<OvlGroup> groups;
  std::vector<OvlChunk> chunks;
  std::vector<uint64_t> zero_rows;
  pl->ngroups.assign(nref, 0);
  pl->groups_off.assign(nref, 0);
  pl->nzero.assign(nref, 0);
  pl->zero_off.assign(nref, 0);
  pl->seglen.assign(nref, 1);
  uint64_t max_targets = 1;
  for (int q = 0; q < nref; ++q) max_targets = std::max<uint64_t>(max_targets, pl->pstart[q + 1] - pl->pstart[q]);
  pl->nseg = (int)std::max<uint64_t>(1, std::min<uint64_t>(64, (kOvlThreadTarget + max_targets - 1) / max_targets));
  for (int q = 0; q < nref; ++q) {
    uint64_t uq = 0, kq = 0;
    pl->groups_off[q] = groups.size();
    pl->zero_off[q] = zero_rows.size();
    for (int p = 0; p < nref; ++p) {
      if (p == q) continue;
      const size_t i = (size_t)q * nref + p;
      a_off[i] = nfac;
      nfac += (uint64_t)pl->na[q] * pl->na[p];
      nfac = (nfac + 1) & ~1ull;  // 16-byte aligned rows of B
      bt_off[i] = nfac;
      nfac += (uint64_t)pl->nb[p] * pl->ldb[q];
      u_off[i] = uq;
      // chunks of the rows of P in sorted order, grouped (a group never spans two parents)
      bool open = false;
      for (uint32_t a = 0; a < pl->na[p]; ++a) {
        const uint64_t r0 = rowstart[ca_off[p] + a], r1 = rowstart[ca_off[p] + a + 1];
        const uint64_t urow = uq + (uint64_t)a * pl->ldb[q];
        const bool multi = r1 - r0 > kOvlChunk;
        if (multi) zero_rows.push_back(urow);
        for (uint64_t c0 = r0; c0 < r1; c0 += kOvlChunk) {
          const uint64_t c1 = std::min<uint64_t>(r1, c0 + kOvlChunk);
          if (!open || c1 - groups.back().t0 > kOvlGroup) {
            groups.push_back(OvlGroup{(uint32_t)chunks.size(), (uint32_t)chunks.size(), (uint32_t)c0, (uint32_t)c0});
            open = true;
          }
          chunks.push_back(OvlChunk{bt_off[i], urow, (uint32_t)c0, (uint32_t)c1, multi ? 1u : 0u, 0u});
          groups.back().c1 = (uint32_t)chunks.size();
          groups.back().t1 = (uint32_t)c1;
        }
      }
      uq += (uint64_t)pl->na[p] * pl->ldb[q];
      kq += pl->na[p];
    }
    pl->ngroups[q] = groups.size() - pl->groups_off[q];
    pl->nzero[q] = zero_rows.size() - pl->zero_off[q];
    pl->seglen[q] = std::max<uint64_t>(1, (kq + pl->nseg - 1) / pl->nseg);
    nu = std::max(nu, uq);
  }
  // one allocation: device arrays, factor tables, work buffers and the MO overlaps of the set-up
  const size_t n2 = (size_t)nmo * nmo;
  const size_t nrr = (size_t)nref * nref;
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) & ~(size_t)255;
    return at;
  };
  const size_t o_det = carve(nd * 4), o_a_ = carve(nd * 4), o_b_ = carve(nd * 4), o_r_ = carve(nd * 8);
  const size_t o_lo = dups ? carve(nd * 4) : 0, o_hi = dups ? carve(nd * 4) : 0;
  const size_t o_groups = carve(std::max<size_t>(1, groups.size()) * sizeof(OvlGroup));
  const size_t o_chunks = carve(std::max<size_t>(1, chunks.size()) * sizeof(OvlChunk));
  const size_t o_zero = carve(std::max<size_t>(1, zero_rows.size()) * 8);
  const size_t o_aoff = carve(nrr * 8), o_uoff = carve(nrr * 8), o_na = carve(nref * 4);
  const size_t o_occa = carve(occ_a.size()), o_occb = carve(occ_b.size());
  const size_t o_fac = carve(std::max<uint64_t>(1, nfac) * 8), o_u = carve(std::max<uint64_t>(1, nu) * 8);
  const size_t o_xs = carve(nd * 8), o_part = carve((size_t)pl->nseg * nd * 8);
  const size_t o_t = carve((size_t)nref * nao * nmo * 8), o_o = carve(2 * nrr * n2 * 8);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && off > free_b) {
    overlap_plan_free(pl);
    return fail(ctx, NW_ERR_ALLOC,
                "the overlap factor tables need " + std::to_string(off >> 20) + " MiB, more than the free device memory");
  }
  if (cudaMalloc(&pl->mem, off) != cudaSuccess) {
    pl->mem = nullptr;
    overlap_plan_free(pl);
    return fail(ctx, NW_ERR_ALLOC, "overlap factor table allocation failed");
  }
  char* base = static_cast<char*>(pl->mem);
  pl->ord_det = reinterpret_cast<uint32_t*>(base + o_det);
  pl->ord_a = reinterpret_cast<uint32_t*>(base + o_a_);
  pl->ord_b = reinterpret_cast<uint32_t*>(base + o_b_);
  pl->ord_r = reinterpret_cast<double*>(base + o_r_);
  pl->run_lo = dups ? reinterpret_cast<uint32_t*>(base + o_lo) : nullptr;
  pl->run_hi = dups ? reinterpret_cast<uint32_t*>(base + o_hi) : nullptr;
  pl->groups = reinterpret_cast<OvlGroup*>(base + o_groups);
  pl->chunks = reinterpret_cast<OvlChunk*>(base + o_chunks);
  pl->zero_rows = reinterpret_cast<uint64_t*>(base + o_zero);
  pl->d_a_off = reinterpret_cast<uint64_t*>(base + o_aoff);
  pl->d_u_off = reinterpret_cast<uint64_t*>(base + o_uoff);
  pl->d_na = reinterpret_cast<uint32_t*>(base + o_na);
  uint8_t* d_occa = reinterpret_cast<uint8_t*>(base + o_occa);
  uint8_t* d_occb = reinterpret_cast<uint8_t*>(base + o_occb);
  pl->fac = reinterpret_cast<double*>(base + o_fac);
  pl->u = reinterpret_cast<double*>(base + o_u);
  pl->xs = reinterpret_cast<double*>(base + o_xs);
  pl->part = reinterpret_cast<double*>(base + o_part);
  double* d_t = reinterpret_cast<double*>(base + o_t);
  double* d_o = reinterpret_cast<double*>(base + o_o);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes == 0 || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream) == cudaSuccess;
  };
  // the padding column of an odd-length B row is summed by stage 1 into a U column nobody reads
  bool ok = cudaMemsetAsync(pl->fac, 0, std::max<uint64_t>(1, nfac) * 8, stream) == cudaSuccess &&
            up(pl->ord_det, order.data(), nd * 4) && up(pl->ord_a, o_a.data(), nd * 4) &&
            up(pl->ord_b, o_b.data(), nd * 4) && up(pl->ord_r, o_r.data(), nd * 8) &&
            up(pl->groups, groups.data(), groups.size() * sizeof(OvlGroup)) &&
            up(pl->chunks, chunks.data(), chunks.size() * sizeof(OvlChunk)) &&
            up(pl->zero_rows, zero_rows.data(), zero_rows.size() * 8) &&
            up(pl->d_a_off, a_off.data(), nrr * 8) && up(pl->d_u_off, u_off.data(), nrr * 8) &&
            up(pl->d_na, pl->na.data(), nref * 4) && up(d_occa, occ_a.data(), occ_a.size()) &&
            up(d_occb, occ_b.data(), occ_b.size());
  if (ok && dups) ok = up(pl->run_lo, run_lo.data(), nd * 4) && up(pl->run_hi, run_hi.data(), nd * 4);
  // O^{QP}_sigma = C_Q^T (S C_P): nmo x nmo per ordered pair and spin, then the factor tables
  for (int spin = 0; ok && spin < 2 && nref > 1; ++spin) {
    const double* c = spin ? ctx->d_cb : ctx->d_ca;
    const long long cs = (long long)nao * nmo;
    ok = dgemm_strided(stream, false, false, nao, nmo, nao, 1.0, ctx->d_s, nao, 0, c, nmo, cs, 0.0, d_t, nmo, cs,
                       nref) == cudaSuccess;
    for (int q = 0; ok && q < nref; ++q)
      ok = dgemm_strided(stream, true, false, nmo, nmo, nao, 1.0, c + q * cs, nmo, 0, d_t, nmo, cs, 0.0,
                         d_o + ((size_t)spin * nrr + (size_t)q * nref) * n2, nmo, (long long)n2, nref) == cudaSuccess;
  }
  auto factors = [&](const double* o, const uint8_t* ot, const uint8_t* os, int nocc, uint32_t nt, uint32_t ns,
                     uint32_t ld, double* out) {
    const uint64_t e = (uint64_t)nt * ns;
    if (e == 0) return;
    if (nocc <= 4)
      ovl_factor_kernel<4><<<grid_of(e), kOvlThreads, 0, stream>>>(o, nmo, ot, os, nocc, nt, ns, 1, ld, out);
    else if (nocc <= 8)
      ovl_factor_kernel<8><<<grid_of(e), kOvlThreads, 0, stream>>>(o, nmo, ot, os, nocc, nt, ns, 1, ld, out);
    else
      ovl_factor_kernel<kOvlMaxOcc><<<grid_of(e), kOvlThreads, 0, stream>>>(o, nmo, ot, os, nocc, nt, ns, 1, ld, out);
  };
  for (int q = 0; ok && q < nref; ++q)
    for (int p = 0; ok && p < nref; ++p) {
      if (p == q) continue;
      const size_t i = (size_t)q * nref + p;
      factors(d_o + i * n2, d_occa + ca_off[q] * pl->oa, d_occa + ca_off[p] * pl->oa, pl->oa, pl->na[q], pl->na[p],
              pl->na[q], pl->fac + a_off[i]);
      factors(d_o + (nrr + i) * n2, d_occb + cb_off[q] * pl->ob, d_occb + cb_off[p] * pl->ob, pl->ob, pl->nb[q],
              pl->nb[p], pl->ldb[q], pl->fac + bt_off[i]);
      ok = cudaGetLastError() == cudaSuccess;
    }
  if (ok) ok = cudaStreamSynchronize(stream) == cudaSuccess;
  if (!ok) {
    overlap_plan_free(pl);
    return fail(ctx, NW_ERR_CUDA, "overlap factor table set-up failed");
  }
  ctx->ovl = pl;
  *out = pl;
  return NW_OK;
}

nw_status overlap_apply(nw_ctx* ctx, const OverlapPlan* pl, const double* x, double* y, cudaStream_t stream) {
  const uint64_t nd = pl->ndet;
  ovl_gather_kernel<<<grid_of(nd), kOvlThreads, 0, stream>>>(nd, pl->ord_det, pl->ord_r, x, pl->xs);
  const int cross = pl->nref > 1 ? 1 : 0;
  for (int q = 0; cross && q < pl->nref; ++q) {
    const uint64_t t0 = pl->pstart[q], t1 = pl->pstart[q + 1];
    if (t1 == t0) continue;
    const uint32_t ldb = pl->ldb[q];
    if (pl->nzero[q] > 0)
      ovl_zero_kernel<<<dim3((unsigned)pl->nzero[q], (ldb + kOvlThreads - 1) / kOvlThreads), kOvlThreads, 0, stream>>>(
          pl->zero_rows + pl->zero_off[q], ldb, pl->u);
    if (pl->ngroups[q] > 0)
      ovl_stage1_kernel<<<dim3((unsigned)pl->ngroups[q], (ldb + 2 * kOvlThreads - 1) / (2 * kOvlThreads)), kOvlThreads, 0,
                          stream>>>(pl->groups + pl->groups_off[q], pl->chunks, pl->ord_b, pl->xs, pl->fac, ldb, pl->u);
    const dim3 g2((unsigned)((t1 - t0 + kOvlThreads - 1) / kOvlThreads), (unsigned)pl->nseg);
    ovl_stage2_kernel<<<g2, kOvlThreads, 0, stream>>>(q, pl->nref, t0, t1, pl->seglen[q], pl->ord_a, pl->ord_b,
                                                      pl->d_na, pl->d_a_off, pl->d_u_off, pl->na[q], ldb, pl->fac,
                                                      pl->u, nd,
                                                      pl->part);
  }
  ovl_finish_kernel<<<grid_of(nd), kOvlThreads, 0, stream>>>(nd, pl->nseg, cross, pl->ord_det, pl->ord_r, pl->run_lo,
                                                             pl->run_hi, pl->xs, pl->part, y);
  NW_CUDA(ctx, cudaGetLastError());
  return NW_OK;
}

}  // namespace nw

extern "C" {

nw_status nw_apply_overlap_device(nw_ctx* ctx, const double* x_dev, double* y_dev, void* stream) {
  if (!ctx || !x_dev || !y_dev) return NW_ERR_INVALID;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  nw::CtxGuard guard(ctx, s);
  NW_CUDA(ctx, cudaSetDevice(ctx->device));
  nw::OverlapPlan* pl = nullptr;
  const nw_status st = nw::overlap_plan_get(ctx, s, &pl);
  if (st != NW_OK) return st;
  return nw::overlap_apply(ctx, pl, x_dev, y_dev, s);
}

}  // extern "C"
