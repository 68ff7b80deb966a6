// CPU oracle (test infrastructure only): lane-batched restatement of the reference's
// fixed-rank SIMD Wick path, the timed CPU baseline of bench.py.  The product library never
// links it.
//
// What it restates (file:line inside dy-cl/noci-rs):
//   * calculate_hs_pairs_wicks_batched                  src/noci/hs.rs:72-130
//       same-parent shortcuts, then one group per ordered reference pair
//   * xw_hamiltonian_overlap_prepared_batched           src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:121-362
//       for m_alpha = m_beta = 0: requests whose spin ranks are all <= 4 and L_alpha + L_beta <= 6
//       go to one of 28 bins, bin = L_alpha (15 - L_alpha) / 2 + L_beta; a full bin (8 lanes with
//       AVX-512, 4 with AVX2 + FMA) is flushed through the fixed (L_alpha, L_beta) kernel; at the
//       end partial bins are padded with their first request; every other request (and every
//       request of an m > 0 reference pair) goes to the scalar generic evaluator
//   * xw_hamiltonian_overlap_m0_{LaLb}_prepared_f64x8   preparehamiltonianoverlap.rs:1001-20300
//       (structure as m0_22, :10027-10300): per lane contraction labels from the excitation
//       caches, D gathered from X0 (i >= j) / Y0 (i < j), determinant, cofactors and second
//       minors vertically across lanes, replacement = sum cof[eta,z] hcol0[c_z, r_eta],
//       J = sum over eta < xi, z < y of (+-) minor * (J[r_eta c_z r_xi c_y] - J[r_eta c_y r_xi c_z]),
//       II = sum cof_a[eta,z] sum cof_b[xi,y] II[r_eta c_z | r_xi c_y], and
//       H = pref (g0 det_a det_b - det_b repl_a - det_a repl_b + J_a det_b + J_b det_a + II)
//       with g0 = E_nuc + F0h_a + V0_a / 2 + F0h_b + V0_b / 2 + V_ab0, S = pref det_a det_b.
// The fixed kernels of the reference are written out by hand per rank pair; here one template
// over (L_alpha, L_beta) generates them, with the determinant algebra as Laplace expansions on
// lane vectors.  The file is compiled twice, with ORC_LANES = 8 (x86-64-v4, AVX-512) and
// ORC_LANES = 4 (x86-64-v3, AVX2 + FMA); wick_eval.cpp picks the widest the host supports at
// run time, as the reference does with is_x86_feature_detected.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "wick_oracle.h"

#ifndef ORC_LANES
#error "ORC_LANES must be 4 or 8"
#endif

#define ORC_CAT2(a, b) a##b
#define ORC_CAT(a, b) ORC_CAT2(a, b)
#define ORC_NS ORC_CAT(binned, ORC_LANES)

namespace orc {
namespace ORC_NS {

constexpr int W = ORC_LANES;
typedef double vd __attribute__((vector_size(8 * W)));

inline vd splat(double x) {
  vd z = {};
  return z + x;
}

template <int N>
struct Sz {
  static constexpr int v = N > 0 ? N : 1;
};

// Determinant of an N x N lane matrix (row-major) by Laplace expansion along the first row.
template <int N>
inline vd det_n(const vd* a) {
  if constexpr (N == 0) {
    return splat(1.0);
  } else if constexpr (N == 1) {
    return a[0];
  } else if constexpr (N == 2) {
    return a[0] * a[3] - a[1] * a[2];
  } else if constexpr (N == 3) {
    return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
           a[2] * (a[3] * a[7] - a[4] * a[6]);
  } else {
    vd acc = {};
    vd mn[(N - 1) * (N - 1)];
    for (int c = 0; c < N; ++c) {
      int k = 0;
      for (int i = 1; i < N; ++i)
        for (int j = 0; j < N; ++j)
          if (j != c) mn[k++] = a[i * N + j];
      const vd t = a[c] * det_n<N - 1>(mn);
      acc = (c & 1) ? acc - t : acc + t;
    }
    return acc;
  }
}

// Determinant of `a` (L x L) with rows r0, r1 and columns c0, c1 removed (r1 = c1 = -1 for a
// single row and column).
template <int L, int K>
inline vd minor_det(const vd* a, int r0, int r1, int c0, int c1) {
  if constexpr (K == 0) return splat(1.0);
  vd mn[Sz<K * K>::v] = {};
  int k = 0;
  for (int i = 0; i < L; ++i) {
    if (i == r0 || i == r1) continue;
    for (int j = 0; j < L; ++j) {
      if (j == c0 || j == c1) continue;
      mn[k++] = a[i * L + j];
    }
  }
  return det_n<K>(mn);
}

// One spin of one flush: labels, D, determinant, cofactors, replacement and J terms.
template <int L>
struct SpinLanes {
  int rows[W][Sz<L>::v], cols[W][Sz<L>::v];
  vd cof[Sz<L * L>::v];
  vd det, repl, jterm;
};

template <int L>
inline void spin_lanes(const SpinView& v, const Det* const* xs, const Det* const* ws, int spin, SpinLanes<L>& o) {
  const int nocc = v.nocc, n = v.nmo, nvirt = n - nocc;
  // contraction labels (prepare.rs:555-595): x particles a - nocc / x holes i, then
  // w holes nvirt + j / w particles b
  for (int l = 0; l < W; ++l) {
    const Det& x = *xs[l];
    const Det& w = *ws[l];
    const int xr = spin ? x.rank_b : x.rank_a;
    const uint8_t* xh = spin ? x.holes_b : x.holes_a;
    const uint8_t* xp = spin ? x.parts_b : x.parts_a;
    const uint8_t* wh = spin ? w.holes_b : w.holes_a;
    const uint8_t* wp = spin ? w.parts_b : w.parts_a;
    for (int i = 0; i < L; ++i) {
      if (i < xr) {
        o.rows[l][i] = (int)xp[i] - nocc;
        o.cols[l][i] = xh[i];
      } else {
        o.rows[l][i] = nvirt + (int)wh[i - xr];
        o.cols[l][i] = wp[i - xr];
      }
    }
  }
  if constexpr (L == 0) {
    o.det = splat(1.0);
    o.repl = vd{};
    o.jterm = vd{};
    return;
  } else {
    vd d[L * L];
    for (int i = 0; i < L; ++i)
      for (int j = 0; j < L; ++j) {
        const double* src = i >= j ? v.x[0] : v.y[0];
        double lane[W];
        for (int l = 0; l < W; ++l) lane[l] = src[(int64_t)o.rows[l][i] * n + o.cols[l][j]];
        vd t;
        for (int l = 0; l < W; ++l) t[l] = lane[l];
        d[i * L + j] = t;
      }
    if constexpr (L == 1) {
      o.cof[0] = splat(1.0);
      o.det = d[0];
    } else {
      for (int r = 0; r < L; ++r)
        for (int c = 0; c < L; ++c) {
          const vd m = minor_det<L, L - 1>(d, r, -1, c, -1);
          o.cof[r * L + c] = ((r + c) & 1) ? -m : m;
        }
      vd det = {};
      for (int c = 0; c < L; ++c) det += d[c] * o.cof[c];
      o.det = det;
    }
    // replacement = sum_{z, eta} cof[eta, z] hcol0[c_z][r_eta] (hcol0 stored transposed)
    vd repl = {};
    for (int z = 0; z < L; ++z)
      for (int e = 0; e < L; ++e) {
        vd t;
        for (int l = 0; l < W; ++l) t[l] = v.hcol0_t[(int64_t)o.cols[l][z] * n + o.rows[l][e]];
        repl += o.cof[e * L + z] * t;
      }
    o.repl = repl;
    vd jt = {};
    if constexpr (L >= 2) {
      const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
      const double* jsl = v.j[0];
      for (int e = 0; e < L; ++e)
        for (int x = e + 1; x < L; ++x)
          for (int z = 0; z < L; ++z)
            for (int y = z + 1; y < L; ++y) {
              vd dir = {}, exc = {};
              for (int l = 0; l < W; ++l) {
                const int64_t base = (int64_t)o.rows[l][e] * n3 + (int64_t)o.rows[l][x] * n;
                dir[l] = jsl[base + (int64_t)o.cols[l][z] * n2 + o.cols[l][y]];
                exc[l] = jsl[base + (int64_t)o.cols[l][y] * n2 + o.cols[l][z]];
              }
              const vd t = minor_det<L, L - 2>(d, e, x, z, y) * (dir - exc);
              jt = ((e + x + z + y) & 1) ? jt - t : jt + t;
            }
    }
    o.jterm = jt;
  }
}

// The fixed (L_alpha, L_beta) kernel over W requests of one reference pair.
template <int LA, int LB>
void flush(const PairView& pv, const Det* const* xs, const Det* const* ws, const double* exc, double enuc, double* h,
           double* s) {
  SpinLanes<LA> a;
  SpinLanes<LB> b;
  spin_lanes<LA>(pv.aa, xs, ws, 0, a);
  spin_lanes<LB>(pv.bb, xs, ws, 1, b);
  vd ii = {};
  if constexpr (LA > 0 && LB > 0) {
    const int n = pv.ab.nmo;
    const double* iisl = pv.ab.ii[0][0][0][0];
    for (int z = 0; z < LA; ++z)
      for (int e = 0; e < LA; ++e) {
        vd inner = {};
        for (int y = 0; y < LB; ++y)
          for (int x = 0; x < LB; ++x) {
            vd t;
            for (int l = 0; l < W; ++l)
              t[l] = iisl[(((int64_t)a.rows[l][e] * n + a.cols[l][z]) * n + b.rows[l][x]) * n + b.cols[l][y]];
            inner += b.cof[x * LB + y] * t;
          }
        ii += a.cof[e * LA + z] * inner;
      }
  }
  const double g0 = enuc + pv.aa.f0h[0] + 0.5 * pv.aa.v0[0] + pv.bb.f0h[0] + 0.5 * pv.bb.v0[0] + pv.ab.vab0[0][0];
  const vd det_ab = a.det * b.det;
  vd core = splat(g0) * det_ab;
  core -= b.det * a.repl;
  core -= a.det * b.repl;
  core += a.jterm * b.det;
  core += b.jterm * a.det;
  core += ii;
  const double ref_pref = pv.aa.phase * pv.aa.tsp * pv.bb.phase * pv.bb.tsp;
  vd ph;
  for (int l = 0; l < W; ++l) ph[l] = exc[l];
  const vd pref = ph * ref_pref;
  const vd hv = core * pref, sv = det_ab * pref;
  for (int l = 0; l < W; ++l) {
    h[l] = hv[l];
    s[l] = sv[l];
  }
}

typedef void (*FlushFn)(const PairView&, const Det* const*, const Det* const*, const double*, double, double*,
                        double*);

template <int LA, int LB>
constexpr FlushFn fn() {
  return &flush<LA, LB>;
}

// bin = la (15 - la) / 2 + lb for la + lb <= 6
constexpr FlushFn kFlush[28] = {
    fn<0, 0>(), fn<0, 1>(), fn<0, 2>(), fn<0, 3>(), fn<0, 4>(), fn<0, 5>(), fn<0, 6>(),
    fn<1, 0>(), fn<1, 1>(), fn<1, 2>(), fn<1, 3>(), fn<1, 4>(), fn<1, 5>(),
    fn<2, 0>(), fn<2, 1>(), fn<2, 2>(), fn<2, 3>(), fn<2, 4>(),
    fn<3, 0>(), fn<3, 1>(), fn<3, 2>(), fn<3, 3>(),
    fn<4, 0>(), fn<4, 1>(), fn<4, 2>(),
    fn<5, 0>(), fn<5, 1>(),
    fn<6, 0>()};

struct Bin {
  const Det* x[W];
  const Det* w[W];
  double ph[W];
  int64_t out[W];
  int n;
};

// xw_hamiltonian_overlap_prepared_batched for the requests `idx` of one ordered reference pair.
void batched_group(const Ctx& c, const PairView& pv, const int64_t* pairs, const int64_t* idx, int64_t nidx,
                   double* h_out, double* s_out) {
  if (pv.aa.m != 0 || pv.bb.m != 0) {
    for (int64_t k = 0; k < nidx; ++k) {
      const int64_t i = idx[k];
      eval_wick_pair(c, c.basis[pairs[2 * i]], c.basis[pairs[2 * i + 1]], &h_out[i], &s_out[i]);
    }
    return;
  }
  Bin bins[28];
  for (Bin& b : bins) b.n = 0;
  double hh[W], ss[W];
  for (int64_t k = 0; k < nidx; ++k) {
    const int64_t i = idx[k];
    const Det& x = c.basis[pairs[2 * i]];
    const Det& w = c.basis[pairs[2 * i + 1]];
    const bool fixed = x.rank_a <= 4 && x.rank_b <= 4 && w.rank_a <= 4 && w.rank_b <= 4;
    const int la = x.rank_a + w.rank_a, lb = x.rank_b + w.rank_b;
    if (fixed && la + lb <= 6) {
      const int bi = la * (15 - la) / 2 + lb;
      Bin& b = bins[bi];
      b.x[b.n] = &x;
      b.w[b.n] = &w;
      b.ph[b.n] = (x.pha * w.pha) * (x.phb * w.phb);
      b.out[b.n] = i;
      if (++b.n == W) {
        kFlush[bi](pv, b.x, b.w, b.ph, c.enuc, hh, ss);
        for (int l = 0; l < W; ++l) {
          h_out[b.out[l]] = hh[l];
          s_out[b.out[l]] = ss[l];
        }
        b.n = 0;
      }
    } else {
      eval_wick_pair(c, x, w, &h_out[i], &s_out[i]);
    }
  }
  for (int bi = 0; bi < 28; ++bi) {
    Bin& b = bins[bi];
    if (b.n == 0) continue;
    for (int l = b.n; l < W; ++l) {
      b.x[l] = b.x[0];
      b.w[l] = b.w[0];
      b.ph[l] = b.ph[0];
    }
    kFlush[bi](pv, b.x, b.w, b.ph, c.enuc, hh, ss);
    for (int l = 0; l < b.n; ++l) {
      h_out[b.out[l]] = hh[l];
      s_out[b.out[l]] = ss[l];
    }
  }
}

}  // namespace ORC_NS

// calculate_hs_pairs_wicks_batched over the requests [i0, i1): same-parent shortcuts, one group
// per ordered reference pair (hs.rs:86-109), then the batched evaluator per group.
void ORC_CAT(hs_pairs_batched, ORC_LANES)(const Ctx& c, const int64_t* pairs, int64_t i0, int64_t i1, double* h_out,
                                          double* s_out) {
  const int ng = c.nref * c.nref;
  std::vector<int64_t> count(ng + 1, 0), order((size_t)(i1 - i0));
  std::vector<int> grp((size_t)(i1 - i0), -1);
  for (int64_t i = i0; i < i1; ++i) {
    const Det& x = c.basis[pairs[2 * i]];
    const Det& w = c.basis[pairs[2 * i + 1]];
    if (x.parent == w.parent) {
      if (popcount128(x.occ_a, w.occ_a) + popcount128(x.occ_b, w.occ_b) > 4) {
        h_out[i] = 0.0;
        s_out[i] = 0.0;
        continue;
      }
      if (c.mo_offs != nullptr && c.mo_orth[x.parent]) {
        hs_orthogonal(c, x, w, &h_out[i], &s_out[i]);
        continue;
      }
    }
    const int g = x.parent * c.nref + w.parent;
    grp[(size_t)(i - i0)] = g;
    ++count[g + 1];
  }
  for (int g = 0; g < ng; ++g) count[g + 1] += count[g];
  std::vector<int64_t> fill(count.begin(), count.end() - 1);
  for (int64_t i = i0; i < i1; ++i) {
    const int g = grp[(size_t)(i - i0)];
    if (g >= 0) order[(size_t)fill[g]++] = i;
  }
  for (int g = 0; g < ng; ++g) {
    const int64_t n = count[g + 1] - count[g];
    if (n == 0) continue;
    const PairView pv = make_view(c.slab, c.offs + (int64_t)g * kNoff, c.vals + (int64_t)g * kNval,
                                  c.ints + (int64_t)g * kNint);
    ORC_NS::batched_group(c, pv, pairs, order.data() + count[g], n, h_out, s_out);
  }
}

}  // namespace orc
