// CPU oracle (test infrastructure only): FP64 Wick (H, S) pair evaluator.
//
// This file restates, in scalar C++, the per-determinant-pair evaluators of dy-cl/noci-rs.
// It is the checker for the CUDA library and the timed CPU baseline of bench.py; the product
// library never links it.  Reference items restated (file:line inside dy-cl/noci-rs):
//   * prepare_same / construct_determinant_indices  src/nonorthogonalwicks/eval/prepare.rs:27-42,555-595
//   * build_d (X on/below the diagonal, Y above)     src/maths/wick.rs:59-75, :129-168
//   * det / adjugate_transpose / minor adjugates     src/maths/wick.rs:1122-1939, :2320-2448
//   * xw_hamiltonian_overlap_m0_gen_prepared          src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:20304-20532
//   * xw_hamiltonian_overlap_gen_prepared (m > 0)     src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:20550-20966
//   * jslot / j_replacement / ii_replacement          src/nonorthogonalwicks/eval/helpers.rs:165-260
//   * column_replacement_{correction,det}             src/nonorthogonalwicks/eval/helpers.rs:306-434
//   * get_det_adjt_diff / minor_adjt                  src/nonorthogonalwicks/eval/helpers.rs:564-670
//   * for_each_m_combination (Gosper's hack)          src/nonorthogonalwicks/eval/helpers.rs:682-712
//   * adjugate_transpose_generic                      src/nonorthogonalwicks/eval/helpers.rs:726-762
//   * xw_overlap (S only)                             src/nonorthogonalwicks/eval/overlap.rs:42-65,2572-2856
//   * calculate_hs_pairs_wicks_batched                src/noci/hs.rs:72-130
//   * calculate_hs_pair_orthogonal                    src/noci/hs.rs:167-362
//
// Storage orders follow the reference slab (src/nonorthogonalwicks/layout.rs): X, Y row-major
// [r,c]; F, V, hcol0, V^alpha, V^beta transposed [c,r]; J in [i,j,r,c]; II in [r,c,i,j].
// The fixed-rank SIMD kernels of the reference are specialisations of the generic evaluators
// restated here and give the same values up to rounding.
//
// Parity status: pinned against reference-produced numbers.  The reference's own energy
// fixtures (tests/fixtures/*/expected.json of noci-rs: reference-space NOCI, deterministic
// SD-space, NOCI-PT2 and selected-NOCI energies of H2, H4, LiH and F2) are reproduced from
// integrals and SCF states rebuilt by tests/golden/make_reference_fixtures.py
// (tests/test_reference_fixtures.py); the oracle is also cross-checked against an independent
// generalised Slater-Condon path and a brute-force Fock-space evaluation.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

#include "wick_oracle.h"

namespace orc {

// ---------------------------------------------------------------------------------------
// Tiny dense linear algebra (src/maths/wick.rs): closed forms for n <= 4, partial-pivot LU
// otherwise.  Cofactor matrices ("adjugate transpose") are formed from explicit minors.
// ---------------------------------------------------------------------------------------
double det_lu(const double* a, int n) {
  double lu[kMaxL * kMaxL];
  std::memcpy(lu, a, sizeof(double) * n * n);
  double sign = 1.0;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double pabs = std::fabs(lu[k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      double v = std::fabs(lu[r * n + k]);
      if (v > pabs) {
        piv = r;
        pabs = v;
      }
    }
    if (pabs == 0.0) return 0.0;
    if (piv != k) {
      for (int c = 0; c < n; ++c) std::swap(lu[k * n + c], lu[piv * n + c]);
      sign = -sign;
    }
    const double p = lu[k * n + k];
    for (int r = k + 1; r < n; ++r) {
      const double f = lu[r * n + k] / p;
      for (int c = k + 1; c < n; ++c) lu[r * n + c] -= f * lu[k * n + c];
    }
  }
  double d = sign;
  for (int i = 0; i < n; ++i) d *= lu[i * n + i];
  return d;
}

double det_n(const double* a, int n) {
  switch (n) {
    case 0:
      return 1.0;
    case 1:
      return a[0];
    case 2:
      return a[0] * a[3] - a[1] * a[2];
    case 3:
      return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
             a[2] * (a[3] * a[7] - a[4] * a[6]);
    case 4: {
      const double m00 = a[5] * (a[10] * a[15] - a[11] * a[14]) - a[6] * (a[9] * a[15] - a[11] * a[13]) +
                         a[7] * (a[9] * a[14] - a[10] * a[13]);
      const double m01 = a[4] * (a[10] * a[15] - a[11] * a[14]) - a[6] * (a[8] * a[15] - a[11] * a[12]) +
                         a[7] * (a[8] * a[14] - a[10] * a[12]);
      const double m02 = a[4] * (a[9] * a[15] - a[11] * a[13]) - a[5] * (a[8] * a[15] - a[11] * a[12]) +
                         a[7] * (a[8] * a[13] - a[9] * a[12]);
      const double m03 = a[4] * (a[9] * a[14] - a[10] * a[13]) - a[5] * (a[8] * a[14] - a[10] * a[12]) +
                         a[6] * (a[8] * a[13] - a[9] * a[12]);
      return a[0] * m00 - a[1] * m01 + a[2] * m02 - a[3] * m03;
    }
    default:
      return det_lu(a, n);
  }
}

void minor_of(double* out, const double* a, int n, int rr, int cc) {
  int k = 0;
  for (int r = 0; r < n; ++r) {
    if (r == rr) continue;
    for (int c = 0; c < n; ++c) {
      if (c == cc) continue;
      out[k++] = a[r * n + c];
    }
  }
}

// Cofactor matrix cof[r][c] = (-1)^{r+c} det(a without row r, column c); returns det(a).
double cofactors(double* cof, const double* a, int n) {
  if (n == 0) return 1.0;
  if (n == 1) {
    cof[0] = 1.0;
    return a[0];
  }
  double mn[kMaxL * kMaxL];
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      minor_of(mn, a, n, r, c);
      const double d = det_n(mn, n - 1);
      cof[r * n + c] = ((r + c) & 1) ? -d : d;
    }
  return det_n(a, n);
}

// adjugate_transpose_generic: fails when |det| <= tol (helpers.rs:726-762).
bool cofactors_tol(double* cof, const double* a, int n, double tol, double* det_out) {
  if (n == 0) {
    *det_out = 1.0;
    return 1.0 > tol;
  }
  double d;
  if (n <= 4) {
    d = cofactors(cof, a, n);
    if (!std::isfinite(d) || std::fabs(d) <= tol) return false;
  } else {
    d = det_n(a, n);
    if (!std::isfinite(d) || std::fabs(d) <= tol) return false;
    cofactors(cof, a, n);
  }
  *det_out = d;
  return true;
}

// minor_adjt: cofactors of the first minor D[row|col], kept only when |det minor| > tol.
bool minor_cof_tol(double* cofm, const double* full, int l, int row, int col, double tol) {
  double mn[kMaxL * kMaxL];
  minor_of(mn, full, l, row, col);
  double d;
  return cofactors_tol(cofm, mn, l - 1, tol, &d);
}

template <typename F>
void for_each_m_combination(int l, int m, F&& f) {
  if (m > l) return;
  if (m == 0) {
    f(0ull);
    return;
  }
  if (m == l) {
    f((1ull << l) - 1);
    return;
  }
  const uint64_t limit = 1ull << l;
  uint64_t x = (1ull << m) - 1;
  while (x < limit) {
    f(x);
    const uint64_t c = x & (~x + 1);
    const uint64_t r = x + c;
    x = (((r ^ x) >> 2) / c) | r;
  }
}

inline int bit(uint64_t b, int k) { return (int)((b >> k) & 1ull); }

void jslot(int mi, int mj, int mk, int ml, int* slot, bool* swap) {
  static const int tbl[16][2] = {
      {0, 0}, {1, 0}, {2, 0}, {3, 0}, {1, 1}, {4, 0}, {5, 0}, {6, 0},
      {2, 1}, {5, 1}, {7, 0}, {8, 0}, {3, 1}, {6, 1}, {8, 1}, {9, 0}};
  const int key = (mi << 3) | (mj << 2) | (mk << 1) | ml;
  *slot = tbl[key][0];
  *swap = tbl[key][1] != 0;
}

struct SpinPrep {
  int l;
  int rows[kMaxL], cols[kMaxL];
  double d0[kMaxL * kMaxL], d1[kMaxL * kMaxL];
};

void prepare_same(const SpinView& w, const uint8_t* xh, const uint8_t* xp, int xr, const uint8_t* wh,
                  const uint8_t* wp, int wr, SpinPrep& s) {
  const int nocc = w.nocc, nvirt = w.nmo - nocc, n = w.nmo;
  int i = 0;
  for (int k = 0; k < xr; ++k) {
    s.rows[i] = xp[k] - nocc;
    s.cols[i] = xh[k];
    ++i;
  }
  for (int k = 0; k < wr; ++k) {
    s.rows[i] = nvirt + wh[k];
    s.cols[i] = wp[k];
    ++i;
  }
  s.l = i;
  const int l = s.l;
  for (int r = 0; r < l; ++r)
    for (int c = 0; c < l; ++c) {
      const int64_t e = (int64_t)s.rows[r] * n + s.cols[c];
      s.d0[r * l + c] = (r >= c) ? w.x[0][e] : w.y[0][e];
      if (w.m > 0) s.d1[r * l + c] = (r >= c) ? w.x[1][e] : w.y[1][e];
    }
}

// ---------------------------------------------------------------------------------------
// m_alpha = m_beta = 0 (preparehamiltonianoverlap.rs:20304-20532)
// ---------------------------------------------------------------------------------------
double same_spin_m0(const SpinView& w, const SpinPrep& p, const double* cof, double det) {
  const int l = p.l, n = w.nmo;
  double same = (w.f0h[0] + 0.5 * w.v0[0]) * det;
  for (int z = 0; z < l; ++z) {
    const int64_t base = (int64_t)p.cols[z] * n;
    for (int e = 0; e < l; ++e) same -= cof[e * l + z] * w.hcol0_t[base + p.rows[e]];
  }
  if (l >= 2) {
    const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
    const double* jsl = w.j[0];
    double mn[kMaxL * kMaxL];
    for (int eta = 0; eta < l; ++eta)
      for (int xi = eta + 1; xi < l; ++xi)
        for (int z = 0; z < l; ++z)
          for (int y = z + 1; y < l; ++y) {
            int ii = 0;
            for (int r = 0; r < l; ++r) {
              if (r == eta || r == xi) continue;
              int mc = 0;
              for (int c = 0; c < l; ++c) {
                if (c == z || c == y) continue;
                mn[ii * (l - 2) + mc] = p.d0[r * l + c];
                ++mc;
              }
              ++ii;
            }
            const double second = det_n(mn, l - 2);
            const int64_t row_eta_n3 = p.rows[eta] * n3, row_xi_n = (int64_t)p.rows[xi] * n;
            const double direct = jsl[row_eta_n3 + p.cols[z] * n2 + row_xi_n + p.cols[y]];
            const double exchange = jsl[row_eta_n3 + p.cols[y] * n2 + row_xi_n + p.cols[z]];
            const double term = second * (direct - exchange);
            if (((eta + xi + z + y) & 1) == 0)
              same += term;
            else
              same -= term;
          }
  }
  return same;
}

void hs_m0(const PairView& w, const SpinPrep& pa, const SpinPrep& pb, double exc_phase, double enuc,
           double* h_out, double* s_out) {
  const int la = pa.l, lb = pb.l;
  double cofa[kMaxL * kMaxL], cofb[kMaxL * kMaxL];
  const double det_a = la == 0 ? 1.0 : cofactors(cofa, pa.d0, la);
  const double det_b = lb == 0 ? 1.0 : cofactors(cofb, pb.d0, lb);
  const double same_a = same_spin_m0(w.aa, pa, cofa, det_a);
  const double same_b = same_spin_m0(w.bb, pb, cofb, det_b);
  double h2ab = w.ab.vab0[0][0] * det_a * det_b;
  if (la > 0 && lb > 0) {
    const int n = w.ab.nmo;
    const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
    const double* iisl = w.ab.ii[0][0][0][0];
    for (int z = 0; z < la; ++z)
      for (int eta = 0; eta < la; ++eta) {
        const int64_t base_a = pa.rows[eta] * n3 + pa.cols[z] * n2;
        double inner = 0.0;
        for (int y = 0; y < lb; ++y)
          for (int xi = 0; xi < lb; ++xi)
            inner += cofb[xi * lb + y] * iisl[base_a + (int64_t)pb.rows[xi] * n + pb.cols[y]];
        h2ab += cofa[eta * la + z] * inner;
      }
  }
  const double sa_pref = w.aa.phase * w.aa.tsp;
  const double sb_pref = w.bb.phase * w.bb.tsp;
  const double s = exc_phase * sa_pref * sb_pref * det_a * det_b;
  *s_out = s;
  *h_out = enuc * s + exc_phase * sa_pref * sb_pref * (same_a * det_b + same_b * det_a + h2ab);
}

// ---------------------------------------------------------------------------------------
// m_alpha > 0 or m_beta > 0 (preparehamiltonianoverlap.rs:20550-20966)
// ---------------------------------------------------------------------------------------
void mix(double* out, const SpinPrep& p, uint64_t cbits) {
  const int l = p.l;
  for (int r = 0; r < l; ++r)
    for (int c = 0; c < l; ++c) out[r * l + c] = bit(cbits, c) ? p.d1[r * l + c] : p.d0[r * l + c];
}

// exact == false restates the reference; exact == true keeps every distribution and minor
// (cofactors exist for singular matrices) and counts the (0,1)/(1,0) scalar term once.
void same_spin_gen(const SpinView& w, const SpinPrep& p, double tol, bool exact, double* s_out,
                   double* h1_out, double* h2_out) {
  const int l = p.l, n = w.nmo;
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double s = 0.0, h1 = 0.0, h2 = 0.0;
  double dm[kMaxL * kMaxL], cof[kMaxL * kMaxL], cofm[kMaxL * kMaxL];
  for_each_m_combination(l + 2, w.m, [&](uint64_t bits) {
    const int m1 = bit(bits, 0), m2 = bit(bits, 1);
    const uint64_t cb = bits >> 2;
    mix(dm, p, cb);
    double det = 1.0;
    bool ok = true;
    if (l > 0) {
      if (exact)
        det = cofactors(cof, dm, l);
      else
        ok = cofactors_tol(cof, dm, l, tol, &det);
    }
    if (ok) {
      if (m1 == 0 && m2 == 0) s += det;
      if (m2 == 0) {
        double contrib = det * w.f0h[m1];
        for (int k = 0; k < l; ++k) {
          const double* fsl = w.fh_t[m1][bit(cb, k)];
          const int64_t base = (int64_t)p.cols[k] * n;
          double corr = 0.0;
          for (int r = 0; r < l; ++r) corr += (fsl[base + p.rows[r]] - dm[r * l + k]) * cof[r * l + k];
          contrib -= det + corr;
        }
        h1 += contrib;
      }
      double contrib = ((exact && m1 + m2 == 1) ? 0.5 : 1.0) * w.v0[m1 + m2] * det;
      for (int k = 0; k < l; ++k) {
        const double* vsl = w.v_t[m1][m2][bit(cb, k)];
        const int64_t base = (int64_t)p.cols[k] * n;
        double corr = 0.0;
        for (int r = 0; r < l; ++r) corr += (vsl[base + p.rows[r]] - dm[r * l + k]) * cof[r * l + k];
        contrib -= 2.0 * (det + corr);
      }
      if (l >= 2) {
        const int lm1 = l - 1;
        for (int i = 0; i < l; ++i)
          for (int j = 0; j < l; ++j) {
            const double ph = ((i + j) & 1) ? -1.0 : 1.0;
            const int ri = p.rows[i], cj = p.cols[j];
            const int mj = bit(cb, j);
            if (exact) {
              double mn[kMaxL * kMaxL];
              minor_of(mn, dm, l, i, j);
              cofactors(cofm, mn, l - 1);
            } else if (!minor_cof_tol(cofm, dm, l, i, j, tol)) {
              continue;
            }
            for (int k2 = 0; k2 < lm1; ++k2) {
              const int kf = k2 < j ? k2 : k2 + 1;
              const int mk = bit(cb, kf);
              int slot;
              bool swap;
              jslot(m1, m2, mk, mj, &slot, &swap);
              const double* jsl = w.j[slot];
              const int cc = p.cols[kf];
              double det_repl = 0.0;
              for (int r = 0; r < lm1; ++r) {
                const int rf = r < i ? r : r + 1;
                const int rr = p.rows[rf];
                const double nv = !swap ? jsl[ri * n3 + cj * n2 + (int64_t)rr * n + cc]
                                        : jsl[rr * n3 + cc * n2 + (int64_t)ri * n + cj];
                det_repl += nv * cofm[r * lm1 + k2];
              }
              contrib += ph * det_repl;
            }
          }
      }
      h2 += contrib;
    } else if (m1 == 0 && m2 == 0) {
      s += det_n(dm, l);
    }
  });
  *s_out = s;
  *h1_out = h1;
  *h2_out = h2;
}

void hs_gen(const PairView& w, const SpinPrep& pa, const SpinPrep& pb, double exc_phase, double enuc,
            double tol, bool exact, double* h_out, double* s_out) {
  const int la = pa.l, lb = pb.l;
  double sa, h1a, h2aa, sb, h1b, h2bb;
  same_spin_gen(w.aa, pa, tol, exact, &sa, &h1a, &h2aa);
  same_spin_gen(w.bb, pb, tol, exact, &sb, &h1b, &h2bb);
  double h2ab = 0.0;
  const int n = w.ab.nmo;
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double dma[kMaxL * kMaxL], dmb[kMaxL * kMaxL], cofa[kMaxL * kMaxL], cofb[kMaxL * kMaxL];
  for_each_m_combination(la + 1, w.aa.m, [&](uint64_t bits_a) {
    const uint64_t cba = bits_a >> 1;
    mix(dma, pa, cba);
    double deta;
    if (exact)
      deta = cofactors(cofa, dma, la);
    else if (!cofactors_tol(cofa, dma, la, tol, &deta))
      return;
    for_each_m_combination(lb + 1, w.bb.m, [&](uint64_t bits_b) {
      const uint64_t cbb = bits_b >> 1;
      mix(dmb, pb, cbb);
      double detb;
      if (exact)
        detb = cofactors(cofb, dmb, lb);
      else if (!cofactors_tol(cofb, dmb, lb, tol, &detb))
        return;
      const int ma0 = bit(bits_a, 0), mb0 = bit(bits_b, 0);
      double contrib = w.ab.vab0[ma0][mb0] * deta * detb;
      for (int k = 0; k < la; ++k) {
        const double* vsl = w.ab.vab_t[ma0][mb0][bit(cba, k)];
        const int64_t base = (int64_t)pa.cols[k] * n;
        double rep = 0.0;
        for (int r = 0; r < la; ++r) rep += vsl[base + pa.rows[r]] * cofa[r * la + k];
        contrib -= rep * detb;
      }
      for (int k = 0; k < lb; ++k) {
        const double* vsl = w.ab.vba_t[mb0][ma0][bit(cbb, k)];
        const int64_t base = (int64_t)pb.cols[k] * n;
        double rep = 0.0;
        for (int r = 0; r < lb; ++r) rep += vsl[base + pb.rows[r]] * cofb[r * lb + k];
        contrib -= rep * deta;
      }
      for (int i = 0; i < la; ++i) {
        const int ra = pa.rows[i];
        for (int j = 0; j < la; ++j) {
          const int ca = pa.cols[j];
          const double cij = cofa[i * la + j];
          const int ma1 = bit(cba, j);
          for (int k = 0; k < lb; ++k) {
            const double* iisl = w.ab.ii[ma0][ma1][mb0][bit(cbb, k)];
            double rep = 0.0;
            for (int r = 0; r < lb; ++r)
              rep += iisl[ra * n3 + ca * n2 + (int64_t)pb.rows[r] * n + pb.cols[k]] * cofb[r * lb + k];
            contrib += cij * rep;
          }
        }
      }
      h2ab += contrib;
    });
  });
  const double pref = exc_phase * (w.aa.phase * w.aa.tsp) * (w.bb.phase * w.bb.tsp);
  *s_out = pref * sa * sb;
  *h_out = pref * (h1a * sb + h1b * sa + 0.5 * h2aa * sb + 0.5 * h2bb * sa + h2ab);
  // The reference leaves E_nuc S out of this path; the exact convention adds it.
  if (exact) *h_out += enuc * *s_out;
}

// Overlap only (overlap.rs:42-65, 2572-2856), one spin.
double overlap_spin(const SpinView& w, const SpinPrep& p) {
  const int l = p.l;
  const double pref = w.phase * w.tsp;
  if (w.m > l) return 0.0;
  if (w.m == 0) return pref * det_n(p.d0, l);
  if (w.m == l) return pref * det_n(p.d1, l);
  double acc = 0.0, dm[kMaxL * kMaxL];
  for_each_m_combination(l, w.m, [&](uint64_t cb) {
    mix(dm, p, cb);
    acc += det_n(dm, l);
  });
  return pref * acc;
}

inline bool occ_bit(const uint64_t* o, int i) { return (o[i >> 6] >> (i & 63)) & 1ull; }

int list_from_mask(const uint64_t* m, int nmo, int* out) {
  int k = 0;
  for (int i = 0; i < nmo; ++i)
    if (occ_bit(m, i)) out[k++] = i;
  return k;
}

double ex_phase_list(const uint64_t* occ_in, const int* holes, int nh, const int* parts, int np) {
  uint64_t occ[2] = {occ_in[0], occ_in[1]};
  auto below = [&](int p) {
    int cnt = 0;
    for (int w = 0; w < 2; ++w) {
      const int lo = w * 64;
      if (p <= lo) break;
      const int nb = std::min(64, p - lo);
      const uint64_t mask = nb == 64 ? ~0ull : ((1ull << nb) - 1);
      cnt += __builtin_popcountll(occ[w] & mask);
    }
    return (cnt & 1) != 0;
  };
  bool odd = false;
  for (int k = nh - 1; k >= 0; --k) {
    odd ^= below(holes[k]);
    occ[holes[k] >> 6] &= ~(1ull << (holes[k] & 63));
  }
  for (int k = 0; k < np; ++k) {
    odd ^= below(parts[k]);
    if (k + 1 != np) occ[parts[k] >> 6] |= 1ull << (parts[k] & 63);
  }
  return odd ? -1.0 : 1.0;
}

// calculate_hs_pair_orthogonal (hs.rs:167-362).
void hs_orthogonal(const Ctx& c, const Det& x, const Det& w, double* h_out, double* s_out) {
  const int n = c.nmo;
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  const int64_t* mo = c.mo_offs + (int64_t)x.parent * 5;
  const double* ha = c.slab + mo[0];
  const double* hb = c.slab + mo[1];
  const double* eaa = c.slab + mo[2];
  const double* ebb = c.slab + mo[3];
  const double* eab = c.slab + mo[4];
  auto E4 = [&](const double* t, int a, int b, int cc, int d) { return t[a * n3 + b * n2 + (int64_t)cc * n + d]; };
  const int ra = popcount128(x.occ_a, w.occ_a) / 2, rb = popcount128(x.occ_b, w.occ_b) / 2;
  const bool same = (x.occ_a[0] == w.occ_a[0] && x.occ_a[1] == w.occ_a[1] && x.occ_b[0] == w.occ_b[0] &&
                     x.occ_b[1] == w.occ_b[1]);
  const double s = same ? (x.pha * w.pha) * (x.phb * w.phb) : 0.0;
  *s_out = s;
  if (ra > 2 || rb > 2 || ra + rb > 2) {
    *h_out = 0.0;
    return;
  }
  int ha_[2] = {0, 0}, pa_[2] = {0, 0}, hb_[2] = {0, 0}, pb_[2] = {0, 0};
  {
    uint64_t m[2];
    int k;
    for (int q = 0; q < 2; ++q) m[q] = w.occ_a[q] & ~x.occ_a[q];
    k = 0;
    for (int i = 0; i < n; ++i)
      if (occ_bit(m, i)) ha_[k++] = i;
    for (int q = 0; q < 2; ++q) m[q] = x.occ_a[q] & ~w.occ_a[q];
    k = 0;
    for (int i = 0; i < n; ++i)
      if (occ_bit(m, i)) pa_[k++] = i;
    for (int q = 0; q < 2; ++q) m[q] = w.occ_b[q] & ~x.occ_b[q];
    k = 0;
    for (int i = 0; i < n; ++i)
      if (occ_bit(m, i)) hb_[k++] = i;
    for (int q = 0; q < 2; ++q) m[q] = x.occ_b[q] & ~w.occ_b[q];
    k = 0;
    for (int i = 0; i < n; ++i)
      if (occ_bit(m, i)) pb_[k++] = i;
  }
  const double phase = ex_phase_list(w.occ_a, ha_, ra, pa_, ra) * ex_phase_list(w.occ_b, hb_, rb, pb_, rb);
  int oxa[128], oxb[128], com[128];
  const int nxa = list_from_mask(x.occ_a, n, oxa), nxb = list_from_mask(x.occ_b, n, oxb);
  if (ra == 0 && rb == 0) {
    double h = c.enuc;
    for (int i = 0; i < nxa; ++i) h += ha[oxa[i] * n + oxa[i]];
    for (int i = 0; i < nxb; ++i) h += hb[oxb[i] * n + oxb[i]];
    for (int i = 0; i < nxa; ++i)
      for (int j = 0; j < nxa; ++j) h += 0.5 * E4(eaa, oxa[i], oxa[i], oxa[j], oxa[j]);
    for (int i = 0; i < nxb; ++i)
      for (int j = 0; j < nxb; ++j) h += 0.5 * E4(ebb, oxb[i], oxb[i], oxb[j], oxb[j]);
    for (int i = 0; i < nxa; ++i)
      for (int j = 0; j < nxb; ++j) h += E4(eab, oxa[i], oxa[i], oxb[j], oxb[j]);
    *h_out = h;
    return;
  }
  if (ra == 1 && rb == 0) {
    const int i = ha_[0], a = pa_[0];
    double h = ha[a * n + i];
    uint64_t m[2] = {x.occ_a[0] & w.occ_a[0], x.occ_a[1] & w.occ_a[1]};
    int nc = list_from_mask(m, n, com);
    for (int q = 0; q < nc; ++q) h += E4(eaa, a, i, com[q], com[q]);
    uint64_t mb[2] = {x.occ_b[0] & w.occ_b[0], x.occ_b[1] & w.occ_b[1]};
    nc = list_from_mask(mb, n, com);
    for (int q = 0; q < nc; ++q) h += E4(eab, a, i, com[q], com[q]);
    *h_out = phase * h;
    return;
  }
  if (ra == 0 && rb == 1) {
    const int i = hb_[0], a = pb_[0];
    double h = hb[a * n + i];
    uint64_t m[2] = {x.occ_b[0] & w.occ_b[0], x.occ_b[1] & w.occ_b[1]};
    int nc = list_from_mask(m, n, com);
    for (int q = 0; q < nc; ++q) h += E4(ebb, a, i, com[q], com[q]);
    uint64_t ma[2] = {x.occ_a[0] & w.occ_a[0], x.occ_a[1] & w.occ_a[1]};
    nc = list_from_mask(ma, n, com);
    for (int q = 0; q < nc; ++q) h += E4(eab, com[q], com[q], i, a);
    *h_out = phase * h;
    return;
  }
  if (ra == 2 && rb == 0) {
    *h_out = phase * E4(eaa, pa_[0], ha_[0], ha_[1], pa_[1]);
    return;
  }
  if (ra == 0 && rb == 2) {
    *h_out = phase * E4(ebb, pb_[0], hb_[0], hb_[1], pb_[1]);
    return;
  }
  if (ra == 1 && rb == 1) {
    *h_out = phase * E4(eab, pa_[0], ha_[0], hb_[0], pb_[0]);
    return;
  }
  *h_out = 0.0;
}

void eval_one(const Ctx& c, int64_t a, int64_t b, double* h, double* s) {
  const Det& x = c.basis[a];
  const Det& w = c.basis[b];
  if (x.parent == w.parent) {
    if (popcount128(x.occ_a, w.occ_a) + popcount128(x.occ_b, w.occ_b) > 4) {
      *h = 0.0;
      *s = 0.0;
      return;
    }
    if (c.mo_offs != nullptr && c.mo_orth[x.parent]) {
      hs_orthogonal(c, x, w, h, s);
      return;
    }
  }
  eval_wick_pair(c, x, w, h, s);
}

void eval_wick_pair(const Ctx& c, const Det& x, const Det& w, double* h, double* s) {
  const int64_t pidx = (int64_t)x.parent * c.nref + w.parent;
  const PairView pv = make_view(c.slab, c.offs + pidx * kNoff, c.vals + pidx * kNval, c.ints + pidx * kNint);
  SpinPrep pa, pb;
  prepare_same(pv.aa, x.holes_a, x.parts_a, x.rank_a, w.holes_a, w.parts_a, w.rank_a, pa);
  prepare_same(pv.bb, x.holes_b, x.parts_b, x.rank_b, w.holes_b, w.parts_b, w.rank_b, pb);
  const double exc = (x.pha * w.pha) * (x.phb * w.phb);
  if (pv.aa.m == 0 && pv.bb.m == 0)
    hs_m0(pv, pa, pb, exc, c.enuc, h, s);
  else
    hs_gen(pv, pa, pb, exc, c.enuc, c.tol, c.exact, h, s);
}

// ---------------------------------------------------------------------------------------
// Fock one-body element and the SNOCI operator M = F - E0 S (onebody.rs:40-520, m.rs:160-197).
// Per pair and spin: F0f[2] (scalar) and ff_t[2][2] (transposed [c][r]) from
// construct_f_scalar (build.rs:564-617).
// ---------------------------------------------------------------------------------------
struct FockSpin {
  double f0f[2];
  const double* ff_t[2][2];
};

// xw_f for one spin: phase * tsp * sum over distributions of the one-body operator
// (m = 0: one distribution, no threshold; m > 0: get_det_adjt_same with pbits = 1).
double xw_f_spin(const SpinView& w, const FockSpin& f, const SpinPrep& p, double tol, bool exact) {
  const int l = p.l, n = w.nmo;
  double acc = 0.0;
  double dm[kMaxL * kMaxL], cof[kMaxL * kMaxL];
  if (w.m == 0) {
    double det = 1.0;
    if (l > 0) det = cofactors(cof, p.d0, l);
    double contrib = det * f.f0f[0];
    for (int b = 0; b < l; ++b) {
      const double* fsl = f.ff_t[0][0];
      const int64_t base = (int64_t)p.cols[b] * n;
      double corr = 0.0;
      for (int r = 0; r < l; ++r) corr += (fsl[base + p.rows[r]] - p.d0[r * l + b]) * cof[r * l + b];
      contrib -= det + corr;
    }
    acc = contrib;
  } else {
    for_each_m_combination(l + 1, w.m, [&](uint64_t bits) {
      const int mi = bit(bits, 0);
      const uint64_t cb = bits >> 1;
      mix(dm, p, cb);
      double det = 1.0;
      bool ok = true;
      if (l > 0) {
        if (exact)
          det = cofactors(cof, dm, l);
        else
          ok = cofactors_tol(cof, dm, l, tol, &det);
      }
      if (!ok) return;
      double contrib = det * f.f0f[mi];
      for (int b = 0; b < l; ++b) {
        const double* fsl = f.ff_t[mi][bit(cb, b)];
        const int64_t base = (int64_t)p.cols[b] * n;
        double corr = 0.0;
        for (int r = 0; r < l; ++r) corr += (fsl[base + p.rows[r]] - dm[r * l + b]) * cof[r * l + b];
        contrib -= det + corr;
      }
      acc += contrib;
    });
  }
  return w.phase * w.tsp * acc;
}

}  // namespace orc

using namespace orc;

extern "C" {

// Layout constants exported so the Python packer and this file agree.
int orc_layout(int which) {
  switch (which) {
    case 0:
      return kNoff;
    case 1:
      return kNval;
    case 2:
      return kNint;
    case 3:
      return (int)sizeof(Det);
    case 4:
      return kMaxL;
    default:
      return -1;
  }
}

// Evaluate (H, S) for npairs requests (a_i, b_i) into the determinant basis, as
// calculate_hs_pairs_wicks_batched does: same-parent pairs further apart than a double
// excitation give (0, 0); same-parent pairs of an orthonormal parent use Slater-Condon;
// all others are grouped by ordered reference pair and evaluated by the Wick path.
int orc_eval_pairs(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int nref,
                   const void* basis, const int64_t* pairs, int64_t npairs, double enuc, double tol,
                   const int64_t* mo_offs, const int32_t* mo_orth, int nmo, int nthreads, int flags,
                   double* h_out, double* s_out) {
  Ctx c{slab, offs, vals, ints, nref, reinterpret_cast<const Det*>(basis), enuc, tol, (flags & 1) != 0,
        mo_offs, mo_orth, nmo};
  // Group by ordered reference pair (hs.rs:86-109) for locality; results land at their
  // original positions.
  const int ng = nref * nref;
  std::vector<int64_t> count(ng + 1, 0), order(npairs);
  for (int64_t i = 0; i < npairs; ++i) {
    const int g = c.basis[pairs[2 * i]].parent * nref + c.basis[pairs[2 * i + 1]].parent;
    ++count[g + 1];
  }
  for (int g = 0; g < ng; ++g) count[g + 1] += count[g];
  std::vector<int64_t> fill(count.begin(), count.end() - 1);
  for (int64_t i = 0; i < npairs; ++i) {
    const int g = c.basis[pairs[2 * i]].parent * nref + c.basis[pairs[2 * i + 1]].parent;
    order[fill[g]++] = i;
  }
  // Dynamic chunks of the grouped order over plain std::threads.
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  std::atomic<int64_t> next{0};
  const int64_t chunk = 512;
  auto worker = [&]() {
    for (;;) {
      const int64_t t0 = next.fetch_add(chunk);
      if (t0 >= npairs) break;
      const int64_t t1 = std::min(npairs, t0 + chunk);
      for (int64_t t = t0; t < t1; ++t) {
        const int64_t i = order[t];
        eval_one(c, pairs[2 * i], pairs[2 * i + 1], &h_out[i], &s_out[i]);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int k = 1; k < nt; ++k) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  return 0;
}

// Wick-path (H, S) for one pair regardless of parents (no same-parent shortcuts).
int orc_eval_wick(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int nref,
                  const void* basis, int64_t a, int64_t b, double enuc, double tol, int flags, double* h,
                  double* s) {
  Ctx c{slab, offs, vals, ints, nref, reinterpret_cast<const Det*>(basis), enuc, tol, (flags & 1) != 0,
        nullptr, nullptr, 0};
  const Det& x = c.basis[a];
  const Det& w = c.basis[b];
  const int64_t pidx = (int64_t)x.parent * nref + w.parent;
  const PairView pv = make_view(slab, offs + pidx * kNoff, vals + pidx * kNval, ints + pidx * kNint);
  SpinPrep pa, pb;
  prepare_same(pv.aa, x.holes_a, x.parts_a, x.rank_a, w.holes_a, w.parts_a, w.rank_a, pa);
  prepare_same(pv.bb, x.holes_b, x.parts_b, x.rank_b, w.holes_b, w.parts_b, w.rank_b, pb);
  const double exc = (x.pha * w.pha) * (x.phb * w.phb);
  if (pv.aa.m == 0 && pv.bb.m == 0)
    hs_m0(pv, pa, pb, exc, enuc, h, s);
  else
    hs_gen(pv, pa, pb, exc, enuc, tol, c.exact, h, s);
  return 0;
}

// Wick-path overlap only: excitation phase times the per-spin xw_overlap values.
int orc_eval_overlap(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int nref,
                     const void* basis, int64_t a, int64_t b, double* s) {
  const Det* bs = reinterpret_cast<const Det*>(basis);
  const Det& x = bs[a];
  const Det& w = bs[b];
  const int64_t pidx = (int64_t)x.parent * nref + w.parent;
  const PairView pv = make_view(slab, offs + pidx * kNoff, vals + pidx * kNval, ints + pidx * kNint);
  SpinPrep pa, pb;
  prepare_same(pv.aa, x.holes_a, x.parts_a, x.rank_a, w.holes_a, w.parts_a, w.rank_a, pa);
  prepare_same(pv.bb, x.holes_b, x.parts_b, x.rank_b, w.holes_b, w.parts_b, w.rank_b, pb);
  const double exc = (x.pha * w.pha) * (x.phb * w.phb);
  *s = exc * overlap_spin(pv.aa, pa) * overlap_spin(pv.bb, pb);
  return 0;
}

// M = F - E0 S for npairs pairs via the Wick path (calculate_m_pair_wicks, m.rs:160-197).
// focks: per ordered pair, per spin, offsets of ff_t[2][2] into fslab and f0f[2] values.
int orc_eval_m_pairs(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int nref,
                     const void* basis, const int64_t* pairs, int64_t npairs, const double* fslab,
                     const int64_t* foffs, const double* fvals, double e0, double tol, int flags, double* m_out,
                     double* f_out, double* s_out) {
  const Det* bs = reinterpret_cast<const Det*>(basis);
  const bool exact = (flags & 1) != 0;
  for (int64_t i = 0; i < npairs; ++i) {
    const Det& x = bs[pairs[2 * i]];
    const Det& w = bs[pairs[2 * i + 1]];
    const int64_t pidx = (int64_t)x.parent * nref + w.parent;
    const PairView pv = make_view(slab, offs + pidx * kNoff, vals + pidx * kNval, ints + pidx * kNint);
    SpinPrep pa, pb;
    prepare_same(pv.aa, x.holes_a, x.parts_a, x.rank_a, w.holes_a, w.parts_a, w.rank_a, pa);
    prepare_same(pv.bb, x.holes_b, x.parts_b, x.rank_b, w.holes_b, w.parts_b, w.rank_b, pb);
    FockSpin fs[2];
    for (int sp = 0; sp < 2; ++sp) {
      const int64_t* fo = foffs + (pidx * 2 + sp) * 4;
      for (int k = 0; k < 4; ++k) fs[sp].ff_t[k >> 1][k & 1] = fslab + fo[k];
      fs[sp].f0f[0] = fvals[(pidx * 2 + sp) * 2];
      fs[sp].f0f[1] = fvals[(pidx * 2 + sp) * 2 + 1];
    }
    const double ph = (x.pha * w.pha) * (x.phb * w.phb);
    const double oa = overlap_spin(pv.aa, pa), ob = overlap_spin(pv.bb, pb);
    double f = 0.0;
    if (ob != 0.0) f += xw_f_spin(pv.aa, fs[0], pa, tol, exact) * ob;
    if (oa != 0.0) f += xw_f_spin(pv.bb, fs[1], pb, tol, exact) * oa;
    f *= ph;
    const double s = ph * oa * ob;
    f_out[i] = f;
    s_out[i] = s;
    m_out[i] = f - e0 * s;
  }
  return 0;
}

// The reference's own CPU path for the same requests: Rayon-style dynamic chunks of requests over
// nthreads threads, each chunk through calculate_hs_pairs_wicks_batched with the lane-batched
// fixed-rank kernels (wick_binned.cpp).  lanes = 8 (AVX-512), 4 (AVX2 + FMA) or 0 for the widest
// the host supports (is_x86_feature_detected in the reference); the lanes used are returned, or
// -1 when the host has neither (the requested width is not supported).
int orc_eval_pairs_binned(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int nref,
                          const void* basis, const int64_t* pairs, int64_t npairs, double enuc, double tol,
                          const int64_t* mo_offs, const int32_t* mo_orth, int nmo, int nthreads, int flags, int lanes,
                          double* h_out, double* s_out) {
  __builtin_cpu_init();
  const bool has8 = __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512dq");
  const bool has4 = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
  if (lanes == 0) lanes = has8 ? 8 : (has4 ? 4 : -1);
  if ((lanes == 8 && !has8) || (lanes == 4 && !has4) || (lanes != 8 && lanes != 4)) return -1;
  Ctx c{slab, offs, vals, ints, nref, reinterpret_cast<const Det*>(basis), enuc, tol, (flags & 1) != 0,
        mo_offs, mo_orth, nmo};
  int nt = nthreads > 0 ? nthreads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  std::atomic<int64_t> next{0};
  const int64_t chunk = 4096;
  auto worker = [&]() {
    for (;;) {
      const int64_t t0 = next.fetch_add(chunk);
      if (t0 >= npairs) break;
      const int64_t t1 = std::min(npairs, t0 + chunk);
      if (lanes == 8)
        hs_pairs_batched8(c, pairs, t0, t1, h_out, s_out);
      else
        hs_pairs_batched4(c, pairs, t0, t1, h_out, s_out);
    }
  };
  std::vector<std::thread> pool;
  for (int k = 1; k < nt; ++k) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  return lanes;
}

}  // extern "C"
