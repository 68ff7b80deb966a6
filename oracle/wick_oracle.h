// CPU oracle (test infrastructure only): types shared by the scalar FP64 evaluators
// (wick_eval.cpp) and the lane-batched restatement of the reference's fixed-rank SIMD path
// (wick_binned.cpp).  Slab orders follow src/nonorthogonalwicks/layout.rs of dy-cl/noci-rs.
#pragma once

#include <cstdint>

namespace orc {


constexpr int kMaxL = 8;
constexpr int kSpinOffs = 27;   // x[2] y[2] fh[2][2] v[2][2][2] hcol0 j[10]
constexpr int kNoff = 2 * kSpinOffs + 32;
constexpr int kSpinVals = 7;    // phase tsp f0h[2] v0[3]
constexpr int kNval = 2 * kSpinVals + 8;
constexpr int kNint = 5;        // m_a nocc_a m_b nocc_b nmo

struct SpinView {
  const double* x[2];
  const double* y[2];
  const double* fh_t[2][2];
  const double* v_t[2][2][2];
  const double* hcol0_t;
  const double* j[10];
  int m, nocc, nmo;
  double phase, tsp, f0h[2], v0[3];
};

struct DiffView {
  const double* vab_t[2][2][2];
  const double* vba_t[2][2][2];
  const double* ii[2][2][2][2];
  double vab0[2][2], vba0[2][2];
  int nmo;
};

struct PairView {
  SpinView aa, bb;
  DiffView ab;
};

// One determinant: parent, per-spin ranks and ascending hole/particle lists, occupation masks.
struct Det {
  int32_t parent;
  int32_t rank_a, rank_b;
  uint8_t holes_a[kMaxL], parts_a[kMaxL], holes_b[kMaxL], parts_b[kMaxL];
  uint64_t occ_a[2], occ_b[2];
  double pha, phb;
};

inline const double* at(const double* base, int64_t off) { return off < 0 ? nullptr : base + off; }

inline PairView make_view(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints) {
  PairView p{};
  SpinView* sv[2] = {&p.aa, &p.bb};
  for (int s = 0; s < 2; ++s) {
    const int64_t* o = offs + s * kSpinOffs;
    SpinView& v = *sv[s];
    int k = 0;
    for (int i = 0; i < 2; ++i) v.x[i] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i) v.y[i] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) v.fh_t[i][j] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        for (int l = 0; l < 2; ++l) v.v_t[i][j][l] = at(slab, o[k++]);
    v.hcol0_t = at(slab, o[k++]);
    for (int i = 0; i < 10; ++i) v.j[i] = at(slab, o[k++]);
    const double* vv = vals + s * kSpinVals;
    v.phase = vv[0];
    v.tsp = vv[1];
    v.f0h[0] = vv[2];
    v.f0h[1] = vv[3];
    v.v0[0] = vv[4];
    v.v0[1] = vv[5];
    v.v0[2] = vv[6];
    v.m = ints[2 * s];
    v.nocc = ints[2 * s + 1];
    v.nmo = ints[4];
  }
  const int64_t* o = offs + 2 * kSpinOffs;
  int k = 0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) p.ab.vab_t[a][b][c] = at(slab, o[k++]);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) p.ab.vba_t[a][b][c] = at(slab, o[k++]);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c)
        for (int d = 0; d < 2; ++d) p.ab.ii[a][b][c][d] = at(slab, o[k++]);
  const double* dv = vals + 2 * kSpinVals;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) p.ab.vab0[a][b] = dv[a * 2 + b];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) p.ab.vba0[a][b] = dv[4 + a * 2 + b];
  p.ab.nmo = ints[4];
  return p;
}

inline int popcount128(const uint64_t* a, const uint64_t* b) {
  return __builtin_popcountll(a[0] ^ b[0]) + __builtin_popcountll(a[1] ^ b[1]);
}

struct Ctx {
  const double* slab;
  const int64_t* offs;
  const double* vals;
  const int32_t* ints;
  int nref;
  const Det* basis;
  double enuc, tol;
  bool exact;
  // Same-parent orthogonal Slater-Condon caches (optional): per parent offsets of
  // ha, hb (n^2), eri_aa_asym, eri_bb_asym, eri_ab_coul (n^4) and the orthogonality flag.
  const int64_t* mo_offs;
  const int32_t* mo_orth;
  int nmo;
};

// Wick-path (H, S) of one pair with the same-parent dispatch of calculate_hs_pairs_wicks_batched
// (src/noci/hs.rs:72-130): the scalar generic evaluators (wick_eval.cpp).
void eval_one(const Ctx& c, int64_t a, int64_t b, double* h, double* s);
// Same-parent pair of an orthonormal parent (hs.rs:167-362), when the context has MO caches.
void hs_orthogonal(const Ctx& c, const Det& x, const Det& w, double* h_out, double* s_out);
// Wick path only (no same-parent shortcuts) of one pair.
void eval_wick_pair(const Ctx& c, const Det& x, const Det& w, double* h, double* s);

// calculate_hs_pairs_wicks_batched over requests [i0, i1) with the lane-batched fixed-rank
// kernels (wick_binned.cpp): 8 lanes (AVX-512 build) or 4 lanes (AVX2 + FMA build).
void hs_pairs_batched8(const Ctx& c, const int64_t* pairs, int64_t i0, int64_t i1, double* h_out, double* s_out);
void hs_pairs_batched4(const Ctx& c, const int64_t* pairs, int64_t i0, int64_t i1, double* h_out, double* s_out);

}  // namespace orc
