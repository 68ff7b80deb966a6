// Per-pair arithmetic of the Wick engine, written once as __host__ __device__ code.
//
// The CUDA kernels in eval.cu and build.cu call these functions on the device.  The same
// source is also compiled for the host by the CPU tests (tests/cpu_mirror), which check the
// index arithmetic and the algebra against the FP64 oracle without a GPU; the shipped
// library has no host evaluation path.
//
// Algorithms (restated from dy-cl/noci-rs, see the citations at each function):
//  * contraction-determinant rows/columns  src/nonorthogonalwicks/eval/prepare.rs:555-595
//  * m_alpha = m_beta = 0 fused (H, S)      src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:20304-20532
//  * m > 0 fused (H, S) over distributions  src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:20550-20966
//  * distribution enumeration               src/nonorthogonalwicks/eval/helpers.rs:682-712
//  * threshold semantics of adjugates       src/nonorthogonalwicks/eval/helpers.rs:636-670,726-762
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define NW_HD __host__ __device__ __forceinline__
#define NW_HD_CALL __host__ __device__ __noinline__  // a real call: its own register allocation
#else
#define NW_HD inline
#define NW_HD_CALL inline
#include <cmath>
using std::fabs;
using std::sqrt;
#endif

#ifndef __CUDACC__
struct double2 {
  double x, y;
};
#endif

namespace nw {

constexpr int kML = 8;  // maximum contraction rank per spin handled by the runtime paths

// ---------------------------------------------------------------------------------------
// Device tables.  For reference pairs without zero-overlap orbitals the evaluator reads the
// fast layout; pairs with m_alpha + m_beta > 0 keep the full intermediate set in the order
// of the noci-rs slab (src/nonorthogonalwicks/layout.rs): F, V, V^alpha, V^beta transposed
// [c][r], J as [i][j][r][c], II as [r][c][i][j].
// ---------------------------------------------------------------------------------------
struct FastSpin {
  const double2* recx;   // n*n records {X^(0)[r][c], hcol0[r][c]}
  const double2* recy;   // n*n records {Y^(0)[r][c], hcol0[r][c]}
  const double* jas;     // n^4, J^(0000)[r1][c1][r2][c2] - J^(0000)[r1][c2][r2][c1] (stored order)
  double pref;           // phase * product of nonzero singular values
  double g0;             // F0h^(0) + V0^(0) / 2
};

struct FastPair {
  FastSpin a, b;
  const double* ii0;     // n^4, II^(0000)[ra][ca][rb][cb]
  double vab0;           // V_ab,0^(0,0)
  double pad;
};

struct GenSpin {
  const double* x[2];
  const double* y[2];
  const double* fh_t[2][2];
  const double* v_t[2][2][2];
  const double* j[10];
  double pref;
  double f0h[2];
  double v0[3];
  int m;
  int pad;
};

struct GenPair {
  GenSpin a, b;
  const double* vab_t[2][2][2];
  const double* vba_t[2][2][2];
  const double* ii[2][2][2][2];
  double vab0[2][2];
  double vba0[2][2];
};

// Fock-operator tables of one ordered reference pair (update_wicks_fock, src/noci/wicks.rs:290-330;
// construct_f_scalar, src/nonorthogonalwicks/build.rs:564-617).  Pairs without zero-overlap
// orbitals read records {X^(0)|Y^(0), F^(00)} gathered like the Hamiltonian records; the
// others read F^(mi,mj) transposed ([c][r]) next to their reference-ordered X/Y.
struct FockSpinTab {
  const double2* recx;       // n*n {X^(0)[r][c], F^(00)[r][c]}
  const double2* recy;       // n*n {Y^(0)[r][c], F^(00)[r][c]}
  const double* ff_t[2][2];  // F^(mi,mj)[c][r]
  double f0f[2];             // F_0^(m) = tr(M^(m) F)
};

struct FockPair {
  FockSpinTab a, b;
};


// ---------------------------------------------------------------------------------------
// Small determinants.
// ---------------------------------------------------------------------------------------
NW_HD double det_lu_rt(const double* a, int n) {
  double lu[kML * kML];
  for (int i = 0; i < n * n; ++i) lu[i] = a[i];
  double sign = 1.0;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double pabs = fabs(lu[k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      const double v = fabs(lu[r * n + k]);
      if (v > pabs) {
        piv = r;
        pabs = v;
      }
    }
    if (pabs == 0.0) return 0.0;
    if (piv != k) {
      for (int c = 0; c < n; ++c) {
        const double t = lu[k * n + c];
        lu[k * n + c] = lu[piv * n + c];
        lu[piv * n + c] = t;
      }
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

NW_HD double det3(double a0, double a1, double a2, double a3, double a4, double a5, double a6, double a7,
                  double a8) {
  return a0 * (a4 * a8 - a5 * a7) - a1 * (a3 * a8 - a5 * a6) + a2 * (a3 * a7 - a4 * a6);
}

NW_HD double det_small(const double* a, int n) {
  switch (n) {
    case 0:
      return 1.0;
    case 1:
      return a[0];
    case 2:
      return a[0] * a[3] - a[1] * a[2];
    case 3:
      return det3(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
    case 4: {
      const double m00 = det3(a[5], a[6], a[7], a[9], a[10], a[11], a[13], a[14], a[15]);
      const double m01 = det3(a[4], a[6], a[7], a[8], a[10], a[11], a[12], a[14], a[15]);
      const double m02 = det3(a[4], a[5], a[7], a[8], a[9], a[11], a[12], a[13], a[15]);
      const double m03 = det3(a[4], a[5], a[6], a[8], a[9], a[10], a[12], a[13], a[14]);
      return a[0] * m00 - a[1] * m01 + a[2] * m02 - a[3] * m03;
    }
    default:
      return det_lu_rt(a, n);
  }
}

NW_HD void minor_rt(double* out, const double* a, int n, int rr, int cc) {
  int k = 0;
  for (int r = 0; r < n; ++r) {
    if (r == rr) continue;
    for (int c = 0; c < n; ++c) {
      if (c == cc) continue;
      out[k++] = a[r * n + c];
    }
  }
}

// Cofactor matrix cof[r][c] = (-1)^{r+c} det(a without r, c) for runtime n <= kML; returns det.
NW_HD double cofactors_rt(double* cof, const double* a, int n) {
  if (n == 0) return 1.0;
  if (n == 1) {
    cof[0] = 1.0;
    return a[0];
  }
  double mn[kML * kML];
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      minor_rt(mn, a, n, r, c);
      const double d = det_small(mn, n - 1);
      cof[r * n + c] = ((r + c) & 1) ? -d : d;
    }
  return det_small(a, n);
}

// adjugate_transpose_generic: false when |det| <= tol (helpers.rs:726-762).
NW_HD bool cofactors_tol_rt(double* cof, const double* a, int n, double tol, double* det_out) {
  if (n == 0) {
    *det_out = 1.0;
    return 1.0 > tol;
  }
  double d;
  if (n <= 4) {
    d = cofactors_rt(cof, a, n);
    if (!(fabs(d) <= 1.7976931348623157e308) || fabs(d) <= tol) return false;
  } else {
    d = det_small(a, n);
    if (!(fabs(d) <= 1.7976931348623157e308) || fabs(d) <= tol) return false;
    cofactors_rt(cof, a, n);
  }
  *det_out = d;
  return true;
}

// Compile-time-size cofactors (L <= 4) kept in registers by full unrolling.
template <int L>
NW_HD double cofactors_ct(double (&cof)[L * L > 0 ? L * L : 1], const double (&a)[L * L > 0 ? L * L : 1]) {
  if (L == 0) return 1.0;
  if (L == 1) {
    cof[0] = 1.0;
    return a[0];
  }
  if (L == 2) {
    cof[0] = a[3];
    cof[1] = -a[2];
    cof[2] = -a[1];
    cof[3] = a[0];
    return a[0] * a[3] - a[1] * a[2];
  }
#pragma unroll
  for (int r = 0; r < L; ++r) {
#pragma unroll
    for (int c = 0; c < L; ++c) {
      double mn[(L - 1) * (L - 1) > 0 ? (L - 1) * (L - 1) : 1];
      int k = 0;
#pragma unroll
      for (int i = 0; i < L; ++i) {
        if (i == r) continue;
#pragma unroll
        for (int j = 0; j < L; ++j) {
          if (j == c) continue;
          mn[k++] = a[i * L + j];
        }
      }
      const double d = det_small(mn, L - 1);
      cof[r * L + c] = ((r + c) & 1) ? -d : d;
    }
  }
  double d = 0.0;
#pragma unroll
  for (int c = 0; c < L; ++c) d += a[c] * cof[c];
  return d;
}

// det of D with rows {e, x} and columns {z, y} removed (the second minor of the J term).
template <int L>
NW_HD double second_minor_ct(const double (&a)[L * L > 0 ? L * L : 1], int e, int x, int z, int y) {
  double mn[(L - 2) * (L - 2) > 0 ? (L - 2) * (L - 2) : 1];
  int k = 0;
#pragma unroll
  for (int r = 0; r < L; ++r) {
    if (r == e || r == x) continue;
#pragma unroll
    for (int c = 0; c < L; ++c) {
      if (c == z || c == y) continue;
      mn[k++] = a[r * L + c];
    }
  }
  return det_small(mn, L - 2);
}

// ---------------------------------------------------------------------------------------
// Contraction-determinant labels (prepare.rs:555-595): bra pairs give rows a - nocc and
// columns i; ket pairs give rows nvirt + j and columns b.
// ---------------------------------------------------------------------------------------
NW_HD int det_labels(int rx, const uint8_t* ix, int rw, const uint8_t* iw, int nocc, int nmo, int* rows,
                     int* cols) {
  const int nvirt = nmo - nocc;
  int k = 0;
  for (int i = 0; i < rx; ++i) {
    rows[k] = (int)ix[4 + i] - nocc;
    cols[k] = ix[i];
    ++k;
  }
  for (int i = 0; i < rw; ++i) {
    rows[k] = nvirt + (int)iw[i];
    cols[k] = iw[4 + i];
    ++k;
  }
  return k;
}

// ---------------------------------------------------------------------------------------
// Same-spin part of the m = 0 fused evaluator for fixed L (<= 4).  rec_lo / rec_up hold
// {X0, hcol0} / {Y0, hcol0}; jas is the antisymmetrised J^(0000).
// ---------------------------------------------------------------------------------------
template <int L>
struct SpinM0 {
  double d[L * L > 0 ? L * L : 1];
  double cof[L * L > 0 ? L * L : 1];
  double det;
  double same;
};

template <int L>
NW_HD void spin_m0_ct(SpinM0<L>& s, const double2* rec_lo, const double2* rec_up, const double* jas, double g0,
                      int n, const int* rows, const int* cols) {
  double hc[L * L > 0 ? L * L : 1];
#pragma unroll
  for (int i = 0; i < L; ++i) {
#pragma unroll
    for (int j = 0; j < L; ++j) {
      const int64_t e = (int64_t)rows[i] * n + cols[j];
#ifdef __CUDA_ARCH__
      const double2 v = __ldg(i >= j ? rec_lo + e : rec_up + e);
#else
      const double2 v = i >= j ? rec_lo[e] : rec_up[e];
#endif
      s.d[i * L + j] = v.x;
      hc[i * L + j] = v.y;
    }
  }
  s.det = cofactors_ct<L>(s.cof, s.d);
  double same = g0 * s.det;
#pragma unroll
  for (int i = 0; i < L * L; ++i) same -= s.cof[i] * hc[i];
  if (L >= 2) {
    const int64_t n2 = (int64_t)n * n;
#pragma unroll
    for (int e = 0; e < L; ++e)
#pragma unroll
      for (int x = e + 1; x < L; ++x)
#pragma unroll
        for (int z = 0; z < L; ++z)
#pragma unroll
          for (int y = z + 1; y < L; ++y) {
            const double sec = second_minor_ct<L>(s.d, e, x, z, y);
            const int64_t idx = ((int64_t)rows[e] * n + cols[z]) * n2 + (int64_t)rows[x] * n + cols[y];
#ifdef __CUDA_ARCH__
            const double jv = __ldg(jas + idx);
#else
            const double jv = jas[idx];
#endif
            const double term = sec * jv;
            same += (((e + x + z + y) & 1) == 0) ? term : -term;
          }
  }
  s.same = same;
}

// Runtime-L version of the same-spin m = 0 part (L up to kML).
NW_HD void spin_m0_rt(int L, double* d, double* cof, double* det_out, double* same_out, const double2* rec_lo,
                      const double2* rec_up, const double* jas, double g0, int n, const int* rows, const int* cols) {
  double hc[kML * kML];
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < L; ++j) {
      const int64_t e = (int64_t)rows[i] * n + cols[j];
      const double2 v = i >= j ? rec_lo[e] : rec_up[e];
      d[i * L + j] = v.x;
      hc[i * L + j] = v.y;
    }
  const double det = cofactors_rt(cof, d, L);
  double same = g0 * det;
  for (int i = 0; i < L * L; ++i) same -= cof[i] * hc[i];
  if (L >= 2) {
    const int64_t n2 = (int64_t)n * n;
    double mn[kML * kML];
    for (int e = 0; e < L; ++e)
      for (int x = e + 1; x < L; ++x)
        for (int z = 0; z < L; ++z)
          for (int y = z + 1; y < L; ++y) {
            int k = 0;
            for (int r = 0; r < L; ++r) {
              if (r == e || r == x) continue;
              for (int c = 0; c < L; ++c) {
                if (c == z || c == y) continue;
                mn[k++] = d[r * L + c];
              }
            }
            const double sec = det_small(mn, L - 2);
            const int64_t idx = ((int64_t)rows[e] * n + cols[z]) * n2 + (int64_t)rows[x] * n + cols[y];
            const double term = sec * jas[idx];
            same += (((e + x + z + y) & 1) == 0) ? term : -term;
          }
  }
  *det_out = det;
  *same_out = same;
}

// ---------------------------------------------------------------------------------------
// m > 0 evaluator (preparehamiltonianoverlap.rs:20550-20966) over the reference-layout
// intermediates.  exact == false restates the reference; exact == true keeps every
// distribution and minor and counts the (0,1)/(1,0) scalar term once.
// ---------------------------------------------------------------------------------------
struct GenSpinIn {
  const double* x[2];
  const double* y[2];
  const double* fh_t[2][2];
  const double* v_t[2][2][2];
  const double* j[10];
  double f0h[2];
  double v0[3];
  int m;
};

NW_HD int bitk(uint64_t b, int k) { return (int)((b >> k) & 1ull); }

NW_HD uint64_t next_combination(uint64_t x) {
  const uint64_t c = x & (~x + 1ull);
  const uint64_t r = x + c;
  return (((r ^ x) >> 2) / c) | r;
}

// Number of distributions and the first one of for_each_m_combination(l, m) (helpers.rs:682-712).
NW_HD bool first_combination(int l, int m, uint64_t* x) {
  if (m > l) return false;
  *x = (m == 0) ? 0ull : ((1ull << m) - 1ull);
  return true;
}
NW_HD bool advance_combination(int l, int m, uint64_t* x) {
  if (m == 0 || m == l) return false;
  const uint64_t nx = next_combination(*x);
  if (nx >= (1ull << l)) return false;
  *x = nx;
  return true;
}

NW_HD void jslot_hd(int mi, int mj, int mk, int ml, int* slot, bool* swap) {
  const int key = (mi << 3) | (mj << 2) | (mk << 1) | ml;
  // (slot, swap) for the 16 binary assignments, SAME_SPIN_J_BRANCHES order (helpers.rs:165-191)
  int s = 0;
  bool w = false;
  switch (key) {
    case 0: s = 0; break;
    case 1: s = 1; break;
    case 4: s = 1; w = true; break;
    case 2: s = 2; break;
    case 8: s = 2; w = true; break;
    case 3: s = 3; break;
    case 12: s = 3; w = true; break;
    case 5: s = 4; break;
    case 6: s = 5; break;
    case 9: s = 5; w = true; break;
    case 7: s = 6; break;
    case 13: s = 6; w = true; break;
    case 10: s = 7; break;
    case 11: s = 8; break;
    case 14: s = 8; w = true; break;
    default: s = 9; break;
  }
  *slot = s;
  *swap = w;
}

NW_HD void mix_rt(double* out, const double* d0, const double* d1, int l, uint64_t cbits) {
  for (int r = 0; r < l; ++r)
    for (int c = 0; c < l; ++c) out[r * l + c] = bitk(cbits, c) ? d1[r * l + c] : d0[r * l + c];
}

NW_HD void build_d_rt(double* d, const double* xm, const double* ym, int n, int l, const int* rows, const int* cols) {
  for (int r = 0; r < l; ++r)
    for (int c = 0; c < l; ++c) {
      const int64_t e = (int64_t)rows[r] * n + cols[c];
      d[r * l + c] = (r >= c) ? xm[e] : ym[e];
    }
}

NW_HD void same_spin_gen_hd(const GenSpinIn& w, int n, int l, const int* rows, const int* cols, const double* d0,
                            const double* d1, double tol, bool exact, double* s_out, double* h1_out,
                            double* h2_out) {
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double s = 0.0, h1 = 0.0, h2 = 0.0;
  double dm[kML * kML], cof[kML * kML], cofm[kML * kML], mn[kML * kML];
  uint64_t bits;
  bool more = first_combination(l + 2, w.m, &bits);
  while (more) {
    const int m1 = bitk(bits, 0), m2 = bitk(bits, 1);
    const uint64_t cb = bits >> 2;
    mix_rt(dm, d0, d1, l, cb);
    double det = 1.0;
    bool ok = true;
    if (l > 0) {
      if (exact)
        det = cofactors_rt(cof, dm, l);
      else
        ok = cofactors_tol_rt(cof, dm, l, tol, &det);
    }
    if (ok) {
      if (m1 == 0 && m2 == 0) s += det;
      if (m2 == 0) {
        double contrib = det * w.f0h[m1];
        for (int k = 0; k < l; ++k) {
          const double* fsl = w.fh_t[m1][bitk(cb, k)];
          const int64_t base = (int64_t)cols[k] * n;
          double corr = 0.0;
          for (int r = 0; r < l; ++r) corr += (fsl[base + rows[r]] - dm[r * l + k]) * cof[r * l + k];
          contrib -= det + corr;
        }
        h1 += contrib;
      }
      double contrib = ((exact && m1 + m2 == 1) ? 0.5 : 1.0) * w.v0[m1 + m2] * det;
      for (int k = 0; k < l; ++k) {
        const double* vsl = w.v_t[m1][m2][bitk(cb, k)];
        const int64_t base = (int64_t)cols[k] * n;
        double corr = 0.0;
        for (int r = 0; r < l; ++r) corr += (vsl[base + rows[r]] - dm[r * l + k]) * cof[r * l + k];
        contrib -= 2.0 * (det + corr);
      }
      if (l >= 2) {
        const int lm1 = l - 1;
        for (int i = 0; i < l; ++i)
          for (int j = 0; j < l; ++j) {
            const double ph = ((i + j) & 1) ? -1.0 : 1.0;
            const int ri = rows[i], cj = cols[j];
            const int mj = bitk(cb, j);
            minor_rt(mn, dm, l, i, j);
            if (exact) {
              cofactors_rt(cofm, mn, lm1);
            } else {
              double dmin;
              if (!cofactors_tol_rt(cofm, mn, lm1, tol, &dmin)) continue;
            }
            for (int k2 = 0; k2 < lm1; ++k2) {
              const int kf = k2 < j ? k2 : k2 + 1;
              const int mk = bitk(cb, kf);
              int slot;
              bool swap;
              jslot_hd(m1, m2, mk, mj, &slot, &swap);
              const double* jsl = w.j[slot];
              const int cc = cols[kf];
              double det_repl = 0.0;
              for (int r = 0; r < lm1; ++r) {
                const int rf = r < i ? r : r + 1;
                const int rr = rows[rf];
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
      s += det_small(dm, l);
    }
    more = advance_combination(l + 2, w.m, &bits);
  }
  *s_out = s;
  *h1_out = h1;
  *h2_out = h2;
}

struct GenDiffIn {
  const double* vab_t[2][2][2];
  const double* vba_t[2][2][2];
  const double* ii[2][2][2][2];
  double vab0[2][2];
};

NW_HD double diff_spin_gen_hd(const GenDiffIn& w, int n, int ma, int mb, int la, const int* rows_a,
                              const int* cols_a, const double* da0, const double* da1, int lb, const int* rows_b,
                              const int* cols_b, const double* db0, const double* db1, double tol, bool exact) {
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double dma[kML * kML], dmb[kML * kML], cofa[kML * kML], cofb[kML * kML];
  double h2ab = 0.0;
  uint64_t bits_a;
  bool more_a = first_combination(la + 1, ma, &bits_a);
  while (more_a) {
    const uint64_t cba = bits_a >> 1;
    mix_rt(dma, da0, da1, la, cba);
    double deta = 1.0;
    bool oka = true;
    if (exact)
      deta = cofactors_rt(cofa, dma, la);
    else
      oka = cofactors_tol_rt(cofa, dma, la, tol, &deta);
    if (oka) {
      uint64_t bits_b;
      bool more_b = first_combination(lb + 1, mb, &bits_b);
      while (more_b) {
        const uint64_t cbb = bits_b >> 1;
        mix_rt(dmb, db0, db1, lb, cbb);
        double detb = 1.0;
        bool okb = true;
        if (exact)
          detb = cofactors_rt(cofb, dmb, lb);
        else
          okb = cofactors_tol_rt(cofb, dmb, lb, tol, &detb);
        if (okb) {
          const int ma0 = bitk(bits_a, 0), mb0 = bitk(bits_b, 0);
          double contrib = w.vab0[ma0][mb0] * deta * detb;
          for (int k = 0; k < la; ++k) {
            const double* vsl = w.vab_t[ma0][mb0][bitk(cba, k)];
            const int64_t base = (int64_t)cols_a[k] * n;
            double rep = 0.0;
            for (int r = 0; r < la; ++r) rep += vsl[base + rows_a[r]] * cofa[r * la + k];
            contrib -= rep * detb;
          }
          for (int k = 0; k < lb; ++k) {
            const double* vsl = w.vba_t[mb0][ma0][bitk(cbb, k)];
            const int64_t base = (int64_t)cols_b[k] * n;
            double rep = 0.0;
            for (int r = 0; r < lb; ++r) rep += vsl[base + rows_b[r]] * cofb[r * lb + k];
            contrib -= rep * deta;
          }
          for (int i = 0; i < la; ++i) {
            const int ra = rows_a[i];
            for (int j = 0; j < la; ++j) {
              const int ca = cols_a[j];
              const double cij = cofa[i * la + j];
              const int ma1 = bitk(cba, j);
              for (int k = 0; k < lb; ++k) {
                const double* iisl = w.ii[ma0][ma1][mb0][bitk(cbb, k)];
                double rep = 0.0;
                for (int r = 0; r < lb; ++r)
                  rep += iisl[ra * n3 + ca * n2 + (int64_t)rows_b[r] * n + cols_b[k]] * cofb[r * lb + k];
                contrib += cij * rep;
              }
            }
          }
          h2ab += contrib;
        }
        more_b = advance_combination(lb + 1, mb, &bits_b);
      }
    }
    more_a = advance_combination(la + 1, ma, &bits_a);
  }
  return h2ab;
}

// Overlap-only sum over distributions for one spin (overlap.rs:42-65, 2572-2856).
NW_HD double overlap_spin_hd(int m, int l, const double* d0, const double* d1) {
  if (m > l) return 0.0;
  if (m == 0) return det_small(d0, l);
  if (m == l) return det_small(d1, l);
  double acc = 0.0, dm[kML * kML];
  uint64_t bits;
  bool more = first_combination(l, m, &bits);
  while (more) {
    mix_rt(dm, d0, d1, l, bits);
    acc += det_small(dm, l);
    more = advance_combination(l, m, &bits);
  }
  return acc;
}

// ---------------------------------------------------------------------------------------
// FP64 one-sided (Hestenes) Jacobi SVD of a small o x o matrix, for the Loewdin pairing of
// the occupied overlap.  On return a holds U*diag(s), u the left vectors (columns), v the
// right vectors, s the singular values in descending order.  Columns of U whose singular
// value is <= tol are completed to an orthonormal basis by Gram-Schmidt against the unit
// vectors.  The sweep count is bounded.
// ---------------------------------------------------------------------------------------
NW_HD int jacobi_svd(int o, double* a, double* u, double* v, double* s, double tol) {
  for (int i = 0; i < o; ++i)
    for (int j = 0; j < o; ++j) v[i * o + j] = (i == j) ? 1.0 : 0.0;
  int sweeps = 0;
  for (; sweeps < 80; ++sweeps) {
    bool rotated = false;
    for (int p = 0; p < o - 1; ++p)
      for (int q = p + 1; q < o; ++q) {
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = 0; i < o; ++i) {
          const double ap = a[i * o + p], aq = a[i * o + q];
          al += ap * ap;
          be += aq * aq;
          ga += ap * aq;
        }
        if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
        rotated = true;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t);
        const double sn = c * t;
        for (int i = 0; i < o; ++i) {
          const double ap = a[i * o + p], aq = a[i * o + q];
          a[i * o + p] = c * ap - sn * aq;
          a[i * o + q] = sn * ap + c * aq;
          const double vp = v[i * o + p], vq = v[i * o + q];
          v[i * o + p] = c * vp - sn * vq;
          v[i * o + q] = sn * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
  for (int k = 0; k < o; ++k) {
    double nrm = 0.0;
    for (int i = 0; i < o; ++i) nrm += a[i * o + k] * a[i * o + k];
    s[k] = sqrt(nrm);
  }
  // sort descending (selection sort), permuting columns of a and v
  for (int k = 0; k < o; ++k) {
    int best = k;
    for (int j = k + 1; j < o; ++j)
      if (s[j] > s[best]) best = j;
    if (best != k) {
      const double ts = s[k];
      s[k] = s[best];
      s[best] = ts;
      for (int i = 0; i < o; ++i) {
        double t = a[i * o + k];
        a[i * o + k] = a[i * o + best];
        a[i * o + best] = t;
        t = v[i * o + k];
        v[i * o + k] = v[i * o + best];
        v[i * o + best] = t;
      }
    }
  }
  // left vectors
  for (int k = 0; k < o; ++k) {
    if (s[k] > tol) {
      for (int i = 0; i < o; ++i) u[i * o + k] = a[i * o + k] / s[k];
    } else {
      for (int i = 0; i < o; ++i) u[i * o + k] = 0.0;
    }
  }
  // complete the null columns of U
  int unit = 0;
  for (int k = 0; k < o; ++k) {
    if (s[k] > tol) continue;
    for (; unit < o; ++unit) {
      double w[64];
      for (int i = 0; i < o; ++i) w[i] = (i == unit) ? 1.0 : 0.0;
      for (int pass = 0; pass < 2; ++pass)
        for (int j = 0; j < o; ++j) {
          if (j == k) continue;
          if (s[j] <= tol && j > k) continue;
          double dot = 0.0;
          for (int i = 0; i < o; ++i) dot += u[i * o + j] * w[i];
          for (int i = 0; i < o; ++i) w[i] -= dot * u[i * o + j];
        }
      double nrm = 0.0;
      for (int i = 0; i < o; ++i) nrm += w[i] * w[i];
      nrm = sqrt(nrm);
      if (nrm > 1e-6) {
        for (int i = 0; i < o; ++i) u[i * o + k] = w[i] / nrm;
        ++unit;
        break;
      }
    }
  }
  return sweeps;
}

// Canonical gauge of the null columns (any zero singular value): with M0 the null columns of
// U (and likewise V), M0^T = Q R by modified Gram-Schmidt over its columns (residual norms
// <= 1e-10 skipped) with R's diagonal positive, and M0 -> M0 Q.  The reference evaluator's
// zero-overlap handling depends on this otherwise free choice; fixing it makes the result
// independent of the SVD routine.
NW_HD void canonical_null_columns(int o, double* mat, const double* s, double tol) {
  int zeros[64];
  int m = 0;
  for (int k = 0; k < o; ++k)
    if (s[k] <= tol) zeros[m++] = k;
  if (m < 1) return;
  // B = M0^T (m x o); modified Gram-Schmidt on its columns gives Q (m x m) with R_jj > 0.
  double q[64 * 8];  // m <= 8 supported for the canonical gauge
  if (m > 8) return;
  int found = 0;
  for (int col = 0; col < o && found < m; ++col) {
    double w[8];
    for (int j = 0; j < m; ++j) w[j] = mat[col * o + zeros[j]];
    for (int pass = 0; pass < 2; ++pass)
      for (int f = 0; f < found; ++f) {
        double dot = 0.0;
        for (int j = 0; j < m; ++j) dot += q[j * 8 + f] * w[j];
        for (int j = 0; j < m; ++j) w[j] -= dot * q[j * 8 + f];
      }
    double nrm = 0.0;
    for (int j = 0; j < m; ++j) nrm += w[j] * w[j];
    nrm = sqrt(nrm);
    if (nrm <= 1e-10) continue;
    for (int j = 0; j < m; ++j) q[j * 8 + found] = w[j] / nrm;
    ++found;
  }
  if (found < m) return;
  // M0 <- M0 Q
  for (int i = 0; i < o; ++i) {
    double row[8];
    for (int f = 0; f < m; ++f) {
      double acc = 0.0;
      for (int j = 0; j < m; ++j) acc += mat[i * o + zeros[j]] * q[j * 8 + f];
      row[f] = acc;
    }
    for (int f = 0; f < m; ++f) mat[i * o + zeros[f]] = row[f];
  }
}

}  // namespace nw

namespace nw {

// In-place partial-pivot LU determinant for a runtime n (a is destroyed).
NW_HD double det_lu_inplace(double* lu, int n) {
  double sign = 1.0;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double pabs = fabs(lu[k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      const double v = fabs(lu[r * n + k]);
      if (v > pabs) {
        piv = r;
        pabs = v;
      }
    }
    if (pabs == 0.0) return 0.0;
    if (piv != k) {
      for (int c = 0; c < n; ++c) {
        const double t = lu[k * n + c];
        lu[k * n + c] = lu[piv * n + c];
        lu[piv * n + c] = t;
      }
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

// Contraction labels for a compile-time L from packed index words (byte k = hole k,
// byte 4 + k = particle k), kept in registers by full unrolling.
template <int L>
NW_HD void det_labels_ct(int rx, uint64_t ix, uint64_t iw, int nocc, int nmo, int* rows, int* cols) {
  const int nvirt = nmo - nocc;
#pragma unroll
  for (int k = 0; k < L; ++k) {
    const bool fx = k < rx;
    const int kx = k & 3;
    const int kw = (k - rx) & 3;
    const int xh = (int)((ix >> (8 * kx)) & 0xFF);
    const int xp = (int)((ix >> (8 * (4 + kx))) & 0xFF);
    const int wh = (int)((iw >> (8 * kw)) & 0xFF);
    const int wp = (int)((iw >> (8 * (4 + kw))) & 0xFF);
    rows[k] = fx ? xp - nocc : nvirt + wh;
    cols[k] = fx ? xh : wp;
  }
}

}  // namespace nw

namespace nw {

// Read-only loads: the texture path on the device, plain loads on the host.
NW_HD double ldg_d(const double* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
NW_HD double2 ldg_d2(const double2* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}

// ---------------------------------------------------------------------------------------
// nw_det unpacking from its four 64-bit words (bytes: 0-3 parent, 4 rank_a, 5-12 idx_a,
// 13 rank_b, 14-21 idx_b, 24-31 phase).
// ---------------------------------------------------------------------------------------
struct DetRec {
  uint32_t parent;
  int ra, rb;
  uint64_t ia, ib;  // per-spin index bytes (holes 0..3, particles 4..7)
  double phase;
};

NW_HD DetRec unpack_det(uint64_t w0, uint64_t w1, uint64_t w2, uint64_t w3) {
  DetRec d;
  d.parent = (uint32_t)(w0 & 0xFFFFFFFFull);
  d.ra = (int)((w0 >> 32) & 0xFF);
  d.ia = (w0 >> 40) | (w1 << 24);
  d.rb = (int)((w1 >> 40) & 0xFF);
  d.ib = (w1 >> 48) | (w2 << 16);
  union {
    uint64_t u;
    double f;
  } cv;
  cv.u = w3;
  d.phase = cv.f;
  return d;
}

NW_HD int ibyte(uint64_t w, int k) { return (int)((w >> (8 * k)) & 0xFF); }

// |A xor B| for the first ra / rb hole (off 0) or particle (off 4) entries.
NW_HD int sym_diff(uint64_t wa, int ra, uint64_t wb, int rb, int off) {
  int common = 0;
  for (int i = 0; i < ra; ++i)
    for (int j = 0; j < rb; ++j) common += (ibyte(wa, off + i) == ibyte(wb, off + j));
  return ra + rb - 2 * common;
}

// Same parent and more than a double excitation apart: (H, S) = (0, 0) (src/noci/hs.rs:96-101).
NW_HD bool far_same_parent(const DetRec& x, const DetRec& w) {
  if (x.parent != w.parent) return false;
  const int d = sym_diff(x.ia, x.ra, w.ia, w.ra, 0) + sym_diff(x.ia, x.ra, w.ia, w.ra, 4) +
                sym_diff(x.ib, x.rb, w.ib, w.rb, 0) + sym_diff(x.ib, x.rb, w.ib, w.rb, 4);
  return d > 4;
}

NW_HD int rank_class(int la, int lb) { return (la <= 4 && lb <= 4) ? la * 5 + lb : 25; }

// ---------------------------------------------------------------------------------------
// Sort keys of the evaluation pipeline.  A pair of a fast reference pair (no zero-overlap
// orbitals) gets  cls * nbucket + ((ket_parent * ndet + bra) >> shift):  class-major, so each
// evaluator kernel walks one contiguous range per class; inside a class the pairs of one ket
// reference come together, ordered by bra (bras are numbered parent by parent), so the pairs
// of one bra determinant lie together (the lanes of a warp share the bra's rows of the
// intermediates) and the grid's window over the class stays inside one ordered reference pair
// (x, w) at a time instead of spreading over the nref pairs (x, *) of the bra's parent -- a
// working set nref times smaller in L2.  Pairs of reference pairs with zero-overlap orbitals follow,
// keyed by (sort position - nfast, L_alpha, L_beta) with the full ranks 0..kML: their
// distribution sums cost about L^7 per spin, so a warp whose lanes mixed ranks would run every
// lane at the pace of its largest L.  Keys are < kRankClasses * nbucket + kGenClasses *
// (nref^2 - nfast).
// ---------------------------------------------------------------------------------------
constexpr int kRankClasses = 26;
constexpr int kGenClasses = (kML + 1) * (kML + 1);

NW_HD uint32_t pair_sort_key(int la, int lb, uint32_t bra, int ket_parent, int ord, int nfast, uint64_t ndet,
                             uint32_t nbucket, int shift) {
  if (ord < nfast)
    return (uint32_t)rank_class(la, lb) * nbucket +
           (uint32_t)((((uint64_t)ket_parent * ndet) + bra) >> shift);
  return (uint32_t)kRankClasses * nbucket + (uint32_t)((ord - nfast) * kGenClasses + la * (kML + 1) + lb);
}

// Smallest shift for which the fast-pair keys, kRankClasses * nbucket, fit in cap (cap >= 26).
NW_HD int sort_key_shift(uint64_t ndet, int nref, uint64_t cap, uint32_t* nbucket) {
  const uint64_t span = ndet * (uint64_t)nref;
  int s = 0;
  while (s < 63 && (uint64_t)kRankClasses * (((span - 1) >> s) + 1) > cap) ++s;
  *nbucket = (uint32_t)(((span - 1) >> s) + 1);
  return s;
}

// 16-bit class descriptor of a determinant record: parent (8 bits), rank_a, rank_b (4 bits each).
NW_HD uint32_t det_desc(uint32_t parent, int ra, int rb) { return parent | ((uint32_t)ra << 8) | ((uint32_t)rb << 12); }

NW_HD void labels_rt(const DetRec& x, const DetRec& w, int spin, int nocc, int n, int* rows, int* cols) {
  uint8_t bx[8], bw[8];
  const uint64_t ix = spin ? x.ib : x.ia, iw = spin ? w.ib : w.ia;
  for (int k = 0; k < 8; ++k) {
    bx[k] = (uint8_t)ibyte(ix, k);
    bw[k] = (uint8_t)ibyte(iw, k);
  }
  det_labels(spin ? x.rb : x.ra, bx, spin ? w.rb : w.ra, bw, nocc, n, rows, cols);
}

// ---------------------------------------------------------------------------------------
// m = 0 fused (H, S) for one pair (preparehamiltonianoverlap.rs:20304-20532) on the fast
// layout, compile-time (L_alpha, L_beta).
// ---------------------------------------------------------------------------------------
template <int LA, int LB>
NW_HD void eval_m0_ct(const FastPair& fp, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                      double* H, double* S) {
  int ra[LA > 0 ? LA : 1], ca[LA > 0 ? LA : 1], rb[LB > 0 ? LB : 1], cb[LB > 0 ? LB : 1];
  det_labels_ct<LA>(x.ra, x.ia, w.ia, oa, n, ra, ca);
  det_labels_ct<LB>(x.rb, x.ib, w.ib, ob, n, rb, cb);
  SpinM0<LA> sa;
  SpinM0<LB> sb;
  spin_m0_ct<LA>(sa, fp.a.recx, fp.a.recy, fp.a.jas, fp.a.g0, n, ra, ca);
  spin_m0_ct<LB>(sb, fp.b.recx, fp.b.recy, fp.b.jas, fp.b.g0, n, rb, cb);
  double h2ab = fp.vab0 * sa.det * sb.det;
  if (LA > 0 && LB > 0) {
    const int64_t n2 = (int64_t)n * n;
#pragma unroll
    for (int e = 0; e < LA; ++e)
#pragma unroll
      for (int z = 0; z < LA; ++z) {
        const double* blk = fp.ii0 + ((int64_t)ra[e] * n + ca[z]) * n2;
        double inner = 0.0;
#pragma unroll
        for (int xx = 0; xx < LB; ++xx)
#pragma unroll
          for (int y = 0; y < LB; ++y) inner += sb.cof[xx * LB + y] * ldg_d(blk + (int64_t)rb[xx] * n + cb[y]);
        h2ab += sa.cof[e * LA + z] * inner;
      }
  }
  const double pref = x.phase * w.phase * fp.a.pref * fp.b.pref;
  const double s = pref * sa.det * sb.det;
  *S = s;
  *H = enuc * s + pref * (sa.same * sb.det + sb.same * sa.det + h2ab);
}

// Runtime-rank version for L_alpha or L_beta above 4 (up to 8).
NW_HD void eval_m0_rt(const FastPair& fp, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                      double* H, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  int ra[kML], ca[kML], rb[kML], cb[kML];
  labels_rt(x, w, 0, oa, n, ra, ca);
  labels_rt(x, w, 1, ob, n, rb, cb);
  double da[kML * kML], cofa[kML * kML], db[kML * kML], cofb[kML * kML];
  double deta, detb, samea, sameb;
  spin_m0_rt(la, da, cofa, &deta, &samea, fp.a.recx, fp.a.recy, fp.a.jas, fp.a.g0, n, ra, ca);
  spin_m0_rt(lb, db, cofb, &detb, &sameb, fp.b.recx, fp.b.recy, fp.b.jas, fp.b.g0, n, rb, cb);
  double h2ab = fp.vab0 * deta * detb;
  if (la > 0 && lb > 0) {
    const int64_t n2 = (int64_t)n * n;
    for (int e = 0; e < la; ++e)
      for (int z = 0; z < la; ++z) {
        const double* blk = fp.ii0 + ((int64_t)ra[e] * n + ca[z]) * n2;
        double inner = 0.0;
        for (int xx = 0; xx < lb; ++xx)
          for (int y = 0; y < lb; ++y) inner += cofb[xx * lb + y] * blk[(int64_t)rb[xx] * n + cb[y]];
        h2ab += cofa[e * la + z] * inner;
      }
  }
  const double pref = x.phase * w.phase * fp.a.pref * fp.b.pref;
  const double s = pref * deta * detb;
  *S = s;
  *H = enuc * s + pref * (samea * detb + sameb * deta + h2ab);
}

#define NW_M0_CASE(A, B)                                   \
  case (A) * 5 + (B):                                      \
    eval_m0_ct<A, B>(fp, x, w, n, oa, ob, enuc, H, S);     \
    return;

NW_HD void eval_m0_pair(const FastPair& fp, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                        double* H, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  if (la <= 4 && lb <= 4) {
    switch (la * 5 + lb) {
      NW_M0_CASE(0, 0) NW_M0_CASE(0, 1) NW_M0_CASE(0, 2) NW_M0_CASE(0, 3) NW_M0_CASE(0, 4)
      NW_M0_CASE(1, 0) NW_M0_CASE(1, 1) NW_M0_CASE(1, 2) NW_M0_CASE(1, 3) NW_M0_CASE(1, 4)
      NW_M0_CASE(2, 0) NW_M0_CASE(2, 1) NW_M0_CASE(2, 2) NW_M0_CASE(2, 3) NW_M0_CASE(2, 4)
      NW_M0_CASE(3, 0) NW_M0_CASE(3, 1) NW_M0_CASE(3, 2) NW_M0_CASE(3, 3) NW_M0_CASE(3, 4)
      NW_M0_CASE(4, 0) NW_M0_CASE(4, 1) NW_M0_CASE(4, 2) NW_M0_CASE(4, 3) NW_M0_CASE(4, 4)
      default:
        break;
    }
  }
  eval_m0_rt(fp, x, w, n, oa, ob, enuc, H, S);
}
#undef NW_M0_CASE

// ---------------------------------------------------------------------------------------
// m > 0 fused (H, S) for one pair on the reference-ordered intermediates.
// ---------------------------------------------------------------------------------------
// Per-spin and mixed-spin tables of one reference pair, as the distribution sums read them.
NW_HD void gen_inputs(const GenPair& g, GenSpinIn* wa, GenSpinIn* wb, GenDiffIn* wd) {
  const GenSpin* src[2] = {&g.a, &g.b};
  GenSpinIn* dst[2] = {wa, wb};
  for (int s = 0; s < 2; ++s) {
    for (int i = 0; i < 2; ++i) {
      dst[s]->x[i] = src[s]->x[i];
      dst[s]->y[i] = src[s]->y[i];
      dst[s]->f0h[i] = src[s]->f0h[i];
      for (int j = 0; j < 2; ++j) {
        dst[s]->fh_t[i][j] = src[s]->fh_t[i][j];
        for (int k = 0; k < 2; ++k) dst[s]->v_t[i][j][k] = src[s]->v_t[i][j][k];
      }
    }
    for (int k = 0; k < 3; ++k) dst[s]->v0[k] = src[s]->v0[k];
    for (int k = 0; k < 10; ++k) dst[s]->j[k] = src[s]->j[k];
    dst[s]->m = src[s]->m;
  }
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      wd->vab0[a][b] = g.vab0[a][b];
      for (int c = 0; c < 2; ++c) {
        wd->vab_t[a][b][c] = g.vab_t[a][b][c];
        wd->vba_t[a][b][c] = g.vba_t[a][b][c];
        for (int d = 0; d < 2; ++d) wd->ii[a][b][c][d] = g.ii[a][b][c][d];
      }
    }
}

NW_HD void eval_gen_pair(const GenPair& g, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                         double tol, bool exact, double* H, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  int ra[kML], ca[kML], rb[kML], cb[kML];
  labels_rt(x, w, 0, oa, n, ra, ca);
  labels_rt(x, w, 1, ob, n, rb, cb);
  double da0[kML * kML], da1[kML * kML], db0[kML * kML], db1[kML * kML];
  build_d_rt(da0, g.a.x[0], g.a.y[0], n, la, ra, ca);
  build_d_rt(da1, g.a.x[1], g.a.y[1], n, la, ra, ca);
  build_d_rt(db0, g.b.x[0], g.b.y[0], n, lb, rb, cb);
  build_d_rt(db1, g.b.x[1], g.b.y[1], n, lb, rb, cb);
  GenSpinIn wa, wb;
  GenDiffIn wd;
  gen_inputs(g, &wa, &wb, &wd);
  double sa, h1a, h2aa, sb, h1b, h2bb;
  same_spin_gen_hd(wa, n, la, ra, ca, da0, da1, tol, exact, &sa, &h1a, &h2aa);
  same_spin_gen_hd(wb, n, lb, rb, cb, db0, db1, tol, exact, &sb, &h1b, &h2bb);
  const double h2ab = diff_spin_gen_hd(wd, n, g.a.m, g.b.m, la, ra, ca, da0, da1, lb, rb, cb, db0, db1, tol, exact);
  const double pref = x.phase * w.phase * g.a.pref * g.b.pref;
  const double s = pref * sa * sb;
  double h = pref * (h1a * sb + h1b * sa + 0.5 * h2aa * sb + 0.5 * h2bb * sa + h2ab);
  if (exact) h += enuc * s;
  *S = s;
  *H = h;
}

// ---------------------------------------------------------------------------------------
// Compile-time-L (<= 4 per spin) twins of same_spin_gen_hd, diff_spin_gen_hd and
// eval_gen_pair: the same terms in the same order, with the distribution matrices, their
// cofactors and the minors of the J term in registers by full unrolling instead of in
// per-thread local memory.
// ---------------------------------------------------------------------------------------
template <int L>
struct Sq {
  static constexpr int v = L * L > 0 ? L * L : 1;
};

template <int L>
NW_HD void mix_ct(double (&out)[Sq<L>::v], const double (&d0)[Sq<L>::v], const double (&d1)[Sq<L>::v],
                  uint64_t cbits) {
#pragma unroll
  for (int r = 0; r < L; ++r)
#pragma unroll
    for (int c = 0; c < L; ++c) out[r * L + c] = bitk(cbits, c) ? d1[r * L + c] : d0[r * L + c];
}

template <int L>
NW_HD void build_d_ct(double (&d)[Sq<L>::v], const double* xm, const double* ym, int n, const int* rows,
                      const int* cols) {
#pragma unroll
  for (int r = 0; r < L; ++r)
#pragma unroll
    for (int c = 0; c < L; ++c) {
      const int64_t e = (int64_t)rows[r] * n + cols[c];
      d[r * L + c] = ldg_d((r >= c ? xm : ym) + e);
    }
}

// cofactors_tol_rt for compile-time L.
template <int L>
NW_HD bool cofactors_tol_ct(double (&cof)[Sq<L>::v], const double (&a)[Sq<L>::v], double tol, double* det_out) {
  const double d = cofactors_ct<L>(cof, a);
  if (!(fabs(d) <= 1.7976931348623157e308) || fabs(d) <= tol) return false;
  *det_out = d;
  return true;
}

template <int L>
NW_HD void minor_ct(double (&out)[Sq<L - 1>::v], const double (&a)[Sq<L>::v], int rr, int cc) {
  int k = 0;
#pragma unroll
  for (int r = 0; r < L; ++r) {
    if (r == rr) continue;
#pragma unroll
    for (int c = 0; c < L; ++c) {
      if (c == cc) continue;
      out[k++] = a[r * L + c];
    }
  }
}

template <int L, typename SpinTab>
NW_HD void same_spin_gen_ct(const SpinTab& w, int n, const int* rows, const int* cols, const double (&d0)[Sq<L>::v],
                            const double (&d1)[Sq<L>::v], double tol, bool exact, double* s_out, double* h1_out,
                            double* h2_out) {
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double s = 0.0, h1 = 0.0, h2 = 0.0;
  uint64_t bits;
  bool more = first_combination(L + 2, w.m, &bits);
  while (more) {
    const int m1 = bitk(bits, 0), m2 = bitk(bits, 1);
    const uint64_t cb = bits >> 2;
    double dm[Sq<L>::v], cof[Sq<L>::v];
    mix_ct<L>(dm, d0, d1, cb);
    double det = 1.0;
    bool ok = true;
    if (L > 0) {
      if (exact)
        det = cofactors_ct<L>(cof, dm);
      else
        ok = cofactors_tol_ct<L>(cof, dm, tol, &det);
    }
    if (ok) {
      if (m1 == 0 && m2 == 0) s += det;
      if (m2 == 0) {
        double contrib = det * w.f0h[m1];
#pragma unroll
        for (int k = 0; k < L; ++k) {
          const double* fsl = w.fh_t[m1][bitk(cb, k)];
          const int64_t base = (int64_t)cols[k] * n;
          double corr = 0.0;
#pragma unroll
          for (int r = 0; r < L; ++r) corr += (ldg_d(fsl + base + rows[r]) - dm[r * L + k]) * cof[r * L + k];
          contrib -= det + corr;
        }
        h1 += contrib;
      }
      double contrib = ((exact && m1 + m2 == 1) ? 0.5 : 1.0) * w.v0[m1 + m2] * det;
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const double* vsl = w.v_t[m1][m2][bitk(cb, k)];
        const int64_t base = (int64_t)cols[k] * n;
        double corr = 0.0;
#pragma unroll
        for (int r = 0; r < L; ++r) corr += (ldg_d(vsl + base + rows[r]) - dm[r * L + k]) * cof[r * L + k];
        contrib -= 2.0 * (det + corr);
      }
      if constexpr (L >= 2) {
        constexpr int LM1 = L - 1;
#pragma unroll
        for (int i = 0; i < L; ++i)
#pragma unroll
          for (int j = 0; j < L; ++j) {
            const double ph = ((i + j) & 1) ? -1.0 : 1.0;
            const int ri = rows[i], cj = cols[j];
            const int mj = bitk(cb, j);
            double mn[Sq<LM1>::v], cofm[Sq<LM1>::v];
            minor_ct<L>(mn, dm, i, j);
            if (exact) {
              cofactors_ct<LM1>(cofm, mn);
            } else {
              double dmin;
              if (!cofactors_tol_ct<LM1>(cofm, mn, tol, &dmin)) continue;
            }
#pragma unroll
            for (int k2 = 0; k2 < LM1; ++k2) {
              const int kf = k2 < j ? k2 : k2 + 1;
              const int mk = bitk(cb, kf);
              int slot;
              bool swap;
              jslot_hd(m1, m2, mk, mj, &slot, &swap);
              const double* jsl = w.j[slot];
              const int cc = cols[kf];
              double det_repl = 0.0;
#pragma unroll
              for (int r = 0; r < LM1; ++r) {
                const int rf = r < i ? r : r + 1;
                const int rr = rows[rf];
                const double nv = ldg_d(!swap ? jsl + (ri * n3 + cj * n2 + (int64_t)rr * n + cc)
                                              : jsl + (rr * n3 + cc * n2 + (int64_t)ri * n + cj));
                det_repl += nv * cofm[r * LM1 + k2];
              }
              contrib += ph * det_repl;
            }
          }
      }
      h2 += contrib;
    } else if (m1 == 0 && m2 == 0) {
      s += det_small(dm, L);
    }
    more = advance_combination(L + 2, w.m, &bits);
  }
  *s_out = s;
  *h1_out = h1;
  *h2_out = h2;
}

template <int LA, int LB, typename DiffTab>
NW_HD double diff_spin_gen_ct(const DiffTab& w, int n, int ma, int mb, const int* rows_a, const int* cols_a,
                              const double (&da0)[Sq<LA>::v], const double (&da1)[Sq<LA>::v], const int* rows_b,
                              const int* cols_b, const double (&db0)[Sq<LB>::v], const double (&db1)[Sq<LB>::v],
                              double tol, bool exact) {
  const int64_t n2 = (int64_t)n * n, n3 = n2 * n;
  double h2ab = 0.0;
  uint64_t bits_a;
  bool more_a = first_combination(LA + 1, ma, &bits_a);
  while (more_a) {
    const uint64_t cba = bits_a >> 1;
    double dma[Sq<LA>::v], cofa[Sq<LA>::v];
    mix_ct<LA>(dma, da0, da1, cba);
    double deta = 1.0;
    bool oka = true;
    if (exact)
      deta = cofactors_ct<LA>(cofa, dma);
    else
      oka = cofactors_tol_ct<LA>(cofa, dma, tol, &deta);
    if (oka) {
      uint64_t bits_b;
      bool more_b = first_combination(LB + 1, mb, &bits_b);
      while (more_b) {
        const uint64_t cbb = bits_b >> 1;
        double dmb[Sq<LB>::v], cofb[Sq<LB>::v];
        mix_ct<LB>(dmb, db0, db1, cbb);
        double detb = 1.0;
        bool okb = true;
        if (exact)
          detb = cofactors_ct<LB>(cofb, dmb);
        else
          okb = cofactors_tol_ct<LB>(cofb, dmb, tol, &detb);
        if (okb) {
          const int ma0 = bitk(bits_a, 0), mb0 = bitk(bits_b, 0);
          double contrib = w.vab0[ma0][mb0] * deta * detb;
#pragma unroll
          for (int k = 0; k < LA; ++k) {
            const double* vsl = w.vab_t[ma0][mb0][bitk(cba, k)];
            const int64_t base = (int64_t)cols_a[k] * n;
            double rep = 0.0;
#pragma unroll
            for (int r = 0; r < LA; ++r) rep += ldg_d(vsl + base + rows_a[r]) * cofa[r * LA + k];
            contrib -= rep * detb;
          }
#pragma unroll
          for (int k = 0; k < LB; ++k) {
            const double* vsl = w.vba_t[mb0][ma0][bitk(cbb, k)];
            const int64_t base = (int64_t)cols_b[k] * n;
            double rep = 0.0;
#pragma unroll
            for (int r = 0; r < LB; ++r) rep += ldg_d(vsl + base + rows_b[r]) * cofb[r * LB + k];
            contrib -= rep * deta;
          }
#pragma unroll
          for (int i = 0; i < LA; ++i) {
            const int ra = rows_a[i];
#pragma unroll
            for (int j = 0; j < LA; ++j) {
              const int ca = cols_a[j];
              const double cij = cofa[i * LA + j];
              const int ma1 = bitk(cba, j);
#pragma unroll
              for (int k = 0; k < LB; ++k) {
                const double* iisl = w.ii[ma0][ma1][mb0][bitk(cbb, k)];
                double rep = 0.0;
#pragma unroll
                for (int r = 0; r < LB; ++r)
                  rep += ldg_d(iisl + (ra * n3 + ca * n2 + (int64_t)rows_b[r] * n + cols_b[k])) * cofb[r * LB + k];
                contrib += cij * rep;
              }
            }
          }
          h2ab += contrib;
        }
        more_b = advance_combination(LB + 1, mb, &bits_b);
      }
    }
    more_a = advance_combination(LA + 1, ma, &bits_a);
  }
  return h2ab;
}

template <int LA, int LB>
NW_HD void eval_gen_ct(const GenPair& g, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                       double tol, bool exact, double* H, double* S) {
  int ra[LA > 0 ? LA : 1], ca[LA > 0 ? LA : 1], rb[LB > 0 ? LB : 1], cb[LB > 0 ? LB : 1];
  det_labels_ct<LA>(x.ra, x.ia, w.ia, oa, n, ra, ca);
  det_labels_ct<LB>(x.rb, x.ib, w.ib, ob, n, rb, cb);
  double da0[Sq<LA>::v], da1[Sq<LA>::v], db0[Sq<LB>::v], db1[Sq<LB>::v];
  build_d_ct<LA>(da0, g.a.x[0], g.a.y[0], n, ra, ca);
  build_d_ct<LA>(da1, g.a.x[1], g.a.y[1], n, ra, ca);
  build_d_ct<LB>(db0, g.b.x[0], g.b.y[0], n, rb, cb);
  build_d_ct<LB>(db1, g.b.x[1], g.b.y[1], n, rb, cb);
  // the tables are read where they lie (the reference pair's GenPair record, global memory on
  // the device): copying their ~100 pointers into per-thread structs indexed at run time put
  // them in local memory
  double sa, h1a, h2aa, sb, h1b, h2bb;
  same_spin_gen_ct<LA>(g.a, n, ra, ca, da0, da1, tol, exact, &sa, &h1a, &h2aa);
  same_spin_gen_ct<LB>(g.b, n, rb, cb, db0, db1, tol, exact, &sb, &h1b, &h2bb);
  const double h2ab = diff_spin_gen_ct<LA, LB>(g, n, g.a.m, g.b.m, ra, ca, da0, da1, rb, cb, db0, db1, tol, exact);
  const double pref = x.phase * w.phase * g.a.pref * g.b.pref;
  const double s = pref * sa * sb;
  double h = pref * (h1a * sb + h1b * sa + 0.5 * h2aa * sb + 0.5 * h2bb * sa + h2ab);
  if (exact) h += enuc * s;
  *S = s;
  *H = h;
}

template <int LA, int LB>
NW_HD_CALL void eval_gen_case(const GenPair& g, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                              double tol, bool exact, double* H, double* S) {
  eval_gen_ct<LA, LB>(g, x, w, n, oa, ob, enuc, tol, exact, H, S);
}

#define NW_GEN_CASE(A, B)                                                 \
  case (A) * 5 + (B):                                                     \
    eval_gen_case<A, B>(g, x, w, n, oa, ob, enuc, tol, exact, H, S);      \
    return;

// m > 0 (H, S) of one pair: the register twin (one call per (L_alpha, L_beta) case) for
// contraction ranks up to 4 per spin, the runtime-size path above that.
NW_HD void eval_gen_any(const GenPair& g, const DetRec& x, const DetRec& w, int n, int oa, int ob, double enuc,
                        double tol, bool exact, double* H, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  if (la <= 4 && lb <= 4) {
    switch (la * 5 + lb) {
      NW_GEN_CASE(0, 0) NW_GEN_CASE(0, 1) NW_GEN_CASE(0, 2) NW_GEN_CASE(0, 3) NW_GEN_CASE(0, 4)
      NW_GEN_CASE(1, 0) NW_GEN_CASE(1, 1) NW_GEN_CASE(1, 2) NW_GEN_CASE(1, 3) NW_GEN_CASE(1, 4)
      NW_GEN_CASE(2, 0) NW_GEN_CASE(2, 1) NW_GEN_CASE(2, 2) NW_GEN_CASE(2, 3) NW_GEN_CASE(2, 4)
      NW_GEN_CASE(3, 0) NW_GEN_CASE(3, 1) NW_GEN_CASE(3, 2) NW_GEN_CASE(3, 3) NW_GEN_CASE(3, 4)
      NW_GEN_CASE(4, 0) NW_GEN_CASE(4, 1) NW_GEN_CASE(4, 2) NW_GEN_CASE(4, 3) NW_GEN_CASE(4, 4)
      default: break;
    }
  }
  eval_gen_pair(g, x, w, n, oa, ob, enuc, tol, exact, H, S);
}
#undef NW_GEN_CASE

// Overlap only for one pair (fast or generic layout).
NW_HD double eval_s_pair(const FastPair* fp, const GenPair* g, const DetRec& x, const DetRec& w, int n, int oa,
                         int ob) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  int ra[kML], ca[kML], rb[kML], cb[kML];
  labels_rt(x, w, 0, oa, n, ra, ca);
  labels_rt(x, w, 1, ob, n, rb, cb);
  double d0[kML * kML], d1[kML * kML];
  double sa, sb, pref;
  if (fp) {
    for (int r = 0; r < la; ++r)
      for (int c = 0; c < la; ++c) {
        const int64_t e = (int64_t)ra[r] * n + ca[c];
        d0[r * la + c] = (r >= c) ? fp->a.recx[e].x : fp->a.recy[e].x;
      }
    sa = det_small(d0, la);
    for (int r = 0; r < lb; ++r)
      for (int c = 0; c < lb; ++c) {
        const int64_t e = (int64_t)rb[r] * n + cb[c];
        d0[r * lb + c] = (r >= c) ? fp->b.recx[e].x : fp->b.recy[e].x;
      }
    sb = det_small(d0, lb);
    pref = fp->a.pref * fp->b.pref;
  } else {
    build_d_rt(d0, g->a.x[0], g->a.y[0], n, la, ra, ca);
    build_d_rt(d1, g->a.x[1], g->a.y[1], n, la, ra, ca);
    sa = overlap_spin_hd(g->a.m, la, d0, d1);
    build_d_rt(d0, g->b.x[0], g->b.y[0], n, lb, rb, cb);
    build_d_rt(d1, g->b.x[1], g->b.y[1], n, lb, rb, cb);
    sb = overlap_spin_hd(g->b.m, lb, d0, d1);
    pref = g->a.pref * g->b.pref;
  }
  return x.phase * w.phase * pref * sa * sb;
}

// ---------------------------------------------------------------------------------------
// Fock one-body element with the overlap (xw_f_overlap_prepared,
// src/nonorthogonalwicks/eval/prepareonebodyoverlap.rs:57-100; xw_f, eval/onebody.rs:40;
// combined per spin as calculate_m_pair_wicks, src/noci/m.rs:160-197).
// Per spin:  F_sigma = F_0 det D - sum_{r,c} cof[r][c] F[row_r][col_c]  (m = 0), and the
// distribution sum over (m_1; m_col...) for m > 0.  With the spin overlaps S_sigma:
//   F = ph (F_alpha S_beta + F_beta S_alpha),  S = ph S_alpha S_beta,
// where a term is skipped when the other spin's overlap is exactly zero (m.rs:187-193).
// ---------------------------------------------------------------------------------------
template <int L>
NW_HD void spin_f_ct(const double2* rec_lo, const double2* rec_up, double f0, int n, const int* rows,
                     const int* cols, double* det_out, double* f_out) {
  if (L == 0) {
    *det_out = 1.0;
    *f_out = f0;
    return;
  }
  double d[L > 0 ? L * L : 1], fc[L > 0 ? L * L : 1], cof[L > 0 ? L * L : 1];
#pragma unroll
  for (int i = 0; i < L; ++i)
#pragma unroll
    for (int j = 0; j < L; ++j) {
      const int64_t e = (int64_t)rows[i] * n + cols[j];
#ifdef __CUDA_ARCH__
      const double2 v = __ldg(i >= j ? rec_lo + e : rec_up + e);
#else
      const double2 v = i >= j ? rec_lo[e] : rec_up[e];
#endif
      d[i * L + j] = v.x;
      fc[i * L + j] = v.y;
    }
  const double det = cofactors_ct<L>(cof, d);
  double f = f0 * det;
#pragma unroll
  for (int i = 0; i < L * L; ++i) f -= cof[i] * fc[i];
  *det_out = det;
  *f_out = f;
}

NW_HD void spin_f_rt(int L, const double2* rec_lo, const double2* rec_up, double f0, int n, const int* rows,
                     const int* cols, double* det_out, double* f_out) {
  if (L == 0) {
    *det_out = 1.0;
    *f_out = f0;
    return;
  }
  double d[kML * kML], fc[kML * kML], cof[kML * kML];
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < L; ++j) {
      const int64_t e = (int64_t)rows[i] * n + cols[j];
      const double2 v = i >= j ? rec_lo[e] : rec_up[e];
      d[i * L + j] = v.x;
      fc[i * L + j] = v.y;
    }
  const double det = cofactors_rt(cof, d, L);
  double f = f0 * det;
  for (int i = 0; i < L * L; ++i) f -= cof[i] * fc[i];
  *det_out = det;
  *f_out = f;
}

// m > 0: sum over the distributions (m_1; m_col_1..L) with sum m (onebody.rs, helpers.rs:682-712);
// the column-replacement correction is formed as in the reference, sum_r (F - D) cof, so that
// det + correction replaces column c by the Fock column.
NW_HD double spin_f_gen_hd(int m, const double* const (*ff_t)[2], const double* f0f, int n, int l, const int* rows,
                           const int* cols, const double* d0, const double* d1, double tol, bool exact) {
  double acc = 0.0;
  double dm[kML * kML], cof[kML * kML];
  uint64_t bits;
  bool more = first_combination(l + 1, m, &bits);
  while (more) {
    const int mi = bitk(bits, 0);
    const uint64_t cb = bits >> 1;
    mix_rt(dm, d0, d1, l, cb);
    double det = 1.0;
    bool ok = true;
    if (l > 0) {
      if (exact)
        det = cofactors_rt(cof, dm, l);
      else
        ok = cofactors_tol_rt(cof, dm, l, tol, &det);
    }
    if (ok) {
      double contrib = det * f0f[mi];
      for (int b = 0; b < l; ++b) {
        const double* fsl = ff_t[mi][bitk(cb, b)];
        const int64_t base = (int64_t)cols[b] * n;
        double corr = 0.0;
        for (int r = 0; r < l; ++r) corr += (fsl[base + rows[r]] - dm[r * l + b]) * cof[r * l + b];
        contrib -= det + corr;
      }
      acc += contrib;
    }
    more = advance_combination(l + 1, m, &bits);
  }
  return acc;
}

NW_HD void combine_fs(double ph, double pa, double deta, double fa, double pb, double detb, double fb, double* F,
                      double* S) {
  const double sa = pa * deta, sb = pb * detb;
  double f = 0.0;
  if (sb != 0.0) f += pa * fa * sb;
  if (sa != 0.0) f += pb * fb * sa;
  *F = ph * f;
  *S = ph * sa * sb;
}

template <int LA, int LB>
NW_HD void eval_fs_m0_ct(const FastPair& fp, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                         int ob, double* F, double* S) {
  int ra[LA > 0 ? LA : 1], ca[LA > 0 ? LA : 1], rb[LB > 0 ? LB : 1], cb[LB > 0 ? LB : 1];
  det_labels_ct<LA>(x.ra, x.ia, w.ia, oa, n, ra, ca);
  det_labels_ct<LB>(x.rb, x.ib, w.ib, ob, n, rb, cb);
  double deta, fa, detb, fb;
  spin_f_ct<LA>(fk.a.recx, fk.a.recy, fk.a.f0f[0], n, ra, ca, &deta, &fa);
  spin_f_ct<LB>(fk.b.recx, fk.b.recy, fk.b.f0f[0], n, rb, cb, &detb, &fb);
  combine_fs(x.phase * w.phase, fp.a.pref, deta, fa, fp.b.pref, detb, fb, F, S);
}

NW_HD void eval_fs_m0_rt(const FastPair& fp, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                         int ob, double* F, double* S) {
  int ra[kML], ca[kML], rb[kML], cb[kML];
  labels_rt(x, w, 0, oa, n, ra, ca);
  labels_rt(x, w, 1, ob, n, rb, cb);
  double deta, fa, detb, fb;
  spin_f_rt(x.ra + w.ra, fk.a.recx, fk.a.recy, fk.a.f0f[0], n, ra, ca, &deta, &fa);
  spin_f_rt(x.rb + w.rb, fk.b.recx, fk.b.recy, fk.b.f0f[0], n, rb, cb, &detb, &fb);
  combine_fs(x.phase * w.phase, fp.a.pref, deta, fa, fp.b.pref, detb, fb, F, S);
}

#define NW_FS_CASE(A, B)                                       \
  case (A) * 5 + (B):                                          \
    eval_fs_m0_ct<A, B>(fp, fk, x, w, n, oa, ob, F, S);        \
    return;

// Rank dispatch of the m = 0 (F, S) evaluator for one pair (the kernels dispatch per class).
NW_HD void eval_fs_m0_pair(const FastPair& fp, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                           int ob, double* F, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  if (la <= 4 && lb <= 4) {
    switch (la * 5 + lb) {
      NW_FS_CASE(0, 0) NW_FS_CASE(0, 1) NW_FS_CASE(0, 2) NW_FS_CASE(0, 3) NW_FS_CASE(0, 4)
      NW_FS_CASE(1, 0) NW_FS_CASE(1, 1) NW_FS_CASE(1, 2) NW_FS_CASE(1, 3) NW_FS_CASE(1, 4)
      NW_FS_CASE(2, 0) NW_FS_CASE(2, 1) NW_FS_CASE(2, 2) NW_FS_CASE(2, 3) NW_FS_CASE(2, 4)
      NW_FS_CASE(3, 0) NW_FS_CASE(3, 1) NW_FS_CASE(3, 2) NW_FS_CASE(3, 3) NW_FS_CASE(3, 4)
      NW_FS_CASE(4, 0) NW_FS_CASE(4, 1) NW_FS_CASE(4, 2) NW_FS_CASE(4, 3) NW_FS_CASE(4, 4)
      default: break;
    }
  }
  eval_fs_m0_rt(fp, fk, x, w, n, oa, ob, F, S);
}
#undef NW_FS_CASE

NW_HD void eval_fs_gen_pair(const GenPair& g, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                            int ob, double tol, bool exact, double* F, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  int ra[kML], ca[kML], rb[kML], cb[kML];
  labels_rt(x, w, 0, oa, n, ra, ca);
  labels_rt(x, w, 1, ob, n, rb, cb);
  double d0[kML * kML], d1[kML * kML];
  build_d_rt(d0, g.a.x[0], g.a.y[0], n, la, ra, ca);
  build_d_rt(d1, g.a.x[1], g.a.y[1], n, la, ra, ca);
  const double deta = overlap_spin_hd(g.a.m, la, d0, d1);
  const double fa = spin_f_gen_hd(g.a.m, fk.a.ff_t, fk.a.f0f, n, la, ra, ca, d0, d1, tol, exact);
  build_d_rt(d0, g.b.x[0], g.b.y[0], n, lb, rb, cb);
  build_d_rt(d1, g.b.x[1], g.b.y[1], n, lb, rb, cb);
  const double detb = overlap_spin_hd(g.b.m, lb, d0, d1);
  const double fb = spin_f_gen_hd(g.b.m, fk.b.ff_t, fk.b.f0f, n, lb, rb, cb, d0, d1, tol, exact);
  combine_fs(x.phase * w.phase, g.a.pref, deta, fa, g.b.pref, detb, fb, F, S);
}

// Compile-time-L (<= 4 per spin) twins of overlap_spin_hd, spin_f_gen_hd and eval_fs_gen_pair:
// the same terms in the same order, with the distribution matrices and cofactors in registers.
template <int L>
NW_HD double overlap_spin_ct(int m, const double (&d0)[Sq<L>::v], const double (&d1)[Sq<L>::v]) {
  if (m > L) return 0.0;
  if (m == 0) return det_small(d0, L);
  if (m == L) return det_small(d1, L);
  double acc = 0.0;
  uint64_t bits;
  bool more = first_combination(L, m, &bits);
  while (more) {
    double dm[Sq<L>::v];
    mix_ct<L>(dm, d0, d1, bits);
    acc += det_small(dm, L);
    more = advance_combination(L, m, &bits);
  }
  return acc;
}

template <int L>
NW_HD double spin_f_gen_ct(int m, const double* const (*ff_t)[2], const double* f0f, int n, const int* rows,
                           const int* cols, const double (&d0)[Sq<L>::v], const double (&d1)[Sq<L>::v], double tol,
                           bool exact) {
  double acc = 0.0;
  uint64_t bits;
  bool more = first_combination(L + 1, m, &bits);
  while (more) {
    const int mi = bitk(bits, 0);
    const uint64_t cb = bits >> 1;
    double dm[Sq<L>::v], cof[Sq<L>::v];
    mix_ct<L>(dm, d0, d1, cb);
    double det = 1.0;
    bool ok = true;
    if (L > 0) {
      if (exact)
        det = cofactors_ct<L>(cof, dm);
      else
        ok = cofactors_tol_ct<L>(cof, dm, tol, &det);
    }
    if (ok) {
      double contrib = det * f0f[mi];
#pragma unroll
      for (int b = 0; b < L; ++b) {
        const double* fsl = ff_t[mi][bitk(cb, b)];
        const int64_t base = (int64_t)cols[b] * n;
        double corr = 0.0;
#pragma unroll
        for (int r = 0; r < L; ++r) corr += (ldg_d(fsl + base + rows[r]) - dm[r * L + b]) * cof[r * L + b];
        contrib -= det + corr;
      }
      acc += contrib;
    }
    more = advance_combination(L + 1, m, &bits);
  }
  return acc;
}

template <int LA, int LB>
NW_HD void eval_fs_gen_ct(const GenPair& g, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                          int ob, double tol, bool exact, double* F, double* S) {
  int ra[LA > 0 ? LA : 1], ca[LA > 0 ? LA : 1], rb[LB > 0 ? LB : 1], cb[LB > 0 ? LB : 1];
  det_labels_ct<LA>(x.ra, x.ia, w.ia, oa, n, ra, ca);
  det_labels_ct<LB>(x.rb, x.ib, w.ib, ob, n, rb, cb);
  double d0[Sq<LA>::v], d1[Sq<LA>::v];
  build_d_ct<LA>(d0, g.a.x[0], g.a.y[0], n, ra, ca);
  build_d_ct<LA>(d1, g.a.x[1], g.a.y[1], n, ra, ca);
  const double deta = overlap_spin_ct<LA>(g.a.m, d0, d1);
  const double fa = spin_f_gen_ct<LA>(g.a.m, fk.a.ff_t, fk.a.f0f, n, ra, ca, d0, d1, tol, exact);
  double e0[Sq<LB>::v], e1[Sq<LB>::v];
  build_d_ct<LB>(e0, g.b.x[0], g.b.y[0], n, rb, cb);
  build_d_ct<LB>(e1, g.b.x[1], g.b.y[1], n, rb, cb);
  const double detb = overlap_spin_ct<LB>(g.b.m, e0, e1);
  const double fb = spin_f_gen_ct<LB>(g.b.m, fk.b.ff_t, fk.b.f0f, n, rb, cb, e0, e1, tol, exact);
  combine_fs(x.phase * w.phase, g.a.pref, deta, fa, g.b.pref, detb, fb, F, S);
}

template <int LA, int LB>
NW_HD_CALL void eval_fs_gen_case(const GenPair& g, const FockPair& fk, const DetRec& x, const DetRec& w, int n,
                                 int oa, int ob, double tol, bool exact, double* F, double* S) {
  eval_fs_gen_ct<LA, LB>(g, fk, x, w, n, oa, ob, tol, exact, F, S);
}

#define NW_FS_GEN_CASE(A, B)                                                   \
  case (A) * 5 + (B):                                                          \
    eval_fs_gen_case<A, B>(g, fk, x, w, n, oa, ob, tol, exact, F, S);          \
    return;

// m > 0 (F, S) of one pair: the register twin (one call per (L_alpha, L_beta) case) for
// contraction ranks up to 4 per spin, the runtime-size path above that.
NW_HD void eval_fs_gen_any(const GenPair& g, const FockPair& fk, const DetRec& x, const DetRec& w, int n, int oa,
                           int ob, double tol, bool exact, double* F, double* S) {
  const int la = x.ra + w.ra, lb = x.rb + w.rb;
  if (la <= 4 && lb <= 4) {
    switch (la * 5 + lb) {
      NW_FS_GEN_CASE(0, 0) NW_FS_GEN_CASE(0, 1) NW_FS_GEN_CASE(0, 2) NW_FS_GEN_CASE(0, 3) NW_FS_GEN_CASE(0, 4)
      NW_FS_GEN_CASE(1, 0) NW_FS_GEN_CASE(1, 1) NW_FS_GEN_CASE(1, 2) NW_FS_GEN_CASE(1, 3) NW_FS_GEN_CASE(1, 4)
      NW_FS_GEN_CASE(2, 0) NW_FS_GEN_CASE(2, 1) NW_FS_GEN_CASE(2, 2) NW_FS_GEN_CASE(2, 3) NW_FS_GEN_CASE(2, 4)
      NW_FS_GEN_CASE(3, 0) NW_FS_GEN_CASE(3, 1) NW_FS_GEN_CASE(3, 2) NW_FS_GEN_CASE(3, 3) NW_FS_GEN_CASE(3, 4)
      NW_FS_GEN_CASE(4, 0) NW_FS_GEN_CASE(4, 1) NW_FS_GEN_CASE(4, 2) NW_FS_GEN_CASE(4, 3) NW_FS_GEN_CASE(4, 4)
      default: break;
    }
  }
  eval_fs_gen_pair(g, fk, x, w, n, oa, ob, tol, exact, F, S);
}
#undef NW_FS_GEN_CASE

// ---------------------------------------------------------------------------------------
// Layout formulas of the build.  T4 buffers hold T(A,B,C,D)[p,q,r,s] at [p][r][q][s].
// ---------------------------------------------------------------------------------------
// antisymmetrised J^(0000): J[a,b,c,d] - J[a,d,c,b] with J in stored [i,j,r,c] order
NW_HD double jas_at(const double* td, const double* te, int64_t n, int64_t a, int64_t b, int64_t c, int64_t d) {
  const int64_t n2 = n * n, n3 = n2 * n;
  return td[c * n3 + a * n2 + d * n + b] - te[c * n3 + d * n2 + a * n + b] - td[c * n3 + a * n2 + b * n + d] +
         te[c * n3 + b * n2 + a * n + d];
}
// J in stored [i,j,r,c] order (layout.rs:367-392): constructed[c,d,a,b]
NW_HD double jstored_at(const double* td, const double* te, int64_t n, int64_t a, int64_t b, int64_t c, int64_t d) {
  const int64_t n2 = n * n, n3 = n2 * n;
  return td[c * n3 + a * n2 + d * n + b] - te[c * n3 + d * n2 + a * n + b];
}
// II in stored [r,c,i,j] order
NW_HD double ii_at(const double* t4, int64_t n, int64_t r, int64_t c, int64_t i, int64_t j) {
  const int64_t n2 = n * n, n3 = n2 * n;
  return t4[r * n3 + i * n2 + c * n + j];
}

}  // namespace nw
