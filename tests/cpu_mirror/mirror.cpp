// CPU build of the engine's per-pair device code, for tests only.
//
// Compiles noci-rs_b200/csrc/wick_math.cuh (the functions the CUDA kernels call) with g++
// and exposes them through a C ABI so the tests can check, without a GPU, the index
// arithmetic, layout formulas, SVD pairing and evaluators of the kernels against the FP64
// oracle.  This library is not part of the product and is never loaded by it.
#include <cstdint>
#include <cstring>

#include "../../noci-rs_b200/csrc/qmc_math.cuh"
#include "../../noci-rs_b200/csrc/wick_math.cuh"

using namespace nw;

namespace {
constexpr int kSpinOffs = 27;
constexpr int kNoff = 2 * kSpinOffs + 32;
constexpr int kNval = 22;
constexpr int kNint = 5;

const double* at(const double* base, int64_t off) { return off < 0 ? nullptr : base + off; }

// GenPair from the oracle's packed reference-order tables (same offsets as oracle/wick_eval.cpp).
GenPair gen_from_oracle(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints) {
  GenPair g;
  std::memset(&g, 0, sizeof(g));
  GenSpin* sv[2] = {&g.a, &g.b};
  for (int s = 0; s < 2; ++s) {
    const int64_t* o = offs + s * kSpinOffs;
    GenSpin& v = *sv[s];
    int k = 0;
    for (int i = 0; i < 2; ++i) v.x[i] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i) v.y[i] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) v.fh_t[i][j] = at(slab, o[k++]);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        for (int l = 0; l < 2; ++l) v.v_t[i][j][l] = at(slab, o[k++]);
    ++k;  // hcol0
    for (int i = 0; i < 10; ++i) v.j[i] = at(slab, o[k++]);
    const double* vv = vals + s * 7;
    v.pref = vv[0] * vv[1];
    v.f0h[0] = vv[2];
    v.f0h[1] = vv[3];
    v.v0[0] = vv[4];
    v.v0[1] = vv[5];
    v.v0[2] = vv[6];
    v.m = ints[2 * s];
  }
  const int64_t* o = offs + 2 * kSpinOffs;
  int k = 0;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) g.vab_t[a][b][c] = at(slab, o[k++]);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) g.vba_t[a][b][c] = at(slab, o[k++]);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c)
        for (int d = 0; d < 2; ++d) g.ii[a][b][c][d] = at(slab, o[k++]);
  const double* dv = vals + 14;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      g.vab0[a][b] = dv[a * 2 + b];
      g.vba0[a][b] = dv[4 + a * 2 + b];
    }
  return g;
}

DetRec rec_at(const void* dets, uint32_t i) {
  uint64_t w[4];
  std::memcpy(w, static_cast<const char*>(dets) + 32ull * i, 32);
  return unpack_det(w[0], w[1], w[2], w[3]);
}
}  // namespace

extern "C" {

// NOCI-QMC arithmetic (qmc_math.cuh).
void mir_philox(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
  const nwq::U4 r = nwq::philox4x32_10(nwq::U4{ctr[0], ctr[1], ctr[2], ctr[3]}, k0, k1);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}
void mir_uniform2(uint64_t seed, uint64_t cycle, uint64_t index, uint32_t purpose, double* out) {
  nwq::uniform2(seed, cycle, index, purpose, &out[0], &out[1]);
}
double mir_fri(double x, double c, double u) { return nwq::fri(x, c, u); }
uint64_t mir_uniform_child(uint64_t g, uint64_t n, double u) { return nwq::uniform_child(g, n, u); }
uint64_t mir_attempts(double n) { return nwq::attempts(n); }
double mir_diagonal_change(int prop, double dt, double es, double h, double s, double n) {
  return nwq::diagonal_change(prop, dt, es, h, s, n);
}

int mir_layout_sizes(int which) { return which == 0 ? kNoff : which == 1 ? kNval : kNint; }

void mir_unpack(const void* dets, int64_t n, int32_t* parent, int32_t* ra, int32_t* rb, uint64_t* ia, uint64_t* ib,
                double* phase) {
  for (int64_t i = 0; i < n; ++i) {
    const DetRec d = rec_at(dets, (uint32_t)i);
    parent[i] = (int32_t)d.parent;
    ra[i] = d.ra;
    rb[i] = d.rb;
    ia[i] = d.ia;
    ib[i] = d.ib;
    phase[i] = d.phase;
  }
}

int mir_far_same_parent(const void* dets, uint32_t a, uint32_t b) {
  return far_same_parent(rec_at(dets, a), rec_at(dets, b)) ? 1 : 0;
}

// The sort keys of the evaluation pipeline (classify_kernel) for a request, with the key plan
// (sort_key_shift) of a counter budget `cap`: keys[i] (0xFFFFFFFF for same-parent pairs that
// are more than a double excitation apart), returns the number of keys, nbucket/shift out.
uint64_t mir_sort_keys(const void* dets, uint64_t ndet, int nref, const int32_t* order, int nfast,
                       const uint32_t* pairs, uint64_t npairs, uint64_t cap, uint32_t* keys, uint32_t* nbucket,
                       int32_t* shift) {
  uint32_t nb = 1;
  const int s = sort_key_shift(ndet, nref, cap, &nb);
  *nbucket = nb;
  *shift = s;
  for (uint64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    const uint32_t dx = det_desc(x.parent, x.ra, x.rb), dw = det_desc(w.parent, w.ra, w.rb);
    const int px = (int)(dx & 0xFF), pw = (int)(dw & 0xFF);
    if (px == pw && far_same_parent(x, w)) {
      keys[i] = 0xFFFFFFFFu;
      continue;
    }
    const int la = (int)((dx >> 8) & 15) + (int)((dw >> 8) & 15), lb = (int)(dx >> 12) + (int)(dw >> 12);
    keys[i] = pair_sort_key(la, lb, pairs[2 * i], pw, order[px * nref + pw], nfast, ndet, nb, s);
  }
  return (uint64_t)kRankClasses * nb + (uint64_t)kGenClasses * ((uint64_t)nref * nref - nfast);
}

// Labels through the register (compile-time L) path and the runtime path.
int mir_labels(const void* dets, uint32_t a, uint32_t b, int spin, int nocc, int n, int32_t* rows_ct, int32_t* cols_ct,
               int32_t* rows_rt, int32_t* cols_rt) {
  const DetRec x = rec_at(dets, a), w = rec_at(dets, b);
  const int L = spin ? x.rb + w.rb : x.ra + w.ra;
  int r[8], c[8];
  labels_rt(x, w, spin, nocc, n, r, c);
  for (int k = 0; k < L; ++k) {
    rows_rt[k] = r[k];
    cols_rt[k] = c[k];
  }
  const int rx = spin ? x.rb : x.ra;
  const uint64_t ix = spin ? x.ib : x.ia, iw = spin ? w.ib : w.ia;
  switch (L) {
    case 1: det_labels_ct<1>(rx, ix, iw, nocc, n, r, c); break;
    case 2: det_labels_ct<2>(rx, ix, iw, nocc, n, r, c); break;
    case 3: det_labels_ct<3>(rx, ix, iw, nocc, n, r, c); break;
    case 4: det_labels_ct<4>(rx, ix, iw, nocc, n, r, c); break;
    default: break;
  }
  for (int k = 0; k < L && L <= 4; ++k) {
    rows_ct[k] = r[k];
    cols_ct[k] = c[k];
  }
  return L;
}

void mir_svd(int o, const double* a_in, double tol, double* u, double* v, double* s, double* phase) {
  double a[64 * 64], scratch[64 * 64];
  std::memcpy(a, a_in, sizeof(double) * o * o);
  jacobi_svd(o, a, u, v, s, tol);
  canonical_null_columns(o, u, s, tol);
  canonical_null_columns(o, v, s, tol);
  std::memcpy(scratch, u, sizeof(double) * o * o);
  const double du = det_lu_inplace(scratch, o);
  std::memcpy(scratch, v, sizeof(double) * o * o);
  const double dv = det_lu_inplace(scratch, o);
  *phase = du * dv;
}

// One ordered reference pair on the fast layout; recx/recy as interleaved {value, hcol0}.
void mir_eval_fast(const double* recx_a, const double* recy_a, const double* jas_a, const double* recx_b,
                   const double* recy_b, const double* jas_b, const double* ii0, double pref_a, double g0_a,
                   double pref_b, double g0_b, double vab0, int n, int oa, int ob, double enuc, const void* dets,
                   const uint32_t* pairs, int64_t npairs, double* hs) {
  FastPair fp;
  fp.a.recx = reinterpret_cast<const double2*>(recx_a);
  fp.a.recy = reinterpret_cast<const double2*>(recy_a);
  fp.a.jas = jas_a;
  fp.a.pref = pref_a;
  fp.a.g0 = g0_a;
  fp.b.recx = reinterpret_cast<const double2*>(recx_b);
  fp.b.recy = reinterpret_cast<const double2*>(recy_b);
  fp.b.jas = jas_b;
  fp.b.pref = pref_b;
  fp.b.g0 = g0_b;
  fp.ii0 = ii0;
  fp.vab0 = vab0;
  fp.pad = 0.0;
  for (int64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    eval_m0_pair(fp, x, w, n, oa, ob, enuc, &hs[2 * i], &hs[2 * i + 1]);
  }
}

// One ordered reference pair on the reference-ordered layout (m > 0 path): the runtime-size
// evaluator for every pair (dispatch 0), or the kernel's dispatch (dispatch 1: the register
// twins up to rank 4 per spin).
void mir_eval_gen(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int n, int oa,
                  int ob, double enuc, double tol, int exact, const void* dets, const uint32_t* pairs, int64_t npairs,
                  double* hs, int dispatch) {
  const GenPair g = gen_from_oracle(slab, offs, vals, ints);
  for (int64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    if (dispatch)
      eval_gen_any(g, x, w, n, oa, ob, enuc, tol, exact != 0, &hs[2 * i], &hs[2 * i + 1]);
    else
      eval_gen_pair(g, x, w, n, oa, ob, enuc, tol, exact != 0, &hs[2 * i], &hs[2 * i + 1]);
  }
}

void mir_eval_s_gen(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints, int n, int oa,
                    int ob, const void* dets, const uint32_t* pairs, int64_t npairs, double* s) {
  const GenPair g = gen_from_oracle(slab, offs, vals, ints);
  for (int64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    s[i] = eval_s_pair(nullptr, &g, x, w, n, oa, ob);
  }
}

// (F, S) on the fast layout: Fock records {X0|Y0, F^(00)} interleaved, F_0^(0) and pref per spin.
void mir_eval_fs_fast(const double* frecx_a, const double* frecy_a, double f0_a, double pref_a, const double* frecx_b,
                      const double* frecy_b, double f0_b, double pref_b, int n, int oa, int ob, const void* dets,
                      const uint32_t* pairs, int64_t npairs, double* fs) {
  FastPair fp;
  std::memset(&fp, 0, sizeof(fp));
  fp.a.pref = pref_a;
  fp.b.pref = pref_b;
  FockPair fk;
  std::memset(&fk, 0, sizeof(fk));
  fk.a.recx = reinterpret_cast<const double2*>(frecx_a);
  fk.a.recy = reinterpret_cast<const double2*>(frecy_a);
  fk.a.f0f[0] = f0_a;
  fk.b.recx = reinterpret_cast<const double2*>(frecx_b);
  fk.b.recy = reinterpret_cast<const double2*>(frecy_b);
  fk.b.f0f[0] = f0_b;
  for (int64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    eval_fs_m0_pair(fp, fk, x, w, n, oa, ob, &fs[2 * i], &fs[2 * i + 1]);
  }
}

// (F, S) on the reference-ordered layout: ff_t[spin][mi*2+mj] transposed Fock columns.
void mir_eval_fs_gen(const double* slab, const int64_t* offs, const double* vals, const int32_t* ints,
                     const double* fslab, const int64_t* foffs, const double* fvals, int n, int oa, int ob, double tol,
                     int exact, const void* dets, const uint32_t* pairs, int64_t npairs, double* fs, int dispatch) {
  const GenPair g = gen_from_oracle(slab, offs, vals, ints);
  FockPair fk;
  std::memset(&fk, 0, sizeof(fk));
  FockSpinTab* t[2] = {&fk.a, &fk.b};
  for (int sp = 0; sp < 2; ++sp) {
    for (int k = 0; k < 4; ++k) t[sp]->ff_t[k >> 1][k & 1] = fslab + foffs[sp * 4 + k];
    t[sp]->f0f[0] = fvals[sp * 2];
    t[sp]->f0f[1] = fvals[sp * 2 + 1];
  }
  for (int64_t i = 0; i < npairs; ++i) {
    const DetRec x = rec_at(dets, pairs[2 * i]), w = rec_at(dets, pairs[2 * i + 1]);
    if (dispatch)  // the kernel's dispatch: register twins up to rank 4 per spin
      eval_fs_gen_any(g, fk, x, w, n, oa, ob, tol, exact != 0, &fs[2 * i], &fs[2 * i + 1]);
    else
      eval_fs_gen_pair(g, fk, x, w, n, oa, ob, tol, exact != 0, &fs[2 * i], &fs[2 * i + 1]);
  }
}

void mir_layout(int which, const double* td, const double* te, int64_t n, double* out) {
  const int64_t n4 = n * n * n * n;
  for (int64_t idx = 0; idx < n4; ++idx) {
    const int64_t a = idx / (n * n * n), b = (idx / (n * n)) % n, c = (idx / n) % n, d = idx % n;
    out[idx] = which == 0 ? jas_at(td, te, n, a, b, c, d)
                          : which == 1 ? jstored_at(td, te, n, a, b, c, d) : ii_at(td, n, a, b, c, d);
  }
}

}  // extern "C"
