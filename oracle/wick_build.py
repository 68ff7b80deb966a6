"""CPU oracle (test infrastructure only): per-reference-pair Wick intermediates in FP64 numpy.

Restates src/nonorthogonalwicks/build.rs of dy-cl/noci-rs for real orbitals.  Only tests/,
the smoke check and the CPU-baseline leg of bench.py may use this module.

Reference items restated (file:line inside dy-cl/noci-rs):
  * SAME_SPIN_J_BRANCHES                 src/nonorthogonalwicks/build.rs:19-30
  * SameSpinBuild::new                   src/nonorthogonalwicks/build.rs:86-334
  * count_zero_overlap_pairs             src/nonorthogonalwicks/build.rs:350-363
  * perform_ortho_and_svd_and_rotate     src/nonorthogonalwicks/build.rs:401-424
  * construct_m                          src/nonorthogonalwicks/build.rs:447-503
  * construct_xy                         src/nonorthogonalwicks/build.rs:526-542
  * construct_f_scalar                   src/nonorthogonalwicks/build.rs:564-617
  * build_j_coulomb / build_k_exchange   src/nonorthogonalwicks/build.rs:627-683
  * DiffSpinBuild::new                   src/nonorthogonalwicks/build.rs:728-926
  * build_cx_xc                          src/nonorthogonalwicks/build.rs:944-991
  * contraction_orbitals                 src/nonorthogonalwicks/build.rs:1008-1031
  * eri_ao2mo_into (real)                src/maths/eri.rs:83-152,258-
  * build_wicks_pair / plan_wicks_pairs  src/noci/wicks.rs:37-121
  * write4ijrc / write2t / write_hcol0    src/nonorthogonalwicks/layout.rs:283-392

Conventions: AO integrals in chemists' order eri[mu,nu,lam,sig] = (mu nu|lam sig)
(scripts/generate.py:14, PySCF int2e s1).  The ordered pair (x, w) is (bra, ket): the
reference calls SameSpinBuild::new(ao, g = ref[w], l = ref[x]).

Parity status: pinned against reference-produced numbers.  The reference's own energy
fixtures (tests/fixtures/*/expected.json of noci-rs: reference-space NOCI, deterministic
SD-space, NOCI-PT2 and selected-NOCI energies of H2, H4, LiH and F2) are reproduced from
integrals and SCF states rebuilt by tests/golden/make_reference_fixtures.py
(tests/test_reference_fixtures.py); the oracle is also cross-checked against an independent
generalised Slater-Condon path and a brute-force Fock-space evaluation.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

SAME_SPIN_J_BRANCHES: List[Tuple[int, int, int, int]] = [
    (0, 0, 0, 0), (0, 0, 0, 1), (0, 0, 1, 0), (0, 0, 1, 1), (0, 1, 0, 1),
    (0, 1, 1, 0), (0, 1, 1, 1), (1, 0, 1, 0), (1, 0, 1, 1), (1, 1, 1, 1),
]


def occ_coeffs(c: np.ndarray, occ: int) -> np.ndarray:
    """Columns of ``c`` selected by the occupation bit string (src/noci/naive.rs:20-32)."""
    idx = [i for i in range(c.shape[1]) if (occ >> i) & 1]
    return c[:, idx]


def contraction_orbitals(cx: np.ndarray, cw: np.ndarray, nocc: int):
    """Row space V_x u O_w and column space O_x u V_w (build.rs:1008-1031).

    Like the reference, this takes the first ``nocc`` columns as the occupied block.
    """
    rowc = np.hstack([cx[:, nocc:], cw[:, :nocc]])
    colc = np.hstack([cx[:, :nocc], cw[:, nocc:]])
    return rowc, colc


def canonical_null_gauge(u: np.ndarray, v: np.ndarray, s: np.ndarray, tol: float):
    """Fix the free rotation of the zero-singular-value columns of U and V.

    The SVD leaves the columns of U and V that belong to zero singular values determined only
    up to independent orthogonal transformations (for one zero, independent signs).  The exact
    matrix elements do not depend on that choice, but the reference evaluator's handling of
    zero-overlap pairs does, so the choice is fixed here by a rule any SVD routine can
    reproduce: with U0 the null columns, B = U0^T is factored B = Q R by modified Gram-Schmidt
    over its columns (a column whose residual norm is <= 1e-10 is skipped) with R's diagonal
    positive, and U0 is replaced by U0 Q; the same for V.  The CUDA build applies the same
    rule (canonical_null_columns in noci-rs_b200/csrc/wick_math.cuh).
    Returns the new (u, v) and the factor det(Q_U) det(Q_V).
    """
    zeros = [k for k, val in enumerate(s) if abs(val) <= tol]
    m = len(zeros)
    if m < 1:
        return u, v, 1.0
    fac = 1.0
    out = []
    for mat in (u, v):
        m0 = mat[:, zeros]
        bt = m0.T                      # m x o; its columns are the rows of U0
        q = np.zeros((m, m))
        found = 0
        for col in range(bt.shape[1]):
            if found == m:
                break
            w = bt[:, col].copy()
            for _ in range(2):
                for f in range(found):
                    w -= q[:, f] * (q[:, f] @ w)
            nrm = float(np.sqrt(w @ w))
            if nrm <= 1e-10:
                continue
            q[:, found] = w / nrm
            found += 1
        if found < m:
            out.append(mat)
            continue
        fac *= float(np.linalg.det(q))
        mat = mat.copy()
        mat[:, zeros] = m0 @ q
        out.append(mat)
    return out[0], out[1], fac


def ortho_svd_rotate(s_ao: np.ndarray, cx_occ: np.ndarray, cw_occ: np.ndarray,
                     tol: float = 0.0, null_gauge: Optional[np.random.Generator] = None,
                     canonical: bool = True):
    """Loewdin pairing: S_occ = U s V^T, rotated occupied sets and phase det(U) det(V).

    Follows build.rs:401-424; when zero singular values are present the null-space gauge is
    fixed by ``canonical_null_gauge``.  ``null_gauge`` (tests only) first applies random
    independent rotations to the null columns of U and V, as a different SVD routine might.
    """
    s_occ = cx_occ.T @ s_ao @ cw_occ
    u, s, vt = np.linalg.svd(s_occ)
    v = vt.T
    zeros = [k for k, val in enumerate(s) if abs(val) <= tol]
    if null_gauge is not None and zeros:
        u, v = u.copy(), v.copy()
        for mat in (u, v):
            q, _ = np.linalg.qr(null_gauge.standard_normal((len(zeros), len(zeros))))
            if null_gauge.random() < 0.5:
                q[:, 0] *= -1.0            # include reflections (one-sided sign flips)
            mat[:, zeros] = mat[:, zeros] @ q
    if canonical:
        u, v, _ = canonical_null_gauge(u, v, s, tol)
    phase = float(np.linalg.det(u) * np.linalg.det(v))
    return s, cw_occ @ v, cx_occ @ u, phase


def construct_m(s: np.ndarray, cx_t: np.ndarray, cw_t: np.ndarray, zeros: List[int], tol: float):
    """M^(0) = W + P_xw + P_ww and M^(1) = P_xw in the AO basis (build.rs:447-503)."""
    nb = cw_t.shape[0]
    scale = np.array([1.0 / v if abs(v) > tol else 0.0 for v in s])
    m0 = (cw_t * scale[None, :]) @ cx_t.T
    m1 = np.zeros((nb, nb))
    for k in zeros:
        m0 += np.outer(cw_t[:, k], cw_t[:, k])
    for k in zeros:
        p = np.outer(cw_t[:, k], cx_t[:, k])
        m1 += p
        m0 += p
    return m0, m1


def construct_xy(rowc, colc, s_ao, m, subtract: bool):
    """X^(m) = C_row^T S M S C_col and Y^(m) (build.rs:526-542)."""
    xr = s_ao @ m @ s_ao
    yr = xr - s_ao if subtract else xr
    return rowc.T @ xr @ colc, rowc.T @ yr @ colc


def build_cx_xc(m, s_ao, cx, cw, nocc: int, i: int):
    """Left/right partial transforms restricted to the determinant rows/columns (build.rs:944-991)."""
    f = float(1 - i)
    ms = m @ s_ao
    mts = m.T @ s_ao
    left_x = mts @ cx - f * cx
    left_w = mts @ cw
    right_x = ms @ cx
    right_w = ms @ cw - f * cw
    cxm = np.hstack([left_x[:, nocc:], left_w[:, :nocc]])
    xcm = np.hstack([right_x[:, :nocc], right_w[:, nocc:]])
    return cxm, xcm


def j_coulomb(eri: np.ndarray, m: np.ndarray) -> np.ndarray:
    """J_st = sum_{mu nu} (st|mu nu) M_{mu nu} (build.rs:627-652)."""
    n = m.shape[0]
    return (eri.reshape(n * n, n * n) @ m.reshape(n * n)).reshape(n, n)


def k_exchange(eri: np.ndarray, m: np.ndarray) -> np.ndarray:
    """K_st = sum_{mu nu} (s mu|nu t) M_{mu nu} (build.rs:654-683)."""
    return np.einsum("smnt,mn->st", eri, m, optimize=True)


def einsum_ba_ab(a: np.ndarray, b: np.ndarray) -> float:
    """sum_{ab} A[b,a] B[a,b] = tr(A B) (src/maths/einsum.rs)."""
    return float(np.einsum("ba,ab->", a, b))


def ao2mo(eri: np.ndarray, c1, c2, c3, c4) -> np.ndarray:
    """out[p,q,r,s] = sum (mu nu|lam sig) c1[mu,p] c2[nu,q] c3[lam,r] c4[sig,s] (eri.rs:258-)."""
    t = np.tensordot(c1, eri, axes=(0, 0))            # p nu lam sig
    t = np.tensordot(t, c2, axes=(1, 0))               # p lam sig q
    t = np.tensordot(t, c3, axes=(1, 0))               # p sig q r
    t = np.tensordot(t, c4, axes=(1, 0))               # p q r s
    return np.ascontiguousarray(t)


@dataclass
class SameSpin:
    """Same-spin intermediates of one ordered reference pair (fields of SameSpinBuild)."""

    x: List[np.ndarray]
    y: List[np.ndarray]
    f0h: List[float]
    fh: List[List[np.ndarray]]
    v0: List[float]
    v: List[List[List[np.ndarray]]]          # v[m1][m3][m2] = cx[m1]^T JK[m2] xc[m3]
    j: Dict[int, np.ndarray]                 # slot -> J tensor in constructed [r,c,i,j] order
    tilde_s_prod: float
    phase: float
    m: int
    nmo: int
    nocc: int
    singular_values: np.ndarray
    f0f: List[float] = field(default_factory=lambda: [0.0, 0.0])
    ff: Optional[List[List[np.ndarray]]] = None
    mao: Optional[List[np.ndarray]] = None
    cx: Optional[List[np.ndarray]] = None
    xc: Optional[List[np.ndarray]] = None


@dataclass
class DiffSpin:
    vab0: List[List[float]]
    vba0: List[List[float]]
    vab: List[List[List[np.ndarray]]]
    vba: List[List[List[np.ndarray]]]
    ii: Dict[Tuple[int, int, int, int], np.ndarray]


@dataclass
class PairBuild:
    aa: SameSpin
    bb: SameSpin
    ab: DiffSpin
    hcol0_a: Optional[np.ndarray]
    hcol0_b: Optional[np.ndarray]


def same_spin_build(s_ao, h, eri, cx, occx: int, cw, occw: int, tol: float,
                    null_gauge: Optional[np.random.Generator] = None) -> SameSpin:
    """SameSpinBuild::new for the ordered pair (bra x, ket w) (build.rs:86-334).

    ``null_gauge`` (tests only) applies a random orthogonal rotation inside the zero-overlap
    singular subspaces, to check that matrix elements do not depend on that SVD gauge.
    """
    nmo = cw.shape[1]
    nocc = bin(occx).count("1")
    rowc, colc = contraction_orbitals(cx, cw, nocc)
    cx_occ = occ_coeffs(cx, occx)
    cw_occ = occ_coeffs(cw, occw)
    sv, cw_t, cx_t, phase = ortho_svd_rotate(s_ao, cx_occ, cw_occ, tol, null_gauge)
    zeros = [k for k, v in enumerate(sv) if abs(v) <= tol]
    tsp = float(np.prod([v for v in sv if abs(v) > tol])) if len(sv) else 1.0
    m = len(zeros)
    m0, m1 = construct_m(sv, cx_t, cw_t, zeros, tol)
    mao = [m0, m1]
    x0, y0 = construct_xy(rowc, colc, s_ao, m0, True)
    x1, y1 = construct_xy(rowc, colc, s_ao, m1, False)
    cxs, xcs = [], []
    for mi in range(2):
        a, b = build_cx_xc(mao[mi], s_ao, cx, cw, nocc, mi)
        cxs.append(a)
        xcs.append(b)
    jk = [j_coulomb(eri, mao[mi]) - k_exchange(eri, mao[mi]) for mi in range(2)]
    fh = [[cxs[mi].T @ h @ xcs[mj] for mj in range(2)] for mi in range(2)]
    f0h = [einsum_ba_ab(mao[0], h), einsum_ba_ab(mao[1], h)]
    v0 = [0.0, 0.0, 0.0]
    v0[0] = einsum_ba_ab(jk[0], mao[0])
    if m >= 1:
        v0[1] = 2.0 * einsum_ba_ab(jk[0], mao[1])
    if m >= 2:
        v0[2] = einsum_ba_ab(jk[1], mao[1])
    v = [[[cxs[mi].T @ jk[mk] @ xcs[mj] for mk in range(2)] for mj in range(2)] for mi in range(2)]
    jt: Dict[int, np.ndarray] = {}
    for slot, (a, b, c, d) in enumerate(SAME_SPIN_J_BRANCHES):
        if a + b + c + d <= m:
            blk = ao2mo(eri, cxs[a], xcs[b], cxs[c], xcs[d])
            exch = ao2mo(eri, cxs[a], cxs[c], xcs[b], xcs[d])
            jt[slot] = blk - exch.transpose(0, 2, 1, 3)
    return SameSpin(x=[x0, x1], y=[y0, y1], f0h=f0h, fh=fh, v0=v0, v=v, j=jt, tilde_s_prod=tsp,
                    phase=phase, m=m, nmo=nmo, nocc=nocc, singular_values=sv, mao=mao,
                    cx=cxs, xc=xcs)


def diff_spin_build(s_ao, eri, a: SameSpin, b: SameSpin) -> DiffSpin:
    """DiffSpinBuild::new reusing the per-spin M, cx and xc (build.rs:728-926)."""
    ja = [j_coulomb(eri, a.mao[i]) for i in range(2)]
    jb = [j_coulomb(eri, b.mao[i]) for i in range(2)]
    vab0 = [[einsum_ba_ab(ja[i], b.mao[j]) for j in range(2)] for i in range(2)]
    vba0 = [[einsum_ba_ab(jb[j], a.mao[i]) for i in range(2)] for j in range(2)]
    vab = [[[a.cx[ma0].T @ jb[mb0] @ a.xc[mak] for mak in range(2)] for mb0 in range(2)]
           for ma0 in range(2)]
    vba = [[[b.cx[mb0].T @ ja[ma0] @ b.xc[mbk] for mbk in range(2)] for ma0 in range(2)]
           for mb0 in range(2)]
    ii = {}
    for ma0 in range(2):
        for maz in range(2):
            for mb0 in range(2):
                for mby in range(2):
                    if ma0 + maz <= a.m and mb0 + mby <= b.m:
                        ii[(ma0, maz, mb0, mby)] = ao2mo(eri, a.cx[ma0], a.xc[maz], b.cx[mb0],
                                                         b.xc[mby])
    return DiffSpin(vab0=vab0, vba0=vba0, vab=vab, vba=vba, ii=ii)


def build_pair(s_ao, h, eri, ref_x, ref_w, tol: float, null_gauge=None) -> PairBuild:
    """build_wicks_pair (src/noci/wicks.rs:37-81) for bra reference x and ket reference w.

    ``ref_*`` are tuples (C_alpha, occ_alpha_mask, C_beta, occ_beta_mask).
    """
    cxa, oxa, cxb, oxb = ref_x
    cwa, owa, cwb, owb = ref_w
    aa = same_spin_build(s_ao, h, eri, cxa, oxa, cwa, owa, tol, null_gauge)
    bb = same_spin_build(s_ao, h, eri, cxb, oxb, cwb, owb, tol, null_gauge)
    ab = diff_spin_build(s_ao, eri, aa, bb)
    hcol0_a = hcol0_b = None
    if aa.m == 0 and bb.m == 0:
        hcol0_a = aa.fh[0][0] + aa.v[0][0][0] + ab.vab[0][0][0]
        hcol0_b = bb.fh[0][0] + bb.v[0][0][0] + ab.vba[0][0][0]
    return PairBuild(aa=aa, bb=bb, ab=ab, hcol0_a=hcol0_a, hcol0_b=hcol0_b)


def construct_f(s_ao, fock, cx, occx, cw, occw, tol):
    """construct_f_scalar (build.rs:564-617): Fock scalar and column intermediates."""
    nocc = bin(occx).count("1")
    cx_occ = occ_coeffs(cx, occx)
    cw_occ = occ_coeffs(cw, occw)
    sv, cw_t, cx_t, _ = ortho_svd_rotate(s_ao, cx_occ, cw_occ, tol)
    zeros = [k for k, v in enumerate(sv) if abs(v) <= tol]
    m0, m1 = construct_m(sv, cx_t, cw_t, zeros, tol)
    mao = [m0, m1]
    cxs, xcs = [], []
    for mi in range(2):
        a, b = build_cx_xc(mao[mi], s_ao, cx, cw, nocc, mi)
        cxs.append(a)
        xcs.append(b)
    f0 = [einsum_ba_ab(mao[0], fock), einsum_ba_ab(mao[1], fock)]
    ff = [[cxs[mi].T @ fock @ xcs[mj] for mj in range(2)] for mi in range(2)]
    return f0, ff


def zero_count(s_ao, cx, occx, cw, occw, tol) -> int:
    """count_zero_overlap_pairs (build.rs:350-363)."""
    s_occ = occ_coeffs(cx, occx).T @ s_ao @ occ_coeffs(cw, occw)
    sv = np.linalg.svd(s_occ, compute_uv=False)
    return int(np.sum(np.abs(sv) <= tol))


def build_all(s_ao, h, eri, refs, tol: float, null_gauge=None, only=None) -> List[Optional[PairBuild]]:
    """All nref^2 ordered pairs, index = x * nref + w (src/noci/wicks.rs:159-190).  With
    ``only`` (a set of ordered-pair indices) the other entries are None: a checker that
    evaluates a few reference-pair groups of a large system builds just those."""
    out = []
    nref = len(refs)
    for ix, x in enumerate(refs):
        for iw, w in enumerate(refs):
            if only is not None and ix * nref + iw not in only:
                out.append(None)
                continue
            out.append(build_pair(s_ao, h, eri, x, w, tol, null_gauge))
    return out
