"""CPU oracle (test infrastructure only): generalised Slater-Condon and orthogonal shortcuts.

Independent FP64 restatement of the comparison paths that noci-rs keeps beside the Wick
engine.  Only tests/, the smoke check and the CPU-baseline leg of bench.py use this module.

Reference items restated (file:line inside dy-cl/noci-rs):
  * calculate_s_red / build_s_pair          src/noci/naive.rs:41-148
  * calculate_codensity_{p,w}_pair          src/noci/naive.rs:160-203
  * one_electron                            src/noci/naive.rs:291-304
  * two_electron_same / two_electron_diff   src/noci/naive.rs:337-409
  * einsum_ba_abcd_cd                       src/maths/einsum.rs:309-318
  * calculate_hs_pair_naive                 src/noci/hs.rs:372-407
  * calculate_hs_pair_orthogonal            src/noci/hs.rs:167-362
  * calculate_s_pair_orthogonal             src/noci/overlap.rs:57-68
  * antisymmetrise                          src/read.rs:17-20
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .basis import Det, excitation_phase, mask_to_list
from .wick_build import ao2mo, occ_coeffs


def antisymmetrise(eri: np.ndarray) -> np.ndarray:
    """(ab||cd) = (ab|cd) - (ac|bd) (src/read.rs:17-20)."""
    return eri - eri.transpose(0, 2, 1, 3)


@dataclass
class SPair:
    s: float
    s_red: float
    zeros: List[int]
    w: Optional[np.ndarray]
    p_i: Optional[np.ndarray]
    p_j: Optional[np.ndarray]
    phase: float


def build_s_pair(cx_occ, cw_occ, s_ao, tol) -> SPair:
    s_ij = cx_occ.T @ s_ao @ cw_occ
    u, ts, vt = np.linalg.svd(s_ij)
    v = vt.T
    phase = float(np.linalg.det(u) * np.linalg.det(v))
    prod, zeros = 1.0, []
    for i, val in enumerate(ts):
        if abs(val) > tol:
            prod *= val
        else:
            zeros.append(i)
    cx_t = cx_occ @ u
    cw_t = cw_occ @ v
    w = None
    if len(zeros) <= 1:
        scale = np.array([1.0 / val if abs(val) > tol else 0.0 for val in ts])
        w = (cw_t * scale[None, :]) @ cx_t.T
    p_i = p_j = None
    if len(zeros) >= 1 and len(zeros) <= 2:
        p_i = np.outer(cw_t[:, zeros[0]], cx_t[:, zeros[0]])
    if len(zeros) == 2:
        p_j = np.outer(cw_t[:, zeros[1]], cx_t[:, zeros[1]])
    s = phase * float(np.prod(ts)) if not zeros else 0.0
    return SPair(s=s, s_red=prod, zeros=zeros, w=w, p_i=p_i, p_j=p_j, phase=phase)


def einsum_ba_abcd_cd(g, t, h) -> float:
    """sum_{abcd} g[b,a] t[a,b,c,d] h[c,d] (src/maths/einsum.rs:309-318)."""
    return float(np.einsum("ba,abcd,cd->", g, t, h, optimize=True))


def one_electron(o, p: SPair) -> float:
    fac = p.phase * p.s_red
    if len(p.zeros) == 0:
        return fac * float(np.einsum("ba,ab->", p.w, o))
    if len(p.zeros) == 1:
        return fac * float(np.einsum("ba,ab->", p.p_i, o))
    return 0.0


def two_electron_same(asym, p: SPair) -> float:
    fac = p.phase * p.s_red
    nz = len(p.zeros)
    if nz == 0:
        return 0.5 * fac * einsum_ba_abcd_cd(p.w, asym, p.w)
    if nz == 1:
        return fac * einsum_ba_abcd_cd(p.p_i, asym, p.w)
    if nz == 2:
        return fac * einsum_ba_abcd_cd(p.p_i, asym, p.p_j)
    return 0.0


def two_electron_diff(coul, pa: SPair, pb: SPair) -> float:
    fa = pa.phase * pa.s_red
    fb = pb.phase * pb.s_red
    za, zb = len(pa.zeros), len(pb.zeros)
    if za == 0 and zb == 0:
        return fa * fb * einsum_ba_abcd_cd(pa.w, coul, pb.w)
    if za == 0 and zb == 1:
        return fa * fb * einsum_ba_abcd_cd(pa.w, coul, pb.p_i)
    if za == 1 and zb == 0:
        return fa * fb * einsum_ba_abcd_cd(pa.p_i, coul, pb.w)
    if za == 1 and zb == 1:
        return fa * fb * einsum_ba_abcd_cd(pa.p_i, coul, pb.p_i)
    return 0.0


def hs_pair_naive(s_ao, h, eri, asym, enuc, ca_x, oa_x, cb_x, ob_x, ca_w, oa_w, cb_w, ob_w,
                  tol):
    """calculate_hs_pair_naive (src/noci/hs.rs:372-407) on explicit occupations.

    The result is the element between canonically ordered determinants (occupied orbitals in
    ascending index order); no excitation phase is applied.
    """
    pa = build_s_pair(occ_coeffs(ca_x, oa_x), occ_coeffs(ca_w, oa_w), s_ao, tol)
    pb = build_s_pair(occ_coeffs(cb_x, ob_x), occ_coeffs(cb_w, ob_w), s_ao, tol)
    s = pa.s * pb.s
    hnuc = enuc * s if (len(pa.zeros) == 0 and len(pb.zeros) == 0) else 0.0
    h1 = pb.s * one_electron(h, pa) + pa.s * one_electron(h, pb)
    h2 = (pb.s * two_electron_same(asym, pa) + pa.s * two_electron_same(asym, pb)
          + two_electron_diff(eri, pa, pb))
    return hnuc + h1 + h2, s


@dataclass
class MOCache:
    ha: np.ndarray
    hb: np.ndarray
    eri_aa_asym: np.ndarray
    eri_bb_asym: np.ndarray
    eri_ab_coul: np.ndarray
    orthogonal: bool


def build_mo_cache(s_ao, h, eri, asym, ca, cb, tol) -> MOCache:
    """build_mo_cache (src/noci/cache.rs) for one parent reference."""
    def orth_err(c):
        return float(np.max(np.abs(c.T @ s_ao @ c - np.eye(c.shape[1]))))
    return MOCache(ha=ca.T @ h @ ca, hb=cb.T @ h @ cb,
                   eri_aa_asym=ao2mo(asym, ca, ca, ca, ca),
                   eri_bb_asym=ao2mo(asym, cb, cb, cb, cb),
                   eri_ab_coul=ao2mo(eri, ca, ca, cb, cb),
                   orthogonal=(orth_err(ca) < tol and orth_err(cb) < tol))


def hs_pair_orthogonal(enuc, cache: MOCache, x: Det, w: Det):
    """Same-parent Slater-Condon shortcut (src/noci/hs.rs:167-362, src/noci/overlap.rs:57-68)."""
    xa, xb = x.occ_a ^ w.occ_a, x.occ_b ^ w.occ_b
    ra, rb = bin(xa).count("1") // 2, bin(xb).count("1") // 2
    s = x.pha * w.pha * x.phb * w.phb if (x.occ_a == w.occ_a and x.occ_b == w.occ_b) else 0.0
    if ra > 2 or rb > 2 or ra + rb > 2:
        return 0.0, s
    holes_a = mask_to_list(w.occ_a & ~x.occ_a)
    parts_a = mask_to_list(x.occ_a & ~w.occ_a)
    holes_b = mask_to_list(w.occ_b & ~x.occ_b)
    parts_b = mask_to_list(x.occ_b & ~w.occ_b)
    phase = excitation_phase(w.occ_a, holes_a, parts_a) * excitation_phase(w.occ_b, holes_b, parts_b)
    occ_xa = mask_to_list(x.occ_a)
    occ_xb = mask_to_list(x.occ_b)
    c = cache
    if ra == 0 and rb == 0:
        hv = enuc
        hv += sum(c.ha[i, i] for i in occ_xa) + sum(c.hb[i, i] for i in occ_xb)
        hv += 0.5 * sum(c.eri_aa_asym[i, i, j, j] for i in occ_xa for j in occ_xa)
        hv += 0.5 * sum(c.eri_bb_asym[i, i, j, j] for i in occ_xb for j in occ_xb)
        hv += sum(c.eri_ab_coul[i, i, j, j] for i in occ_xa for j in occ_xb)
        return hv, s
    if ra == 1 and rb == 0:
        i, a = holes_a[0], parts_a[0]
        hv = c.ha[a, i]
        hv += sum(c.eri_aa_asym[a, i, j, j] for j in mask_to_list(x.occ_a & w.occ_a))
        hv += sum(c.eri_ab_coul[a, i, j, j] for j in mask_to_list(x.occ_b & w.occ_b))
        return phase * hv, s
    if ra == 0 and rb == 1:
        i, a = holes_b[0], parts_b[0]
        hv = c.hb[a, i]
        hv += sum(c.eri_bb_asym[a, i, j, j] for j in mask_to_list(x.occ_b & w.occ_b))
        hv += sum(c.eri_ab_coul[j, j, i, a] for j in mask_to_list(x.occ_a & w.occ_a))
        return phase * hv, s
    if ra == 2 and rb == 0:
        i, j = holes_a
        a, b = parts_a
        return phase * c.eri_aa_asym[a, i, j, b], s
    if ra == 0 and rb == 2:
        i, j = holes_b
        a, b = parts_b
        return phase * c.eri_bb_asym[a, i, j, b], s
    if ra == 1 and rb == 1:
        i, j = holes_a[0], holes_b[0]
        a, b = parts_a[0], parts_b[0]
        return phase * c.eri_ab_coul[a, i, j, b], s
    return 0.0, s
