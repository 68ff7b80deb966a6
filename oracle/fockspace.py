"""CPU oracle (test infrastructure only): brute-force Fock-space matrix elements.

An evaluation of <Phi_x|H|Phi_w> and <Phi_x|Phi_w> that shares no algorithm with either
the Wick engine or the generalised Slater-Condon rules: each determinant is expanded in the
full space of determinants over an orthonormal AO basis (coefficients are minors of its
orbital matrix), and the second-quantised Hamiltonian

    H = E_nuc + sum_pq h_pq E_pq + 1/2 sum_pqrs (pq|rs) (E_pq E_rs - delta_qr E_ps)

is applied to the expanded ket.  Only small systems (a few hundred to a few thousand
determinants) are practical; it is used by tests to pin the Wick and naive restatements.

Determinant convention: occupied orbitals in ascending index order, all alpha creators to the
left of all beta creators, which is the canonical ordering the naive path of noci-rs assumes.
"""
from __future__ import annotations

from itertools import combinations
from typing import Dict, List, Tuple

import numpy as np


class FockSpace:
    def __init__(self, nmo: int, nocc_a: int, nocc_b: int):
        self.n = nmo
        self.sa = [sum(1 << i for i in c) for c in combinations(range(nmo), nocc_a)]
        self.sb = [sum(1 << i for i in c) for c in combinations(range(nmo), nocc_b)]
        self.ia = {s: i for i, s in enumerate(self.sa)}
        self.ib = {s: i for i, s in enumerate(self.sb)}
        self.exa = self._single_excitations(self.sa, self.ia)
        self.exb = self._single_excitations(self.sb, self.ib)

    def _single_excitations(self, strings, index) -> Dict[Tuple[int, int], Tuple[np.ndarray, np.ndarray, np.ndarray]]:
        """For each (p, q): arrays (src, dst, sign) with a^+_p a_q |src> = sign |dst>."""
        n = self.n
        out = {}
        for p in range(n):
            for q in range(n):
                src, dst, sgn = [], [], []
                for i, s in enumerate(strings):
                    if not (s >> q) & 1:
                        continue
                    t = s & ~(1 << q)
                    sign = -1 if bin(s & ((1 << q) - 1)).count("1") & 1 else 1
                    if (t >> p) & 1:
                        continue
                    sign *= -1 if bin(t & ((1 << p) - 1)).count("1") & 1 else 1
                    t |= 1 << p
                    src.append(i)
                    dst.append(index[t])
                    sgn.append(sign)
                out[(p, q)] = (np.array(src, np.int64), np.array(dst, np.int64),
                               np.array(sgn, np.float64))
        return out

    def det_vector(self, ca: np.ndarray, occ_a: int, cb: np.ndarray, occ_b: int) -> np.ndarray:
        """Coefficients of the determinant on alpha x beta AO strings (orthonormal AO basis)."""
        oa = [i for i in range(ca.shape[1]) if (occ_a >> i) & 1]
        ob = [i for i in range(cb.shape[1]) if (occ_b >> i) & 1]
        va = np.array([np.linalg.det(ca[[i for i in range(self.n) if (s >> i) & 1]][:, oa])
                       for s in self.sa])
        vb = np.array([np.linalg.det(cb[[i for i in range(self.n) if (s >> i) & 1]][:, ob])
                       for s in self.sb])
        return np.outer(va, vb)

    def _epq(self, p: int, q: int, v: np.ndarray) -> np.ndarray:
        out = np.zeros_like(v)
        src, dst, sgn = self.exa[(p, q)]
        if src.size:
            np.add.at(out, dst, sgn[:, None] * v[src, :])
        src, dst, sgn = self.exb[(p, q)]
        if src.size:
            # beta operators sit to the right of every alpha creator; an alpha string of fixed
            # length contributes (-1)^{N_alpha} twice, which cancels inside E_pq.
            np.add.at(out.T, dst, sgn[:, None] * v.T[src, :])
        return out

    def apply_h(self, h: np.ndarray, eri: np.ndarray, enuc: float, v: np.ndarray) -> np.ndarray:
        n = self.n
        out = enuc * v
        k = h - 0.5 * np.einsum("prrq->pq", eri)
        e = {(r, s): self._epq(r, s, v) for r in range(n) for s in range(n)}
        for p in range(n):
            for q in range(n):
                t = np.zeros_like(v)
                for r in range(n):
                    for s in range(n):
                        g = eri[p, q, r, s]
                        if g != 0.0:
                            t += g * e[(r, s)]
                out = out + k[p, q] * e[(p, q)] + 0.5 * self._epq(p, q, t)
        return out


def hs_element(fs: FockSpace, h, eri, enuc, bra, ket) -> Tuple[float, float]:
    """(<bra|H|ket>, <bra|ket>) for determinants given as (C_a, occ_a, C_b, occ_b)."""
    vx = fs.det_vector(*bra)
    vw = fs.det_vector(*ket)
    hv = fs.apply_h(h, eri, enuc, vw)
    return float(np.sum(vx * hv)), float(np.sum(vx * vw))
