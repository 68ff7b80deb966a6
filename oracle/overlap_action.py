"""CPU restatement of the spin-factorised overlap action y += S x over a determinant basis
(test infrastructure only: tests/ and the CPU legs of bench.py use it, the product library never
does).

The overlap of two determinants is the product of their alpha and beta single-spin overlaps.
Determinants of one parent reference share single-spin components (an alpha string is used by
every determinant with the same alpha excitation), so S restricted to the determinants of a
target parent Q and a source parent P is a sum of Kronecker-structured terms
S_{w Omega} = A^{QP}[a_w][a_Omega] B^{QP}[b_w][b_Omega], and S x is two small contractions per
ordered parent pair instead of a dense product over all determinant pairs.

Reference items restated (paths inside dy-cl/noci-rs):
  * SpinFactorisation::new, parent-local alpha / beta component ids
        src/noci/factorise/mod.rs:56-88
  * build_overlap_factors / build_spin_overlap_factors (A^{QP}, B^{QP} per ordered parent pair)
        src/noci/factorise/overlap.rs:280-397, 1361-1438
  * apply_overlap_sparse with the B-first contraction (U = sum_b B x, then A U)
        src/noci/factorise/overlap.rs:434-498, 1276-1360
  * same-parent blocks: determinants of one parent are orthonormal (overlap.rs:965-1019)
  * apply_overlap_population_changes  src/stochastic/metric.rs:97-232
  * initialise_populations (N_0 = S c_0 scaled to the initial 1-norm)  src/stochastic/init.rs:32-83

The single-spin factor is det(C_Q[:, occ(abar)]^T S_AO C_P[:, occ(a)]) with the occupied columns
in ascending order; the reference evaluates the same number through its per-spin Wick overlap
(xw_overlap_same_f64_batched).  Matrix elements are between canonically ordered determinants, so a
record whose phase differs from the excitation phase of its holes and particles
(excitation_phase_bits, src/basis/excitation.rs:110-146) carries the ratio r = phase * canonical
phase on both sides: S_wick(w, x) = r_w r_x S_canonical(w, x).
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from .basis import excitation_phase_bits


def spin_key(rank: int, idx: np.ndarray) -> Tuple[int, ...]:
    """Holes and particles of one spin (ascending, as the nw_det record stores them)."""
    r = int(rank)
    return tuple(int(v) for v in idx[:r]) + tuple(int(v) for v in idx[4:4 + r])


def spin_occupation(nocc: int, key: Tuple[int, ...]) -> List[int]:
    """Occupied orbitals of a single-spin string, ascending: the parent's first nocc orbitals
    with the holes removed and the particles added."""
    r = len(key) // 2
    holes, parts = set(key[:r]), key[r:]
    return sorted([i for i in range(nocc) if i not in holes] + list(parts))


def canonical_phase(nocc: int, key: Tuple[int, ...]) -> float:
    r = len(key) // 2
    hmask = sum(1 << h for h in key[:r])
    pmask = sum(1 << p for p in key[r:])
    return excitation_phase_bits((1 << nocc) - 1, hmask, pmask)


class OverlapFactorisation:
    """Spin components of a basis of nw_det records and the factor tables of its parent pairs."""

    def __init__(self, s_ao: np.ndarray, refs: Sequence, nocc_a: int, nocc_b: int, basis: np.ndarray):
        self.nref = len(refs)
        self.ndet = basis.shape[0]
        self.parent = basis["parent"].astype(np.int64)
        self.aid = np.zeros(self.ndet, np.int64)
        self.bid = np.zeros(self.ndet, np.int64)
        comps: List[List[Dict[Tuple[int, ...], int]]] = [[{}, {}] for _ in range(self.nref)]
        self.r = np.empty(self.ndet)
        for d in range(self.ndet):
            p = int(self.parent[d])
            ka = spin_key(basis["rank_a"][d], basis["idx_a"][d])
            kb = spin_key(basis["rank_b"][d], basis["idx_b"][d])
            self.aid[d] = comps[p][0].setdefault(ka, len(comps[p][0]))
            self.bid[d] = comps[p][1].setdefault(kb, len(comps[p][1]))
            self.r[d] = float(basis["phase"][d]) * canonical_phase(nocc_a, ka) * canonical_phase(nocc_b, kb)
        self.occ = [[[spin_occupation(no, k) for k in sorted(comps[p][s], key=comps[p][s].get)]
                     for s, no in ((0, nocc_a), (1, nocc_b))] for p in range(self.nref)]
        # MO overlaps O^{QP}_sigma = C_Q^T S C_P and the single-spin factor tables
        cs = [[np.asarray(ref[0]), np.asarray(ref[2])] for ref in refs]
        self.fac: Dict[Tuple[int, int, int], np.ndarray] = {}
        for q in range(self.nref):
            for p in range(self.nref):
                if q == p:
                    continue
                for s in range(2):
                    o = cs[q][s].T @ s_ao @ cs[p][s]
                    tq, tp = self.occ[q][s], self.occ[p][s]
                    f = np.empty((len(tq), len(tp)))
                    for i, oi in enumerate(tq):
                        for j, oj in enumerate(tp):
                            f[i, j] = np.linalg.det(o[np.ix_(oi, oj)]) if oi else 1.0
                    self.fac[(q, p, s)] = f

    def apply(self, x: np.ndarray) -> np.ndarray:
        """S x by the B-first contraction: U[a][bbar] = sum_{Omega in P, a_Omega = a}
        B^{QP}[bbar][b_Omega] x'_Omega, then y_w = r_w sum_a A^{QP}[a_w][a] U[a][b_w]; same-parent
        blocks are the identity on identical spin-component pairs."""
        xs = self.r * np.asarray(x, float)
        y = np.zeros(self.ndet)
        for q in range(self.nref):
            tq = np.nonzero(self.parent == q)[0]
            for p in range(self.nref):
                sp = np.nonzero(self.parent == p)[0]
                if q == p:
                    key = self.aid[sp] * (self.bid.max() + 1) + self.bid[sp]
                    acc: Dict[int, float] = {}
                    for k, d in zip(key, sp):
                        acc[int(k)] = acc.get(int(k), 0.0) + xs[d]
                    tk = self.aid[tq] * (self.bid.max() + 1) + self.bid[tq]
                    y[tq] += np.array([acc.get(int(k), 0.0) for k in tk])
                    continue
                a_tab, b_tab = self.fac[(q, p, 0)], self.fac[(q, p, 1)]
                u = np.zeros((a_tab.shape[1], b_tab.shape[0]))
                for d in sp:
                    u[self.aid[d]] += xs[d] * b_tab[:, self.bid[d]]
                y[tq] += np.einsum("ta,at->t", a_tab[self.aid[tq]], u[:, self.bid[tq]])
        return self.r * y

    def dense(self, rows=None) -> np.ndarray:
        """Rows of the overlap matrix S_wick of the basis from the factor tables (all rows when
        rows is None), filled one (bra parent, ket parent) block at a time."""
        rows = np.arange(self.ndet) if rows is None else np.asarray(rows, np.int64)
        s = np.zeros((rows.shape[0], self.ndet))
        for q in range(self.nref):
            wi = np.nonzero(self.parent[rows] == q)[0]
            w = rows[wi]
            for p in range(self.nref):
                xs = np.nonzero(self.parent == p)[0]
                if q == p:
                    v = ((self.aid[w][:, None] == self.aid[xs][None, :])
                         & (self.bid[w][:, None] == self.bid[xs][None, :])).astype(float)
                else:
                    v = (self.fac[(q, p, 0)][np.ix_(self.aid[w], self.aid[xs])]
                         * self.fac[(q, p, 1)][np.ix_(self.bid[w], self.bid[xs])])
                s[np.ix_(wi, xs)] = v
        return self.r[rows][:, None] * s * self.r[None, :]
