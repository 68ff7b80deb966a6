"""Seeded synthetic nonorthogonal-determinant systems and determinant-pair workloads.

The molecular workloads of noci-rs need PySCF integrals, which this image does not have, so
every workload here is a seeded synthetic stand-in with the same dimensions:

* an orthonormal AO basis (S = I);
* a symmetric one-electron matrix h with N(0, sigma_h) entries;
* two-electron integrals (mu nu|lam sig) = sum_P L^P_{mu nu} L^P_{lam sig} from naux symmetric
  Cholesky-like vectors with N(0, sigma_L) entries, so the tensor has 8-fold symmetry and is
  positive semidefinite;
* reference orbital sets C = Q exp(K) from a random orthonormal Q and antisymmetric K, drawn
  separately for alpha and beta; the occupied orbitals are the first nocc columns;
* optional zero-overlap reference pairs: occupied orbitals of one reference are rotated into
  the virtual space of another so that 1 or 2 paired singular values of their occupied
  overlap vanish (the m > 0 path of the Wick engine).

The determinant basis is every single and double excitation of each reference (and the
reference itself), enumerated in the order of noci-rs ``generate_excited_basis``
(src/basis/excitation.rs:276-372), with the fermionic phases of ``excitation_phase_bits``
(src/basis/excitation.rs:110-146).  Determinants are packed into the 32-byte ``nw_det``
record declared in include/nociwick.h.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import combinations
from typing import List, Optional, Sequence, Tuple

import numpy as np

# nw_det: uint32 parent; uint8 rank_a; uint8 idx_a[8] (holes 0-3, particles 4-7);
# uint8 rank_b; uint8 idx_b[8]; uint8 pad[2]; double phase  (32 bytes).
NW_DET_DTYPE = np.dtype({
    "names": ["parent", "rank_a", "idx_a", "rank_b", "idx_b", "pad", "phase"],
    "formats": ["<u4", "u1", ("u1", (8,)), "u1", ("u1", (8,)), ("u1", (2,)), "<f8"],
    "offsets": [0, 4, 5, 13, 14, 22, 24],
    "itemsize": 32,
})


@dataclass
class System:
    """AO data and reference orbitals of one synthetic system."""

    nmo: int
    nocc_a: int
    nocc_b: int
    s: np.ndarray
    h: np.ndarray
    eri: np.ndarray                     # (mu nu|lam sig), shape (n, n, n, n)
    chol: np.ndarray                    # L^P_{mu nu}, shape (naux, n, n)
    enuc: float
    refs: List[Tuple[np.ndarray, int, np.ndarray, int]]   # (C_a, occ_a, C_b, occ_b)
    zero_pairs: List[Tuple[int, int, int, int]] = field(default_factory=list)  # (x, w, m_a, m_b)

    @property
    def nref(self) -> int:
        return len(self.refs)


def _expm_antisym(k: np.ndarray) -> np.ndarray:
    """exp(K) of a real antisymmetric matrix through the eigendecomposition of K^2 = -K^T K."""
    w, v = np.linalg.eigh(k @ k)          # K^2 symmetric negative semidefinite
    theta = np.sqrt(np.clip(-w, 0.0, None))
    c = np.cos(theta)
    s = np.where(theta > 1e-14, np.sin(theta) / np.where(theta > 1e-14, theta, 1.0), 1.0)
    # exp(K) = cos(sqrt(-K^2)) + K sinc(sqrt(-K^2)), both functions of K^2 commute with K.
    cosm = (v * c[None, :]) @ v.T
    sincm = (v * s[None, :]) @ v.T
    return cosm + k @ sincm


def _random_orthonormal(rng: np.random.Generator, n: int) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))[None, :]


def _rotation(rng: np.random.Generator, n: int, scale: float) -> np.ndarray:
    a = rng.normal(0.0, scale, (n, n))
    return _expm_antisym(np.triu(a, 1) - np.triu(a, 1).T)


def _force_zero_overlap(rng, cx: np.ndarray, cw: np.ndarray, nocc: int, k: int) -> np.ndarray:
    """Return a new orthonormal C_w whose first k occupied orbitals are orthogonal to x's occupied
    space, so the occupied overlap C_x,occ^T C_w,occ has k zero singular values."""
    n = cw.shape[0]
    proj = np.eye(n) - cx[:, :nocc] @ cx[:, :nocc].T
    cols = []
    for _ in range(k):
        v = proj @ rng.standard_normal(n)
        for c in cols:
            v -= c * (c @ v)
        cols.append(v / np.linalg.norm(v))
    mat = np.hstack([np.stack(cols, axis=1), cw[:, k:]])
    q, r = np.linalg.qr(mat)
    return q * np.sign(np.diag(r))[None, :]


def make_system(nmo: int, nocc_a: int, nocc_b: int, nref: int, naux: int, seed: int,
                sigma_h: float = 0.5, sigma_l: float = 0.1, k_scale: float = 0.3,
                zero_pairs: Sequence[Tuple[int, int, int, int]] = (), enuc: float = 0.0,
                uhf_like: bool = False, orbital_energies: Optional[np.ndarray] = None) -> System:
    """Build a seeded synthetic system.

    ``zero_pairs`` lists (x, w, k_alpha, k_beta): reference w is modified so that the ordered
    pairs (x, w) and (w, x) have k_alpha / k_beta zero-overlap orbital pairs.  With
    ``uhf_like`` the references are an RHF-like set (C_a = C_b = Q) followed by alternating
    spin-polarised sets (C_a = Q exp(K), C_b = Q exp(-K), then alpha and beta swapped), as in
    the RHF + UHF(+,-) + UHF(-,+) reference spaces of noci-rs inputs.  ``orbital_energies``
    adds Q diag(eps) Q^T to h, so the base orbitals carry molecule-like orbital energies
    (occupied first) and the excited determinants lie above the references.
    """
    rng = np.random.default_rng(seed)
    n = nmo
    a = rng.normal(0.0, sigma_h, (n, n))
    h = 0.5 * (a + a.T)
    b = rng.normal(0.0, sigma_l, (naux, n, n))
    chol = 0.5 * (b + b.transpose(0, 2, 1))
    eri = np.tensordot(chol, chol, axes=(0, 0))       # (mu nu|lam sig)
    s = np.eye(n)
    q = _random_orthonormal(rng, n)
    if orbital_energies is not None:
        h = h + q @ np.diag(np.asarray(orbital_energies, float)) @ q.T
    refs = []
    if uhf_like:
        refs.append((q.copy(), (1 << nocc_a) - 1, q.copy(), (1 << nocc_b) - 1))
        k = 1
        while len(refs) < nref:
            r = _rotation(rng, n, k_scale)
            ca, cb = q @ r, q @ r.T
            refs.append((ca, (1 << nocc_a) - 1, cb, (1 << nocc_b) - 1))
            if len(refs) < nref:
                refs.append((cb.copy(), (1 << nocc_a) - 1, ca.copy(), (1 << nocc_b) - 1))
            k += 1
    else:
        for _ in range(nref):
            ca = q @ _rotation(rng, n, k_scale)
            cb = q @ _rotation(rng, n, k_scale)
            refs.append((ca, (1 << nocc_a) - 1, cb, (1 << nocc_b) - 1))
    for (x, w, ka, kb) in zero_pairs:
        cxa, oa, cxb, ob = refs[x]
        cwa, _, cwb, _ = refs[w]
        if ka:
            cwa = _force_zero_overlap(rng, cxa, cwa, nocc_a, ka)
        if kb:
            cwb = _force_zero_overlap(rng, cxb, cwb, nocc_b, kb)
        refs[w] = (cwa, refs[w][1], cwb, refs[w][3])
    return System(nmo=n, nocc_a=nocc_a, nocc_b=nocc_b, s=s, h=h, eri=np.ascontiguousarray(eri),
                  chol=np.ascontiguousarray(chol), enuc=enuc, refs=refs,
                  zero_pairs=list(zero_pairs))


def _phase_bits(occ: int, holes: Sequence[int], parts: Sequence[int]) -> float:
    """excitation_phase_bits (src/basis/excitation.rs:110-146) for ascending index lists."""
    odd = 0
    for i in sorted(holes, reverse=True):
        odd ^= bin(occ & ((1 << i) - 1)).count("1") & 1
        occ &= ~(1 << i)
    for k, p in enumerate(sorted(parts)):
        odd ^= bin(occ & ((1 << p) - 1)).count("1") & 1
        if k + 1 != len(parts):
            occ |= 1 << p
    return -1.0 if odd else 1.0


def _spin_excitations(nocc: int, nmo: int, k: int):
    """All (holes, parts, phase) of rank k from an aufbau occupation, lexicographic order."""
    occ = (1 << nocc) - 1
    out = []
    for hs in combinations(range(nocc), k):
        for ps in combinations(range(nocc, nmo), k):
            out.append((hs, ps, _phase_bits(occ, hs, ps)))
    return out


def sd_basis(nmo: int, nocc_a: int, nocc_b: int, nref: int, orders: Sequence[int] = (1, 2),
             include_refs: bool = True) -> np.ndarray:
    """Every excitation of the given total orders on each aufbau reference, as nw_det records.

    Ordering follows generate_excited_basis: per reference, the reference itself, then for
    each order k, each split k = k_alpha + k_beta with k_alpha ascending, then alpha holes,
    alpha particles, beta holes, beta particles in lexicographic order.
    """
    per_spin_a = {k: _spin_excitations(nocc_a, nmo, k) for k in range(0, max(orders) + 1)}
    per_spin_b = {k: _spin_excitations(nocc_b, nmo, k) for k in range(0, max(orders) + 1)}
    recs: List[np.ndarray] = []

    def pack(ex_a, ex_b):
        na, nb = len(ex_a), len(ex_b)
        out = np.zeros(na * nb, dtype=NW_DET_DTYPE)
        ra = len(ex_a[0][0]) if na else 0
        rb = len(ex_b[0][0]) if nb else 0
        idx_a = np.zeros((na, 8), np.uint8)
        ph_a = np.empty(na)
        for i, (hs, ps, ph) in enumerate(ex_a):
            idx_a[i, :len(hs)] = hs
            idx_a[i, 4:4 + len(ps)] = ps
            ph_a[i] = ph
        idx_b = np.zeros((nb, 8), np.uint8)
        ph_b = np.empty(nb)
        for i, (hs, ps, ph) in enumerate(ex_b):
            idx_b[i, :len(hs)] = hs
            idx_b[i, 4:4 + len(ps)] = ps
            ph_b[i] = ph
        out["rank_a"] = ra
        out["rank_b"] = rb
        out["idx_a"] = np.repeat(idx_a, nb, axis=0)
        out["idx_b"] = np.tile(idx_b, (na, 1))
        out["phase"] = np.repeat(ph_a, nb) * np.tile(ph_b, na)
        return out

    for parent in range(nref):
        parts = []
        if include_refs:
            parts.append(pack([((), (), 1.0)], [((), (), 1.0)]))
        for k in sorted(set(orders)):
            for ka in range(k + 1):
                kb = k - ka
                ex_a, ex_b = per_spin_a[ka], per_spin_b[kb]
                if ex_a and ex_b:
                    parts.append(pack(ex_a, ex_b))
        blk = np.concatenate(parts)
        blk["parent"] = parent
        recs.append(blk)
    return np.concatenate(recs)


def det_ranks(basis: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    return basis["rank_a"].astype(np.int64), basis["rank_b"].astype(np.int64)


def sample_pairs(basis: np.ndarray, npairs: int, seed: int, distinct_parents: bool = True,
                 canonical: bool = True) -> np.ndarray:
    """Uniform ordered determinant pairs (a, b); with ``distinct_parents`` b's parent differs.

    Returns an int64 array of shape (npairs, 2).  With ``canonical`` each pair is ordered
    a <= b, the convention of calculate_hs_pairs_wicks_batched (src/noci/hs.rs:60-78).
    """
    rng = np.random.default_rng(seed)
    ndet = basis.shape[0]
    parent = basis["parent"].astype(np.int64)
    a = rng.integers(0, ndet, npairs)
    if distinct_parents:
        nref = int(parent.max()) + 1
        per = ndet // nref
        assert per * nref == ndet, "equal-size reference blocks expected"
        b = rng.integers(0, ndet - per, npairs)
        pa = parent[a]
        b = np.where(b >= pa * per, b + per, b)
    else:
        b = rng.integers(0, ndet, npairs)
    pairs = np.stack([a, b], axis=1)
    if canonical:
        pairs.sort(axis=1)
    return np.ascontiguousarray(pairs.astype(np.int64))


def sample_pairs_by_rank(basis: np.ndarray, npairs: int, seed: int,
                         max_total: int = 4) -> np.ndarray:
    """Pairs whose contraction rank L_alpha + L_beta is uniform over 0..max_total.

    Each determinant has rank <= 2, so a total t is split as t = r_x + r_w with
    r_x, r_w in {0, 1, 2}, uniform over the admissible splits; the determinants are then drawn
    uniformly among those of that rank, from different parents.
    """
    rng = np.random.default_rng(seed)
    parent = basis["parent"].astype(np.int64)
    rank = (basis["rank_a"].astype(np.int64) + basis["rank_b"].astype(np.int64))
    by_rank = {r: np.nonzero(rank == r)[0] for r in range(3)}
    totals = rng.integers(0, max_total + 1, npairs)
    out = np.empty((npairs, 2), np.int64)
    for t in range(max_total + 1):
        sel = np.nonzero(totals == t)[0]
        splits = [(rx, t - rx) for rx in range(3) if 0 <= t - rx <= 2]
        pick = rng.integers(0, len(splits), sel.size)
        for si, (rx, rw) in enumerate(splits):
            s2 = sel[pick == si]
            if s2.size == 0:
                continue
            xa = by_rank[rx][rng.integers(0, by_rank[rx].size, s2.size)]
            wb = by_rank[rw][rng.integers(0, by_rank[rw].size, s2.size)]
            # redraw same-parent pairs
            bad = parent[xa] == parent[wb]
            while bad.any():
                wb[bad] = by_rank[rw][rng.integers(0, by_rank[rw].size, int(bad.sum()))]
                bad = parent[xa] == parent[wb]
            out[s2, 0] = xa
            out[s2, 1] = wb
    return out


def config1_system(seed: int = 1) -> System:
    """Linear-H2/cc-pVDZ stand-in (n = 10, 1 + 1 electrons, RHF-like + two spin-polarised
    references, E_nuc of H2 at 1.5 Angstrom); the basis is the three references."""
    return make_system(10, 1, 1, 3, 40, seed, k_scale=0.75, uhf_like=True, enuc=0.35275)


def config2_system(seed: int = 2) -> System:
    """Stand-in for linear H6/cc-pVDZ: n = 30, 3 alpha + 3 beta electrons, RHF + 2 UHF refs."""
    return make_system(30, 3, 3, 3, 120, seed, k_scale=0.08, uhf_like=True, enuc=0.0)


def config4_system(seed: int = 4) -> System:
    """Linear-H8/cc-pVDZ NOCISD(3)-QMC stand-in dimensions: n = 40, 4 + 4 electrons, an RHF-like
    and two spin-polarised references (all singles and doubles: 85755 determinants).  Unlike the
    unstructured stand-ins it carries orbital energies (occupied -1.0..-0.5, virtual 0.2..2.5 Eh)
    and weak random couplings, so excited determinants lie above the references and the
    off-diagonal row sums of H and S stay molecule-like (sum_w |S_xw| < 1)."""
    eps = np.concatenate([np.linspace(-1.0, -0.5, 4), np.linspace(0.2, 2.5, 36)])
    return make_system(40, 4, 4, 3, 160, seed, sigma_h=0.02, sigma_l=0.02, k_scale=0.3, uhf_like=True,
                       enuc=0.0, orbital_energies=eps)


def config5_system(seed: int = 5) -> System:
    """F2/cc-pVDZ selected-NOCI + NOCI-PT2 stand-in dimensions: n = 28, 9 + 9 electrons, an
    RHF-like and two spin-polarised references; all singles and doubles of the three
    references give 125688 determinants (125685 PT2 candidates).  Orbital energies as in the
    QMC stand-in (occupied -1.5..-0.5, virtual 0.2..2.5 Eh) with weak random couplings."""
    eps = np.concatenate([np.linspace(-1.5, -0.5, 9), np.linspace(0.2, 2.5, 19)])
    return make_system(28, 9, 9, 3, 112, seed, sigma_h=0.02, sigma_l=0.02, k_scale=0.3, uhf_like=True,
                       enuc=0.0, orbital_energies=eps)


def reference_fock(system: System, r: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """AO Fock matrices of reference r's determinant: F_s = h + J[D_a + D_b] - K[D_s] with
    D_s = C_s[:, :nocc_s] C_s[:, :nocc_s]^T (orthonormal AO basis)."""
    ca, _, cb, _ = system.refs[r]
    da = ca[:, :system.nocc_a] @ ca[:, :system.nocc_a].T
    db = cb[:, :system.nocc_b] @ cb[:, :system.nocc_b].T
    j = np.einsum("pqrs,rs->pq", system.eri, da + db)
    ka = np.einsum("prqs,rs->pq", system.eri, da)
    kb = np.einsum("prqs,rs->pq", system.eri, db)
    return system.h + j - ka, system.h + j - kb


def config3_system(seed: int = 3, nmo: int = 64, nref: int = 8) -> System:
    """Synthetic stress system: n = 64, 6 + 6 electrons, naux = 256, 8 references, zero-overlap
    pairs forced in 3 unordered reference pairs (6 of 64 ordered pairs)."""
    zp = [(0, 1, 1, 0), (2, 3, 0, 2), (4, 5, 1, 1)] if nref >= 6 else [(0, 1, 1, 0)]
    return make_system(nmo, 6, 6, nref, 256, seed, k_scale=0.3, zero_pairs=zp)
