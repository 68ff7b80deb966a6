"""CPU oracle (test infrastructure only): determinant spaces, excitation phases and caches.

This module restates, in plain Python integer arithmetic, how noci-rs builds the excited
determinant basis that the Wick matrix-element path consumes.  Only tests/, the smoke check
and the CPU-baseline leg of bench.py may use it; the product library never does.

Reference files restated here (paths inside dy-cl/noci-rs):
  * src/basis/excitation.rs:110-146  ``excitation_phase_bits``
  * src/basis/excitation.rs:63-100   ``excitation_phase`` (hole/particle lists)
  * src/basis/excitation.rs:276-372  ``generate_excited_basis``
  * src/lib.rs:114-167                ``ExcitationSpin::cache`` / ``ExcitationSpinCache``
  * src/lib.rs:230-266                ``ReducedTwoSpinDetState`` (phase = pha * phb)

Parity status: pinned against reference-produced numbers.  The reference's own energy
fixtures (tests/fixtures/*/expected.json of noci-rs: reference-space NOCI, deterministic
SD-space, NOCI-PT2 and selected-NOCI energies of H2, H4, LiH and F2) are reproduced from
integrals and SCF states rebuilt by tests/golden/make_reference_fixtures.py
(tests/test_reference_fixtures.py); the oracle is also cross-checked against an independent
generalised Slater-Condon path and a brute-force Fock-space evaluation.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from itertools import combinations
from typing import List, Sequence, Tuple


def _below_odd(bits: int, p: int) -> bool:
    """Parity of the number of set bits strictly below orbital ``p``."""
    if p == 0:
        return False
    return (bin(bits & ((1 << p) - 1)).count("1") & 1) != 0


def excitation_phase_bits(occ: int, holes: int, parts: int) -> float:
    """Fermionic sign of removing ``holes`` (highest first) then adding ``parts`` (lowest first).

    Follows src/basis/excitation.rs:110-146: holes are annihilated from the highest index down,
    each contributing the parity of occupied orbitals below it; particles are created from the
    lowest index up, each contributing the parity below it, and every particle except the last
    is added to the running occupation.
    """
    odd = False
    while holes:
        i = holes.bit_length() - 1
        odd ^= _below_odd(occ, i)
        occ &= ~(1 << i)
        holes &= ~(1 << i)
    while parts:
        a = (parts & -parts).bit_length() - 1
        odd ^= _below_odd(occ, a)
        parts &= parts - 1
        if parts:
            occ |= 1 << a
    return -1.0 if odd else 1.0


def excitation_phase(occ: int, holes: Sequence[int], parts: Sequence[int]) -> float:
    """List form used by the same-parent Slater-Condon shortcut (src/basis/excitation.rs:63-100)."""
    odd = False
    for i in reversed(list(holes)):
        odd ^= _below_odd(occ, i)
        occ &= ~(1 << i)
    for k, a in enumerate(parts):
        odd ^= _below_odd(occ, a)
        if k + 1 != len(parts):
            occ |= 1 << a
    return -1.0 if odd else 1.0


def mask_to_list(mask: int) -> List[int]:
    out = []
    while mask:
        low = mask & -mask
        out.append(low.bit_length() - 1)
        mask ^= low
    return out


@dataclass
class SpinExcitation:
    """Hole and particle bit masks of one spin sector (src/lib.rs:114-119)."""

    holes: int = 0
    parts: int = 0

    @property
    def rank(self) -> int:
        return bin(self.holes).count("1")

    def cache(self) -> Tuple[int, List[int]]:
        """``ExcitationSpinCache``: rank plus the first four holes then first four particles."""
        idx = [0] * 8
        h = mask_to_list(self.holes)
        p = mask_to_list(self.parts)
        for i in range(4):
            if i < len(h):
                idx[i] = h[i]
            if i < len(p):
                idx[4 + i] = p[i]
        return self.rank, idx


@dataclass
class Det:
    """One determinant of the excited basis: parent reference, occupations, phases, excitation."""

    parent: int
    occ_a: int
    occ_b: int
    pha: float
    phb: float
    exc_a: SpinExcitation = field(default_factory=SpinExcitation)
    exc_b: SpinExcitation = field(default_factory=SpinExcitation)

    @property
    def phase(self) -> float:
        return self.pha * self.phb


def first_n_mask(n: int) -> int:
    return (1 << n) - 1


def generate_excited_basis(ref_occs: Sequence[Tuple[int, int]], nmo: int, orders: Sequence[int],
                           include_refs: bool = True) -> List[Det]:
    """Enumerate all excitations of the requested total orders on top of each reference.

    Restates src/basis/excitation.rs:276-372 for references that are themselves unexcited
    (parent == reference index): for each order k, every split k = k_alpha + k_beta, and all
    hole/particle combinations in lexicographic order.
    """
    out: List[Det] = []
    for parent, (oa, ob) in enumerate(ref_occs):
        if include_refs:
            out.append(Det(parent, oa, ob, 1.0, 1.0))
        occ_a = [i for i in range(nmo) if (oa >> i) & 1]
        vir_a = [i for i in range(nmo) if not (oa >> i) & 1]
        occ_b = [i for i in range(nmo) if (ob >> i) & 1]
        vir_b = [i for i in range(nmo) if not (ob >> i) & 1]
        for k in sorted(set(orders)):
            for ka in range(k + 1):
                kb = k - ka
                for ha in combinations(occ_a, ka):
                    for pa in combinations(vir_a, ka):
                        for hb in combinations(occ_b, kb):
                            for pb in combinations(vir_b, kb):
                                hma = sum(1 << i for i in ha)
                                pma = sum(1 << i for i in pa)
                                hmb = sum(1 << i for i in hb)
                                pmb = sum(1 << i for i in pb)
                                noa = (oa & ~hma) | pma
                                nob = (ob & ~hmb) | pmb
                                out.append(Det(parent, noa, nob,
                                               excitation_phase_bits(oa, hma, pma),
                                               excitation_phase_bits(ob, hmb, pmb),
                                               SpinExcitation(hma, pma), SpinExcitation(hmb, pmb)))
    return out


def count_excited_basis(nocc_a: int, nocc_b: int, nmo: int, orders: Sequence[int], nref: int,
                        include_refs: bool = True) -> int:
    from math import comb
    va, vb = nmo - nocc_a, nmo - nocc_b
    per = 1 if include_refs else 0
    for k in sorted(set(orders)):
        for ka in range(k + 1):
            kb = k - ka
            per += comb(nocc_a, ka) * comb(va, ka) * comb(nocc_b, kb) * comb(vb, kb)
    return per * nref
