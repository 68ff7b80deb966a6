"""Pins of the FP64 oracle (CPU only).

The reference (Rust) cannot be built here and its only data for this path are whole-pipeline
energies that need PySCF integrals, so the oracle is pinned by independent evaluations of the
same matrix elements:

* the generalised Slater-Condon path that noci-rs keeps beside the Wick engine (its own
  "wicks.compare" check, src/noci/matrix.rs:224-249 and tests/snoci.rs:352-469, restated);
* a brute-force Fock-space evaluation that shares no algorithm with either;
* the same-parent Slater-Condon shortcut (src/noci/hs.rs:167-362);
* identities: symmetry, overlap of a determinant with itself, SVD-gauge invariance.
"""
import numpy as np
import pytest

from nociwick import synthetic as sy
from oracle import basis as B
from oracle.fockspace import FockSpace, hs_element
from oracle.oracle import Oracle

TIGHT = 1e-12


def _sample(basis, k, seed, same=False):
    rng = np.random.default_rng(seed)
    return rng.integers(0, basis.shape[0], (k, 2))


def test_excitation_phase_hand_cases():
    # |01> -> a+_2 a_0 |01>: a_0 a+_0 a+_1 = a+_1, then a+_2 a+_1 = -a+_1 a+_2
    assert B.excitation_phase_bits(0b11, 0b01, 0b100) == -1.0
    assert B.excitation_phase_bits(0b11, 0b10, 0b100) == 1.0
    # double i,j = 0,1 -> a,b = 2,3 from |0011>: a+_b a+_a a_j a_i gives +1 in this convention
    assert B.excitation_phase_bits(0b11, 0b11, 0b1100) == B.excitation_phase(0b11, [0, 1], [2, 3])
    for occ in (0b0111, 0b1011, 0b11001):
        holes = [i for i in range(5) if (occ >> i) & 1][:2]
        parts = [i for i in range(6) if not (occ >> i) & 1][:2]
        hm = sum(1 << i for i in holes)
        pm = sum(1 << i for i in parts)
        assert B.excitation_phase_bits(occ, hm, pm) == B.excitation_phase(occ, holes, parts)


def test_basis_generation_matches_reference_order():
    """synthetic.sd_basis (vectorised) reproduces the enumeration and phases of
    generate_excited_basis (src/basis/excitation.rs:276-372) restated in oracle.basis."""
    nmo, oa, ob, nref = 7, 2, 3, 2
    recs = sy.sd_basis(nmo, oa, ob, nref, orders=(1, 2))
    dets = B.generate_excited_basis([((1 << oa) - 1, (1 << ob) - 1)] * nref, nmo, (1, 2))
    assert recs.shape[0] == len(dets) == B.count_excited_basis(oa, ob, nmo, (1, 2), nref)
    for r, d in zip(recs, dets):
        assert int(r["parent"]) == d.parent
        ra, ia = d.exc_a.cache()
        rb, ib = d.exc_b.cache()
        assert int(r["rank_a"]) == ra and int(r["rank_b"]) == rb
        assert list(r["idx_a"]) == ia and list(r["idx_b"]) == ib
        assert float(r["phase"]) == d.phase


def test_config2_determinant_count():
    assert sy.sd_basis(30, 3, 3, 3).shape[0] == 26490


@pytest.fixture(scope="module")
def small_m0():
    system = sy.make_system(6, 2, 2, 3, 12, seed=1, k_scale=0.3, enuc=0.41)
    basis = sy.sd_basis(6, 2, 2, 3, orders=(1, 2, 3, 4))
    orc = Oracle.from_system(system, tol=1e-8)
    return system, basis, orc, orc.oracle_basis(basis), FockSpace(6, 2, 2)


def test_wick_m0_equals_naive_and_fockspace(small_m0):
    system, basis, orc, ob, fs = small_m0
    for a, b in _sample(basis, 120, 3):
        hw, sw = orc.eval_wick(ob, int(a), int(b))
        hn, sn = orc.naive(ob, int(a), int(b))
        assert abs(hw - hn) < TIGHT and abs(sw - sn) < TIGHT
    for a, b in _sample(basis, 25, 4):
        hw, sw = orc.eval_wick(ob, int(a), int(b))
        hf, sf = hs_element(fs, orc.h, orc.eri, orc.enuc, orc.det_orbitals(ob, int(a)), orc.det_orbitals(ob, int(b)))
        assert abs(hw - hf) < TIGHT and abs(sw - sf) < TIGHT


def test_symmetry_and_self_overlap(small_m0):
    system, basis, orc, ob, fs = small_m0
    for a, b in _sample(basis, 200, 5):
        h1, s1 = orc.eval_wick(ob, int(a), int(b))
        h2, s2 = orc.eval_wick(ob, int(b), int(a))
        assert abs(h1 - h2) < TIGHT and abs(s1 - s2) < TIGHT
    for a in range(0, basis.shape[0], 37):
        _, s = orc.eval_wick(ob, a, a)
        assert abs(s - 1.0) < 1e-12


def test_same_parent_shortcut_equals_wick(small_m0):
    """Same-parent pairs: the orthogonal Slater-Condon shortcut (with the far-pair zero rule)
    and the Wick path on the (x, x) intermediates agree."""
    system, basis, orc, ob, fs = small_m0
    par = basis["parent"]
    rng = np.random.default_rng(6)
    idx = np.nonzero(par == 1)[0]
    pairs = np.stack([rng.choice(idx, 400), rng.choice(idx, 400)], axis=1)
    h, s = orc.eval_pairs(ob, pairs)
    for k, (a, b) in enumerate(pairs):
        hw, sw = orc.eval_wick(ob, int(a), int(b))
        assert abs(h[k] - hw) < TIGHT and abs(s[k] - sw) < TIGHT


def test_overlap_only_matches_hs_path(small_m0):
    system, basis, orc, ob, fs = small_m0
    for a, b in _sample(basis, 200, 7):
        assert abs(orc.eval_overlap(ob, int(a), int(b)) - orc.eval_wick(ob, int(a), int(b))[1]) < TIGHT


ZERO_PATTERNS = [[(0, 1, 1, 0)], [(0, 1, 0, 1)], [(0, 1, 1, 1)], [(0, 1, 2, 0)], [(0, 1, 0, 2)], [(0, 1, 2, 1)]]


@pytest.mark.parametrize("zp", ZERO_PATTERNS)
def test_exact_convention_equals_fockspace(zp):
    """Zero-overlap reference pairs: the exact convention reproduces brute force, and does not
    depend on how the SVD rotates the zero-singular-value subspace."""
    system = sy.make_system(6, 2, 2, 2, 12, seed=1, k_scale=0.3, zero_pairs=zp, enuc=0.37)
    basis = sy.sd_basis(6, 2, 2, 2)
    orc = Oracle.from_system(system, tol=1e-8)
    orc_g = Oracle.from_system(system, tol=1e-8, null_gauge=np.random.default_rng(3))
    ob = orc.oracle_basis(basis)
    fs = FockSpace(6, 2, 2)
    per = basis.shape[0] // 2
    rng = np.random.default_rng(0)
    assert orc.builds[1].aa.m == zp[0][2] and orc.builds[1].bb.m == zp[0][3]
    for _ in range(15):
        a, b = int(rng.integers(0, per)), int(per + rng.integers(0, per))
        hf, sf = hs_element(fs, orc.h, orc.eri, orc.enuc, orc.det_orbitals(ob, a), orc.det_orbitals(ob, b))
        he, se = orc.eval_wick(ob, a, b, exact=True)
        hg, sg = orc_g.eval_wick(ob, a, b, exact=True)
        assert abs(he - hf) < TIGHT and abs(se - sf) < TIGHT
        assert abs(hg - hf) < TIGHT
        # the naive generalised Slater-Condon path agrees as well
        hn, sn = orc.naive(ob, a, b)
        assert abs(hn - hf) < TIGHT and abs(sn - sf) < TIGHT


@pytest.mark.parametrize("zp", [[(0, 1, 1, 0)], [(0, 1, 0, 1)], [(0, 1, 2, 0)], [(0, 1, 0, 2)], [(0, 1, 2, 1)]])
def test_reference_convention_is_reproducible_after_gauge_fix(zp):
    """The reference evaluator depends on the SVD null-space gauge (for one zero, on the
    relative sign of the paired null vectors); the canonical gauge makes the restatement
    independent of the SVD routine."""
    system = sy.make_system(8, 3, 3, 2, 12, seed=1, k_scale=0.3, zero_pairs=zp)
    basis = sy.sd_basis(8, 3, 3, 2)
    orc = Oracle.from_system(system, tol=1e-8)
    orc_g = Oracle.from_system(system, tol=1e-8, null_gauge=np.random.default_rng(9))
    ob = orc.oracle_basis(basis)
    per = basis.shape[0] // 2
    rng = np.random.default_rng(1)
    for _ in range(200):
        a, b = int(rng.integers(0, per)), int(per + rng.integers(0, per))
        assert abs(orc.eval_wick(ob, a, b)[0] - orc_g.eval_wick(ob, a, b)[0]) < 1e-12


def test_reference_convention_double_counts_mixed_scalar_term():
    """Characterises the reference's m > 0 quirk on reference determinants (L = 0, m_alpha = 1):
    xw_hamiltonian_overlap_gen_prepared applies v0[1] (which already holds the (0,1) and (1,0)
    assignments, build.rs:229-232) to both distributions, so H_ref - H_exact = pref * v0[1] / 2."""
    system = sy.make_system(6, 2, 2, 2, 12, seed=1, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.0)
    basis = sy.sd_basis(6, 2, 2, 2)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    per = basis.shape[0] // 2
    h_ref, s_ref = orc.eval_wick(ob, 0, per)
    h_ex, s_ex = orc.eval_wick(ob, 0, per, exact=True)
    b = orc.builds[1]
    pref = b.aa.phase * b.aa.tilde_s_prod * b.bb.phase * b.bb.tilde_s_prod
    assert s_ref == 0.0 and s_ex == 0.0
    assert abs((h_ref - h_ex) - pref * b.aa.v0[1] / 2.0) < TIGHT
    fs = FockSpace(6, 2, 2)
    hf, _ = hs_element(fs, orc.h, orc.eri, 0.0, orc.det_orbitals(ob, 0), orc.det_orbitals(ob, per))
    assert abs(h_ex - hf) < TIGHT and abs(h_ref - hf) > 1e-6


def test_reference_and_exact_agree_without_zero_overlap(small_m0):
    system, basis, orc, ob, fs = small_m0
    for a, b in _sample(basis, 100, 8):
        assert orc.eval_wick(ob, int(a), int(b)) == orc.eval_wick(ob, int(a), int(b), exact=True)


@pytest.mark.parametrize("zp", [[], [(0, 1, 1, 0)], [(0, 1, 0, 2)]])
def test_fock_m_operator_matches_naive(zp):
    """SNOCI operator M = F - E0 S (calculate_m_pair_wicks, src/noci/m.rs:160-197) from the Fock
    intermediates of update_wicks_fock equals the generalised Slater-Condon M
    (calculate_m_pair_naive) for m = 0 and, in the exact convention, for m > 0."""
    system = sy.make_system(8, 3, 3, 3, 20, seed=1, k_scale=0.3, zero_pairs=zp)
    orc = Oracle.from_system(system, tol=1e-8)
    rng = np.random.default_rng(1)
    a = rng.standard_normal((8, 8))
    b = rng.standard_normal((8, 8))
    fa, fb = a + a.T, b + b.T
    orc.set_fock(fa, fb)
    basis = sy.sd_basis(8, 3, 3, 3)
    ob = orc.oracle_basis(basis)
    pairs = sy.sample_pairs(basis, 300, seed=2, distinct_parents=False)
    m, f, s = orc.eval_m_pairs(ob, pairs, -1.7, exact=True)
    for k, (x, w) in enumerate(pairs):
        mn, fn, sn = orc.naive_m(ob, int(x), int(w), fa, fb, -1.7)
        assert abs(m[k] - mn) < 1e-12 and abs(s[k] - sn) < 1e-12
    if not zp:
        mr, _, _ = orc.eval_m_pairs(ob, pairs, -1.7, exact=False)
        assert np.array_equal(mr, m)
