"""CPU checks of the oracle's spin-factorised overlap action (oracle/overlap_action.py) and of the
direct-overlap report of the QMC oracle (oracle/qmc.py), the checkers of the GPU overlap action
and of the direct-overlap propagator.

* The factorised S (single-spin determinants of the two parents' strings, identity inside a
  parent, r = record phase x canonical phase) equals the oracle's Wick overlap of every pair,
  with and without zero-overlap reference pairs, with a duplicated determinant and with a
  non-canonical record phase, on the reference's LiH 6-31G fixture and through quadruple
  excitations in one spin; the B-first contraction equals the dense product.
* Direct overlap: the populations start at S c_0 scaled to the initial 1-norm, and a report adds
  S times the report's accumulated change (here a fixed change) instead of the change itself.
"""
import numpy as np
import pytest

from nociwick import synthetic as sy
from oracle.oracle import Oracle
from oracle.overlap_action import OverlapFactorisation, canonical_phase, spin_key
from oracle.qmc import OracleQmc


def _all_pairs_overlap(system, basis):
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    g = np.arange(basis.shape[0])
    pairs = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    _, s = orc.eval_pairs(ob, pairs)
    return s.reshape(basis.shape[0], basis.shape[0]), orc, ob


@pytest.mark.parametrize("zero_pairs", [(), ((0, 1, 1, 0), (1, 2, 0, 2))])
def test_factorised_overlap_equals_wick_overlap(zero_pairs):
    system = sy.make_system(8, 2, 2, 3, 12, seed=7, k_scale=0.3, zero_pairs=list(zero_pairs), enuc=0.5)
    basis = sy.sd_basis(8, 2, 2, 3)
    s, _, _ = _all_pairs_overlap(system, basis)
    f = OverlapFactorisation(system.s, system.refs, 2, 2, basis)
    assert np.abs(f.r - 1.0).max() == 0.0       # sd_basis records carry the canonical phases
    assert np.abs(f.dense() - s).max() < 1e-14
    x = np.random.default_rng(1).standard_normal(basis.shape[0])
    assert np.abs(f.apply(x) - s @ x).max() < 1e-13 * np.abs(x).sum()


def test_factorised_overlap_duplicates_and_phases():
    system = sy.make_system(8, 2, 2, 2, 12, seed=3, k_scale=0.3)
    basis = sy.sd_basis(8, 2, 2, 2)
    basis = np.concatenate([basis, basis[[4, 120]]])
    basis["phase"][9] *= -1.0
    s, _, _ = _all_pairs_overlap(system, basis)
    f = OverlapFactorisation(system.s, system.refs, 2, 2, basis)
    assert f.r[9] == -1.0
    assert abs(s[4, basis.shape[0] - 2] - 1.0) < 1e-15
    assert np.abs(f.dense() - s).max() < 1e-14
    x = np.random.default_rng(4).standard_normal(basis.shape[0])
    assert np.abs(f.apply(x) - s @ x).max() < 1e-13 * np.abs(x).sum()


def test_canonical_phase_is_the_basis_phase():
    basis = sy.sd_basis(9, 3, 2, 1, orders=(1, 2, 3, 4))
    for d in basis[:: max(1, basis.shape[0] // 400)]:
        ph = canonical_phase(3, spin_key(d["rank_a"], d["idx_a"])) * canonical_phase(2, spin_key(d["rank_b"], d["idx_b"]))
        assert ph == d["phase"]


def test_direct_overlap_report_applies_the_overlap():
    system = sy.make_system(8, 2, 2, 2, 12, seed=5, k_scale=0.3)
    basis = sy.sd_basis(8, 2, 2, 2)
    s, orc, ob = _all_pairs_overlap(system, basis)
    f = OverlapFactorisation(system.s, system.refs, 2, 2, basis)
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    c0 = np.zeros(basis.shape[0])
    c0[refs] = [0.7, -0.4]
    q = OracleQmc(orc, ob, c0, refs, dt=0.01, initial_population=200.0, ncycles=1, propagator="direct-overlap",
                  overlap=f.apply, seed=3)
    sc0 = s @ c0
    assert np.abs(q.pop - 200.0 * sc0 / np.abs(sc0).sum()).max() < 1e-12
    fixed = np.random.default_rng(8).standard_normal(basis.shape[0])
    q.cycle_delta = lambda: fixed
    before = q.pop.copy()
    rep = q.report()
    assert np.abs((q.pop - before) - s @ fixed).max() < 1e-12
    assert abs(rep["nw"] - np.abs(q.pop).sum()) < 1e-9
    with pytest.raises(ValueError):
        OracleQmc(orc, ob, c0, refs, dt=0.01, propagator="direct-overlap")


def test_direct_overlap_report_is_unbiased_in_the_oracle():
    """The oracle's direct-overlap report from fixed populations N changes them, on average over
    independent reports, by S (-dt (H - E_s S) N): FRI sampling, uniform spawning, spawn
    rounding and the FRI-compressed update all keep the expectation (z < 6 per determinant)."""
    system = sy.make_system(6, 2, 2, 2, 10, seed=4, k_scale=0.3)
    basis = sy.sd_basis(6, 2, 2, 2)
    n = basis.shape[0]
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    g = np.arange(n)
    pairs = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    h, s = orc.eval_pairs(ob, pairs)
    h, s = h.reshape(n, n), s.reshape(n, n)
    f = OverlapFactorisation(system.s, system.refs, 2, 2, basis)
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    c0 = np.zeros(n)
    c0[refs] = 1.0
    es, dt = -2.0, 0.01
    q = OracleQmc(orc, ob, c0, refs, dt=dt, initial_population=60.0, sampling_cutoff=0.5, spawn_cutoff=0.05,
                  initial_shift=es, ncycles=1, propagator="direct-overlap", overlap=f.apply, seed=11,
                  update_cutoff=0.05, target_population=1e9)
    pop = np.random.default_rng(3).normal(0.0, 1.0, n) * (np.random.default_rng(4).random(n) < 0.4)
    reps = 1500
    d = np.empty((reps, n))
    for k in range(reps):
        q.pop = pop.copy()
        q.report()
        d[k] = q.pop - pop
    expected = s @ (-dt * (h - es * s) @ pop)
    mean, se = d.mean(axis=0), d.std(axis=0, ddof=1) / np.sqrt(reps)
    live = se > 1e-12
    assert np.all(np.abs(mean[~live] - expected[~live]) < 1e-12)
    assert np.max(np.abs(mean[live] - expected[live]) / se[live]) < 6.0


def test_factorised_overlap_on_a_reference_fixture():
    """The reference's direct-overlap LiH 6-31G fixture (its integrals and UHF states rebuilt by
    tests/golden/make_reference_fixtures.py): the factorised S x equals the oracle's Wick S x over
    the 866 singles and doubles of the two references."""
    import reffix
    system, meta = reffix.load("QMC_LiH_6-31G_2_8_TRAJECTORY_DIRECT_OVERLAP")
    basis = sy.sd_basis(system.nmo, system.nocc_a, system.nocc_b, len(system.refs), orders=(1, 2))
    s, _, _ = _all_pairs_overlap(system, basis)
    f = OverlapFactorisation(system.s, system.refs, system.nocc_a, system.nocc_b, basis)
    x = np.random.default_rng(5).standard_normal(basis.shape[0])
    assert basis.shape[0] == 866
    assert np.abs(f.apply(x) - s @ x).max() < 1e-12 * np.abs(x).sum()


def test_factorised_overlap_through_quadruple_excitations():
    """Triple and quadruple excitations in one spin (spin keys of rank 3 and 4, unequal occupied
    counts 4 and 3): 64 rows of the factorised S equal the oracle's Wick overlaps."""
    system = sy.make_system(8, 4, 3, 2, 12, seed=12, k_scale=0.3)
    basis = sy.sd_basis(8, 4, 3, 2, orders=(1, 2, 3, 4))
    assert basis["rank_a"].max() == 4
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    n = basis.shape[0]
    rows = np.random.default_rng(0).choice(n, 64, replace=False)
    pairs = np.stack(np.meshgrid(rows, np.arange(n), indexing="ij"), -1).reshape(-1, 2)
    _, s = orc.eval_pairs(ob, pairs)
    f = OverlapFactorisation(system.s, system.refs, 4, 3, basis)
    assert np.abs(f.dense(rows) - s.reshape(len(rows), n)).max() < 1e-14
