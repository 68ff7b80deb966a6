"""Host logic of the selected-NOCI driver (nociwick/snoci.py), on the CPU:

* candidate generation from the references equals the engine's SD basis enumeration
  (generate_excited_basis, src/basis/excitation.rs:276-372): order, orbitals and phases;
* excitations of an already excited state are re-expressed relative to its parent reference
  (total holes / particles, excitation_phase_bits) and labelled by the generating state;
* the candidate pool update removes selected labels and skips labels already present
  (src/snoci/candidate.rs);
* the NOCI density (src/noci/naive.rs:231) without the excitation phases contracts with any
  one-body operator F to c^T F c of the oracle's Fock matrix elements (generalised
  Slater-Condon, src/noci/m.rs); with them (the reference's weighting) it is the density of the
  phase-weighted coefficients; the Fock builder follows src/scf/kernels.rs:46;
* select_candidates keeps the highest scores above sigma in decreasing order.
"""
import numpy as np
import pytest

from nociwick import snoci as sn
from nociwick import synthetic as sy
from oracle.oracle import Oracle


@pytest.mark.parametrize("dims", [(8, 2, 2, 2), (10, 3, 2, 3)])
def test_reference_candidates_match_sd_basis(dims):
    nmo, na, nb, nref = dims
    st, lab = sn.reference_states(nref, na, nb)
    cand, labels = sn.generate_excited_basis(st, lab, nmo)
    d = sn.to_nw_dets(cand)
    ref = sy.sd_basis(nmo, na, nb, nref, include_refs=False)
    for f in ("parent", "rank_a", "idx_a", "rank_b", "idx_b", "phase"):
        assert np.array_equal(d[f], ref[f]), f
    assert len(set(labels)) == len(labels)


def test_excitations_of_an_excited_state():
    nmo, na, nb = 8, 3, 2
    st, lab = sn.reference_states(2, na, nb)
    cand, labels = sn.generate_excited_basis(st, lab, nmo)
    x = int(np.nonzero((cand["parent"] == 1) & (cand["ha"] == 0b011) & (cand["hb"] == 0))[0][0])
    base, base_label = cand[x:x + 1], [labels[x]]
    kids, kid_labels = sn.generate_excited_basis(base, base_label, nmo)
    nocc_a, nvir_a = na, nmo - na
    nocc_b, nvir_b = nb, nmo - nb
    from math import comb
    n_expected = sum(comb(nocc_a, ka) * comb(nvir_a, ka) * comb(nocc_b, k - ka) * comb(nvir_b, k - ka)
                     for k in (1, 2) for ka in range(k + 1))
    assert kids.shape[0] == n_expected
    ref_a, ref_b = (1 << na) - 1, (1 << nb) - 1
    for k in kids:
        assert int(k["parent"]) == 1
        assert int(k["ha"]) == ref_a & ~int(k["oa"]) and int(k["pa"]) == int(k["oa"]) & ~ref_a
        assert int(k["hb"]) == ref_b & ~int(k["ob"]) and int(k["pb"]) == int(k["ob"]) & ~ref_b
        pa = sy._phase_bits(ref_a, sn._bits(int(k["ha"])), sn._bits(int(k["pa"])))
        pb = sy._phase_bits(ref_b, sn._bits(int(k["hb"])), sn._bits(int(k["pb"])))
        assert k["phase"] == pa * pb
    assert all(kl[0] == base_label[0] for kl in kid_labels)
    # one child returns to the parent reference itself (total excitation empty)
    back = [i for i, k in enumerate(kids) if int(k["oa"]) == ref_a and int(k["ob"]) == ref_b]
    assert len(back) == 1 and kid_labels[back[0]][1:] == (0, 0, 0, 0)


def test_pool_update_semantics():
    nmo = 8
    st, lab = sn.reference_states(2, 2, 2)
    pool = sn.CandidatePool(st, lab, nmo)
    n0 = pool.states.shape[0]
    pick = [3, 10]
    new_states, new_labels = pool.states[pick], [pool.labels[i] for i in pick]
    sel_labels = lab + new_labels
    pool.update(sel_labels, new_states, new_labels)
    assert not (set(new_labels) & set(pool.labels))
    assert len(set(pool.labels)) == len(pool.labels)
    kids, kid_labels = sn.generate_excited_basis(new_states, new_labels, nmo)
    assert pool.states.shape[0] == n0 - 2 + len(kid_labels)


def test_rank_limit_is_enforced():
    st = np.zeros(1, sn.STATE_DTYPE)
    st["ha"] = 0b11111
    st["pa"] = 0b11111 << 5
    with pytest.raises(ValueError):
        sn.to_nw_dets(st)


def test_select_candidates():
    s = np.array([0.1, 0.5, 1e-9, 0.5, 0.3])
    assert list(sn.select_candidates(s, 1e-6, 3)) == [1, 3, 4]
    assert list(sn.select_candidates(s, 0.4, 10)) == [1, 3]


def test_density_contracts_to_fock_elements():
    eps = np.concatenate([np.linspace(-1.0, -0.5, 2), np.linspace(0.2, 2.5, 6)])
    system = sy.make_system(8, 2, 2, 2, 20, seed=3, sigma_h=0.05, sigma_l=0.05, k_scale=0.3, uhf_like=True,
                            orbital_energies=eps)
    st, lab = sn.reference_states(2, 2, 2)
    cand, labels = sn.generate_excited_basis(st, lab, 8)
    states = np.concatenate([st, cand[[0, 5, 40, 220, 300]]])
    basis = sn.to_nw_dets(states)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    rng = np.random.default_rng(4)
    c = rng.normal(size=states.shape[0])
    a = rng.normal(size=(8, 8))
    fa, fb = a + a.T, np.diag(np.arange(8.0)) + 0.1 * (a + a.T)
    orc.set_fock(fa, fb)
    n = states.shape[0]
    pairs = np.array([(i, j) for i in range(n) for j in range(n)])
    _, f, s = orc.eval_m_pairs(ob, pairs, 0.0)
    # the density of sum_i c_i |Phi_i> in the engine's (canonical) determinant convention
    da, db = sn.noci_density(system, states, c, 1e-8, phases=False)
    assert abs(np.sum(fa * da) + np.sum(fb * db) - c @ f.reshape(n, n) @ c) < 1e-10
    assert np.any(states["phase"] < 0)
    # the reference's convention weights each pair by the excitation phases as well
    pa_, pb_ = sn.noci_density(system, states, c, 1e-8, phases=True)
    qa, qb = sn.noci_density(system, states, c * states["phase"], 1e-8, phases=False)
    assert np.allclose(pa_, qa, atol=1e-13) and np.allclose(pb_, qb, atol=1e-13)
    # a single determinant: the projector onto its occupied orbitals
    da1, db1 = sn.noci_density(system, st[:1], np.ones(1), 1e-8)
    ca, _, cb, _ = system.refs[0]
    assert np.allclose(da1, ca[:, :2] @ ca[:, :2].T, atol=1e-12)
    assert np.allclose(db1, cb[:, :2] @ cb[:, :2].T, atol=1e-12)
    ga, gb = sn.fock(system.h, system.eri, da1, db1)
    ra, rb = sy.reference_fock(system, 0)
    assert np.allclose(ga, ra, atol=1e-12) and np.allclose(gb, rb, atol=1e-12)
