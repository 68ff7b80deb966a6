"""GPU dense NOCI matrices (nw_build_hs_matrix / nw_build_fs_matrix) and the FP64 generalised
eigensolve (nw_general_evp) against the oracle.

* Plain reference NOCI, H2/cc-pVDZ stand-in (n = 10, 1 + 1 electrons, three references): the
  3 x 3 S and H agree with the oracle to 1e-12 Eh, and so do the NOCI energies.
* NOCISD-like space on n = 8: matrix blocks (symmetric and rectangular) against per-pair
  oracle values, and the projected eigenproblem against the oracle's general_evp restatement
  (eigenvalues; eigenvectors through S-orthonormality and the residual, which do not depend on
  the sign or degenerate-subspace choices of the eigensolver).
"""
import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy
from oracle import linalg as LA
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _engine(system, tol=1e-8):
    return nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=tol).build()


def _oracle_matrix(orc, ob, left, right):
    pairs = np.array([(a, b) for a in left for b in right], dtype=np.int64)
    h, s = orc.eval_pairs(ob, pairs)
    return h.reshape(len(left), len(right)), s.reshape(len(left), len(right))


def test_reference_noci_h2_standin():
    system = sy.config1_system()
    basis = sy.sd_basis(10, 1, 1, 3, orders=(0,), include_refs=False)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    idx = np.arange(3)
    h_ref, s_ref = _oracle_matrix(orc, ob, idx, idx)
    with _engine(system) as w:
        w.set_basis(basis)
        h, s = w.build_hs_matrix()
        assert np.max(np.abs(h - h_ref)) <= 1e-12 and np.max(np.abs(s - s_ref)) <= 1e-12
        e, c = w.general_evp(h, s, project=True, tol=1e-8)
    e_ref, c_ref = LA.general_evp(h_ref, s_ref, True, 1e-8)
    assert e.shape == e_ref.shape
    assert np.max(np.abs(e - e_ref)) <= 1e-12
    # same eigenvectors up to sign (non-degenerate 3 x 3 problem)
    sign = np.sign(np.sum(c * c_ref, axis=0))
    assert np.max(np.abs(c * sign - c_ref)) <= 1e-10


def test_sd_space_matrices_and_projected_evp():
    system = sy.make_system(8, 3, 3, 3, 20, seed=4, k_scale=0.3, enuc=0.21)
    basis = sy.sd_basis(8, 3, 3, 3)
    nd = basis.shape[0]
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    rng = np.random.default_rng(1)
    with _engine(system) as w:
        w.set_basis(basis)
        h, s = w.build_hs_matrix()
        assert np.array_equal(h, h.T) and np.array_equal(s, s.T)
        # symmetric blocks: every upper-triangle element against the oracle on a sample of rows
        rows = np.sort(rng.choice(nd, 24, replace=False))
        hr, sr = _oracle_matrix(orc, ob, rows, np.arange(nd))
        for k, i in enumerate(rows):
            j = np.arange(i, nd)
            assert np.max(np.abs(h[i, j] - hr[k, j])) <= 1e-10
            assert np.max(np.abs(s[i, j] - sr[k, j])) <= 1e-10
        # rectangular block
        left = rng.choice(nd, 40, replace=False).astype(np.uint32)
        right = rng.choice(nd, 70, replace=False).astype(np.uint32)
        hb, sb = w.build_hs_matrix(left, right, symmetric=False)
        hbr, sbr = _oracle_matrix(orc, ob, left, right)
        assert np.max(np.abs(hb - hbr)) <= 1e-10 and np.max(np.abs(sb - sbr)) <= 1e-10
        e, c = w.general_evp(h, s, project=True, tol=1e-8)
    e_ref, _ = LA.general_evp(h, s, True, 1e-8)
    assert e.shape == e_ref.shape
    assert np.max(np.abs(e - e_ref)) <= 1e-8
    assert np.max(np.abs(c.T @ s @ c - np.eye(c.shape[1]))) <= 1e-8
    assert np.max(np.abs(h @ c - s @ c * e[None, :])) <= 1e-7


def test_unprojected_evp_and_fock_matrix():
    system = sy.make_system(8, 3, 3, 2, 20, seed=6, k_scale=0.2)
    basis = sy.sd_basis(8, 3, 3, 2, orders=(1,))
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    nd = basis.shape[0]
    fa = system.h + 0.05 * np.eye(8)
    fb = system.h - 0.03 * np.eye(8)
    orc.set_fock(fa, fb)
    with _engine(system) as w:
        w.set_basis(basis)
        h, s = w.build_hs_matrix()
        e, c = w.general_evp(h, s, project=False)
        w.update_fock(fa, fb)
        f, s2 = w.build_fs_matrix()
    e_ref, _ = LA.general_evp(h, s, False, 1e-8)
    assert c.shape == (nd, nd)
    assert np.max(np.abs(e - e_ref)) <= 1e-8
    assert np.max(np.abs(h @ c - s @ c * e[None, :])) <= 1e-7
    pairs = np.array([(a, b) for a in range(nd) for b in range(nd)], dtype=np.int64)
    _, f_ref, s_ref = orc.eval_m_pairs(ob, pairs, 0.0)
    assert np.max(np.abs(f - f_ref.reshape(nd, nd))) <= 1e-10
    assert np.max(np.abs(s2 - s_ref.reshape(nd, nd))) <= 1e-10
    assert np.max(np.abs(s2 - s)) <= 1e-13
