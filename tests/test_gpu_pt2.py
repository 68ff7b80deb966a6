"""GPU NOCI-PT2 solve (nw_pt2_*) against the CPU restatement (oracle/pt2.py) on dense matrices
built by the oracle: the stored M = F - E0 S and its mat-vec, GMRES on the projected operator
with both preconditioners, and E_PT2 = a.M^Omega.a + 2 a.v."""
import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy
from oracle import linalg as LA
from oracle import pt2 as PT
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def snoci_system():
    eps = np.concatenate([np.linspace(-1.0, -0.5, 2), np.linspace(0.2, 2.5, 6)])
    system = sy.make_system(8, 2, 2, 2, 20, seed=3, sigma_h=0.05, sigma_l=0.05, k_scale=0.3, uhf_like=True,
                            orbital_energies=eps)
    basis = sy.sd_basis(8, 2, 2, 2)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    nd = basis.shape[0]
    pairs = np.array([(a, b) for a in range(nd) for b in range(nd)])
    h, s = orc.eval_pairs(ob, pairs)
    h, s = h.reshape(nd, nd), s.reshape(nd, nd)
    orc.set_fock(system.h, system.h)
    _, f, _ = orc.eval_m_pairs(ob, pairs, 0.0)
    f = f.reshape(nd, nd)
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    ec, cc = LA.general_evp(h[np.ix_(refs, refs)], s[np.ix_(refs, refs)], True, 1e-8)
    c = cc[:, 0]
    e0 = float(c @ f[np.ix_(refs, refs)] @ c)
    return system, basis, h, s, f, refs, c, float(ec[0]), e0


def _pieces(h, s, f, refs, c, ecur, e0, cand):
    m = f[np.ix_(cand, cand)] - e0 * s[np.ix_(cand, cand)]
    p = {"e0": e0, "s_a0": s[np.ix_(cand, refs)] @ c, "s_0a": s[np.ix_(refs, cand)].T @ c,
         "f_a0": f[np.ix_(cand, refs)] @ c, "f_0a": f[np.ix_(refs, cand)].T @ c}
    v = h[np.ix_(cand, refs)] @ c - ecur * p["s_a0"]
    return m, p, v


@pytest.mark.parametrize("kind", ["woodbury", "diag"])
def test_pt2_single_parent_candidates(snoci_system, kind):
    """Candidates of one parent (orthonormal among themselves): a unique solution, reached in
    a few iterations by both the GPU and the CPU GMRES."""
    system, basis, h, s, f, refs, c, ecur, e0 = snoci_system
    cand = np.nonzero((basis["parent"] == 0) & ((basis["rank_a"] + basis["rank_b"]) > 0))[0].astype(np.uint32)
    m, p, v = _pieces(h, s, f, refs, c, ecur, e0, cand)
    pre = PT.preconditioner(np.diag(m), p, kind)
    x_ref, res_ref, it_ref, _ = PT.gmres(lambda z: PT.apply_omega(m, p, z), pre, -v, max_iter=100, restart=30,
                                         res_tol=1e-10)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        w.update_fock(system.h, system.h)
        with nociwick.Pt2(w, cand, e0) as pt:
            xv = np.random.default_rng(1).normal(size=cand.shape[0])
            assert np.max(np.abs(pt.apply_m(xv) - m @ xv)) <= 1e-10
            x, info = pt.solve(e0, p["s_a0"], p["s_0a"], p["f_a0"], p["f_0a"], -v, max_iter=100, restart=30,
                               res_tol=1e-10, preconditioner=kind)
    assert info["converged"] and info["residual_rms"] <= 1e-10
    assert abs(info["iterations"] - it_ref) <= 1
    assert np.max(np.abs(x - x_ref)) <= 1e-8


def test_pt2_full_candidate_pool(snoci_system):
    """All non-reference determinants as candidates: the pool is linearly dependent (singular
    projected operator), so GMRES stops on its iteration limit; the GPU mat-vec matches the
    dense product and E_PT2 agrees with the CPU restatement."""
    system, basis, h, s, f, refs, c, ecur, e0 = snoci_system
    cand = np.setdiff1d(np.arange(basis.shape[0]), refs).astype(np.uint32)
    m, p, v = _pieces(h, s, f, refs, c, ecur, e0, cand)
    a = np.array([PT.apply_omega(m, p, e) for e in np.eye(cand.shape[0])]).T
    pre = PT.preconditioner(np.diag(m), p, "woodbury")
    x_ref, _, _, _ = PT.gmres(lambda z: PT.apply_omega(m, p, z), pre, -v, max_iter=120, restart=40, res_tol=1e-10)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        w.update_fock(system.h, system.h)
        with nociwick.Pt2(w, cand, e0) as pt:
            xv = np.random.default_rng(2).normal(size=cand.shape[0])
            y = pt.apply_m(xv)
            x, info = pt.solve(e0, p["s_a0"], p["s_0a"], p["f_a0"], p["f_0a"], -v, max_iter=120, restart=40,
                               res_tol=1e-10)
    assert np.max(np.abs(y - m @ xv)) <= 1e-9 * max(1.0, np.abs(m @ xv).max())
    ept2 = x @ a @ x + 2 * x @ v
    ept2_ref = x_ref @ a @ x_ref + 2 * x_ref @ v
    assert abs(ept2 - ept2_ref) <= 1e-7
    assert np.linalg.norm(a @ x + v) / np.sqrt(cand.shape[0]) <= 1e-5


def test_matrix_free_operator_matches_packed(snoci_system):
    """nw_pt2_create_matrix_free (apply_candidate_m without a cached matrix,
    src/snoci/operators.rs:424-471): M x re-evaluated pair by pair equals the packed product and
    the dense oracle M x over candidates of every parent (most pairs nonorthogonal Wick pairs),
    and GMRES through it reaches the packed solve's solution on the single-parent candidates."""
    system, basis, h, s, f, refs, c, ecur, e0 = snoci_system
    cand = np.nonzero((basis["rank_a"] + basis["rank_b"]) > 0)[0].astype(np.uint32)
    one = np.nonzero((basis["parent"] == 0) & ((basis["rank_a"] + basis["rank_b"]) > 0))[0].astype(np.uint32)
    m, _, _ = _pieces(h, s, f, refs, c, ecur, e0, cand)
    _, p, v = _pieces(h, s, f, refs, c, ecur, e0, one)
    xv = np.random.default_rng(2).normal(size=cand.shape[0])
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        w.update_fock(system.h, system.h)
        with nociwick.Pt2(w, cand, e0) as pk, nociwick.Pt2(w, cand, e0, matrix_free=True) as mf:
            y_pk, y_mf = pk.apply_m(xv), mf.apply_m(xv)
        args = (e0, p["s_a0"], p["s_0a"], p["f_a0"], p["f_0a"], -v)
        kw = dict(max_iter=100, restart=30, res_tol=1e-10, preconditioner="woodbury")
        with nociwick.Pt2(w, one, e0) as pk, nociwick.Pt2(w, one, e0, matrix_free=True) as mf:
            a_pk, info_pk = pk.solve(*args, **kw)
            a_mf, info_mf = mf.solve(*args, **kw)
    scale = np.abs(m) @ np.abs(xv)
    assert np.all(np.abs(y_mf - m @ xv) <= 1e-12 * scale + 1e-14)
    assert np.all(np.abs(y_mf - y_pk) <= 1e-12 * scale + 1e-14)
    assert info_mf["converged"] and info_pk["converged"]
    assert np.max(np.abs(a_mf - a_pk)) <= 1e-8 * max(1.0, np.max(np.abs(a_pk)))


def test_matrix_free_tiles_match_packed_and_dense():
    """Candidates spanning several 256 x 256 tiles (diagonal, off-diagonal and partial edge
    tiles of the matrix-free product): the matrix-free M x equals the packed product and the
    dense F - E0 S from nw_build_fs_matrix."""
    system = sy.make_system(10, 3, 3, 3, 16, seed=8, k_scale=0.3)
    basis = sy.sd_basis(10, 3, 3, 3)
    cand = np.nonzero((basis["rank_a"] + basis["rank_b"]) > 0)[0].astype(np.uint32)
    assert cand.shape[0] > 5 * 256
    e0 = -3.7
    xv = np.random.default_rng(4).normal(size=cand.shape[0])
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        w.update_fock(system.h, system.h)
        f, s = w.build_fs_matrix(cand, cand)
        with nociwick.Pt2(w, cand, e0) as pk, nociwick.Pt2(w, cand, e0, matrix_free=True) as mf:
            y_pk, y_mf = pk.apply_m(xv), mf.apply_m(xv)
    m = f - e0 * s
    scale = np.abs(m) @ np.abs(xv)
    assert np.all(np.abs(y_mf - m @ xv) <= 1e-12 * scale + 1e-14)
    assert np.all(np.abs(y_mf - y_pk) <= 1e-12 * scale + 1e-14)


def test_matrix_free_blocks_match_packed():
    """More candidates than one block of 1024 tiles (13022 candidates: 1128 tiles, two blocks of
    the matrix-free product): matrix-free and packed M x agree."""
    system = sy.make_system(18, 4, 4, 3, 16, seed=12, k_scale=0.3)
    basis = sy.sd_basis(18, 4, 4, 3)
    cand = np.nonzero((basis["rank_a"] + basis["rank_b"]) > 0)[0].astype(np.uint32)
    nb = (cand.shape[0] + 255) // 256
    assert nb * (nb + 1) // 2 > 1024
    e0 = -5.1
    xv = np.random.default_rng(6).normal(size=cand.shape[0])
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        w.update_fock(system.h, system.h)
        with nociwick.Pt2(w, cand, e0) as pk, nociwick.Pt2(w, cand, e0, matrix_free=True) as mf:
            y_pk, y_mf = pk.apply_m(xv), mf.apply_m(xv)
    scale = np.abs(y_pk).max() + np.abs(xv).max()
    assert np.abs(y_mf - y_pk).max() <= 1e-11 * scale, np.abs(y_mf - y_pk).max() / scale
