"""The per-reference-pair and host-buffer entry points of the C ABI against the resident-basis
path and the FP64 oracle:

* nw_eval_hs_batched (xw_hamiltonian_overlap_prepared_batched,
  src/nonorthogonalwicks/eval/preparehamiltonianoverlap.rs:121-362): requests grouped by
  ordered reference pair with caller-held excitation caches give the same (H, S) as the same
  pairs through nw_eval_hs_pairs, on blocks with and without zero-overlap orbitals, and on
  diagonal blocks (far same-parent requests exactly 0); invalid caches are refused;
* nw_eval_s_pairs (host-buffer overlap) against the device entry and the oracle;
* nw_ctx_create_cholesky: a context from the Cholesky factors of the integrals gives the
  elements of the full-tensor context within FP64 rounding.
"""
import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick import synthetic as sy
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
ATOL = 1e-10


def _system():
    return sy.make_system(10, 3, 3, 3, 20, seed=2, k_scale=0.3, zero_pairs=[(0, 1, 1, 0), (1, 2, 0, 2)], enuc=0.37)


def test_batched_blocks_match_resident_pairs_and_oracle():
    system = _system()
    basis = sy.sd_basis(10, 3, 3, 3)
    # not canonicalised (a <= b would keep the bra's parent <= the ket's): every block occurs
    pairs = sy.sample_pairs(basis, 40_000, seed=8, distinct_parents=False, canonical=False).astype(np.int64)
    orc = Oracle.from_system(system, tol=1e-8)
    h_ref, s_ref = orc.eval_pairs(orc.oracle_basis(basis), pairs)
    caches = L.exc_caches(basis)
    par = basis["parent"].astype(np.int64)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        w.build().set_basis(basis)
        hs_res = w.eval_pairs(pairs)
        got = np.full((pairs.shape[0], 2), np.nan)
        m = w.zero_counts()
        blocks_m = set()
        for lp in range(3):
            for gp in range(3):
                sel = np.nonzero((par[pairs[:, 0]] == lp) & (par[pairs[:, 1]] == gp))[0]
                if sel.size == 0:
                    continue
                a, b = pairs[sel, 0], pairs[sel, 1]
                ph = basis["phase"][a] * basis["phase"][b]
                got[sel] = w.eval_batched(lp, gp, caches[a], caches[b], ph)
                if m[lp, gp].sum() > 0:
                    blocks_m.add((lp, gp))
    assert len(blocks_m) == 4
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - hs_res)) <= 1e-12
    assert np.max(np.abs(got[:, 0] - h_ref)) <= ATOL and np.max(np.abs(got[:, 1] - s_ref)) <= ATOL
    # far same-parent requests of diagonal blocks are exactly zero, as calculate_hs_pairs_wicks_batched has them
    same = par[pairs[:, 0]] == par[pairs[:, 1]]
    far = same & (h_ref == 0.0) & (s_ref == 0.0)
    assert far.any() and np.all(got[far] == 0.0)


def test_batched_overlap_and_fock_blocks_match_resident_pairs():
    """nw_eval_s_batched and nw_eval_fs_batched on the same per-reference-pair blocks equal the
    resident-basis overlap and (F, S) calls, every block (zero-overlap ones included)."""
    system = _system()
    basis = sy.sd_basis(10, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 20_000, seed=9, distinct_parents=False, canonical=False).astype(np.int64)
    caches = L.exc_caches(basis)
    par = basis["parent"].astype(np.int64)
    rng = np.random.default_rng(3)
    fa = rng.standard_normal((10, 10))
    fa = fa + fa.T
    fb = fa + 0.2 * np.eye(10)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        w.build().set_basis(basis)
        w.update_fock(fa, fb)
        s_res = w.eval_overlap(pairs)
        fs_res = w.eval_fs_pairs(pairs)
        s_got = np.full(pairs.shape[0], np.nan)
        fs_got = np.full((pairs.shape[0], 2), np.nan)
        for lp in range(3):
            for gp in range(3):
                sel = np.nonzero((par[pairs[:, 0]] == lp) & (par[pairs[:, 1]] == gp))[0]
                if sel.size == 0:
                    continue
                a, b = pairs[sel, 0], pairs[sel, 1]
                ph = basis["phase"][a] * basis["phase"][b]
                s_got[sel] = w.eval_batched(lp, gp, caches[a], caches[b], ph, kind="s")
                fs_got[sel] = w.eval_batched(lp, gp, caches[a], caches[b], ph, kind="fs")
    assert np.all(np.isfinite(s_got)) and np.all(np.isfinite(fs_got))
    assert np.max(np.abs(s_got - s_res)) <= 1e-13
    assert np.max(np.abs(fs_got - fs_res)) <= 1e-12


def test_batched_rejects_invalid_caches():
    system = _system()
    basis = sy.sd_basis(10, 3, 3, 3)
    caches = L.exc_caches(basis[:8])
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        w.build()
        bad = caches.copy()
        bad["rank_a"][3] = 5                                    # rank above 4
        with pytest.raises(L.NwError):
            w.eval_batched(0, 2, bad, caches, np.ones(8))
        bad = caches.copy()
        bad["rank_b"][2] = 1
        bad["idx_b"][2, 0] = 3                                   # hole not occupied (nocc = 3)
        with pytest.raises(L.NwError):
            w.eval_batched(0, 2, caches, bad, np.ones(8))
        with pytest.raises(L.NwError):
            w.eval_batched(0, 3, caches, caches, np.ones(8))    # reference index out of range
        out = w.eval_batched(0, 2, caches, caches, np.ones(8))  # still usable
        assert np.all(np.isfinite(out))


def test_host_overlap_entry():
    torch = pytest.importorskip("torch")
    system = _system()
    basis = sy.sd_basis(10, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 20_000, seed=9, distinct_parents=False).astype(np.uint32)
    orc = Oracle.from_system(system, tol=1e-8)
    _, s_ref = orc.eval_pairs(orc.oracle_basis(basis), pairs.astype(np.int64))
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        w.build().set_basis(basis)
        s_host = w.eval_overlap(pairs)
        dp = torch.from_numpy(pairs.view(np.int32)).cuda()
        ds = torch.empty(pairs.shape[0], dtype=torch.float64, device="cuda")
        w.eval_overlap_device(dp.data_ptr(), pairs.shape[0], ds.data_ptr(), torch.cuda.current_stream().cuda_stream)
        w.sync(torch.cuda.current_stream().cuda_stream)
        assert np.array_equal(s_host, ds.cpu().numpy())
        assert np.max(np.abs(s_host - s_ref)) <= ATOL
        with pytest.raises(L.NwError):
            w.eval_overlap(np.array([[0, basis.shape[0]]], np.uint32))


def test_cholesky_context_matches_full_tensor_context():
    system = sy.make_system(12, 3, 3, 3, 40, seed=6, k_scale=0.3, zero_pairs=[(0, 2, 1, 1)], enuc=0.2)
    basis = sy.sd_basis(12, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 30_000, seed=10, distinct_parents=False).astype(np.uint32)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        hs_full = w.build().set_basis(basis).eval_pairs(pairs)
    with nociwick.WicksShared(system.s, system.h, None, system.enuc, system.refs, chol=system.chol) as w:
        hs_chol = w.build().set_basis(basis).eval_pairs(pairs)
    assert np.max(np.abs(hs_chol - hs_full)) <= 1e-11 * max(1.0, np.max(np.abs(hs_full)))
