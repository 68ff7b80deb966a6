"""GPU parity of the Fock (F, S) path: nw_update_fock + nw_eval_fs_pairs[_device] against the
oracle's calculate_m_pair_wicks restatement (M = F - E0 S with E0 = 0 gives F).

Tolerances as in test_gpu_parity: 1e-10 for well-conditioned workloads, 1e-9 for the stress
systems with nearly singular reference pairs.
"""
import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
ATOL = 1e-10
ATOL_STRESS = 1e-9


def _fock(system, seed):
    rng = np.random.default_rng(seed)
    n = system.h.shape[0]
    out = []
    for _ in range(2):
        a = rng.normal(0.0, 0.3, (n, n))
        out.append(system.h + 0.5 * (a + a.T))
    return out


def _engine(system, tol=1e-8, convention="reference"):
    return nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=tol,
                                convention=convention).build()


@pytest.mark.parametrize("zero_pairs", [[], [(0, 1, 1, 0)], [(0, 1, 0, 2)], [(1, 2, 1, 1)]])
@pytest.mark.parametrize("convention", ["reference", "exact"])
def test_fs_small_all_ranks(zero_pairs, convention):
    system = sy.make_system(8, 3, 3, 3, 20, seed=1, k_scale=0.3, zero_pairs=zero_pairs, enuc=0.37)
    basis = sy.sd_basis(8, 3, 3, 3, orders=(1, 2, 3, 4))
    pairs = sy.sample_pairs(basis, 6000, seed=3, distinct_parents=False)
    fa, fb = _fock(system, 11)
    orc = Oracle.from_system(system, tol=1e-8)
    orc.set_fock(fa, fb)
    _, f_ref, s_ref = orc.eval_m_pairs(orc.oracle_basis(basis), pairs, 0.0, exact=(convention == "exact"))
    with _engine(system, convention=convention) as w:
        w.set_basis(basis)
        w.update_fock(fa, fb)
        fs = w.eval_fs_pairs(pairs)
    assert np.max(np.abs(fs[:, 0] - f_ref)) <= ATOL_STRESS
    assert np.max(np.abs(fs[:, 1] - s_ref)) <= ATOL_STRESS


def test_fs_config2_sample_device_and_refresh():
    """Config-2 stand-in, 20000 pairs: host and device entry points agree bit for bit, match the
    oracle, and a second nw_update_fock with other matrices replaces the tables."""
    import torch
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 20000, seed=77)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    with _engine(system) as w:
        w.set_basis(basis)
        with pytest.raises(nociwick.NwError):
            w.eval_fs_pairs(pairs[:10])        # before any Fock matrices: state error
        for seed in (5, 6):
            fa, fb = _fock(system, seed)
            orc.set_fock(fa, fb)
            _, f_ref, s_ref = orc.eval_m_pairs(ob, pairs, 0.0)
            w.update_fock(fa, fb)
            host = w.eval_fs_pairs(pairs)
            stream = torch.cuda.current_stream().cuda_stream
            dp = torch.from_numpy(pairs.astype(np.uint32).view(np.int32)).cuda()
            out = torch.empty((pairs.shape[0], 2), dtype=torch.float64, device="cuda")
            w.eval_fs_pairs_device(dp.data_ptr(), pairs.shape[0], out.data_ptr(), stream)
            w.sync(stream)
            assert np.array_equal(out.cpu().numpy(), host)
            assert np.max(np.abs(host[:, 0] - f_ref)) <= ATOL
            assert np.max(np.abs(host[:, 1] - s_ref)) <= ATOL
        # the Hamiltonian path is unaffected by the Fock tables
        hs = w.eval_pairs(pairs[:2000])
        h_ref, s_ref2 = orc.eval_pairs(ob, pairs[:2000])
        assert np.max(np.abs(hs[:, 0] - h_ref)) <= ATOL and np.max(np.abs(hs[:, 1] - s_ref2)) <= ATOL
