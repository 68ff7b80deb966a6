"""Blocked (out-of-core) evaluation (nw_eval_hs_pairs_blocked): with a slab budget that holds
only part of the reference pairs' intermediates, the request is evaluated block by block and
every element equals the full build's bit for bit (each block computes its reference pairs'
intermediates with the same products), on a system with both pair layouts; afterwards the
context refuses the other evaluation calls until it is rebuilt, and a budget below one
reference pair's intermediates is refused."""
import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu


def test_blocked_evaluation_matches_full_build():
    import torch
    system = sy.make_system(12, 3, 3, 3, 24, seed=5, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.2)
    basis = sy.sd_basis(12, 3, 3, 3, orders=(1, 2, 3))
    pairs = sy.sample_pairs(basis, 100000, seed=8, distinct_parents=False).astype(np.uint32)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build() as w:
        w.set_basis(basis)
        full = w.eval_pairs(pairs)
        m = w.zero_counts()
        slab = w.info()["slab_bytes"]
        assert m.sum() > 0
        stream = torch.cuda.current_stream().cuda_stream
        dp = torch.from_numpy(pairs.view(np.int32)).cuda()
        out = torch.full((pairs.shape[0], 2), float("nan"), dtype=torch.float64, device="cuda")
        nb = w.eval_pairs_blocked(dp.data_ptr(), pairs.shape[0], out.data_ptr(), slab // 3, stream)
        torch.cuda.synchronize()
        assert nb >= 3
        assert np.array_equal(out.cpu().numpy(), full)
        with pytest.raises(L.NwError) as e:
            w.eval_pairs(pairs)
        assert e.value.status == 5
        out.fill_(float("nan"))
        with pytest.raises(L.NwError) as e:
            w.eval_pairs_blocked(dp.data_ptr(), pairs.shape[0], out.data_ptr(), 4096, stream)
        assert e.value.status == 3
        # a budget that holds everything: one block, a full build
        assert w.eval_pairs_blocked(dp.data_ptr(), pairs.shape[0], out.data_ptr(), 0, stream) == 1
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), full)
        assert np.array_equal(w.eval_pairs(pairs), full)
        w.build()
        assert np.array_equal(w.eval_pairs(pairs), full)
