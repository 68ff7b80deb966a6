"""nw_eval_hs_pairs_noalloc: pair evaluation without device allocation.

Some callers cannot allocate device memory at the point where they evaluate matrix elements:
for example a host program whose own memory pool has already reserved nearly all of HBM, or
a tight loop (QMC spawning, an iterative solver) that cannot absorb cudaMalloc's implicit
device synchronisation or handle an allocation failure halfway through.  The allocation-free
entry point serves them by keeping its per-call scratch in one fixed device array that lives
in the library.

This file is named so that pytest collects it last; it must pass both on its own in a fresh
process and after the rest of the GPU suite.
"""
import ctypes

import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu
ATOL = 1e-10


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    torch = pytest.importorskip("torch")
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 300_000, seed=77, distinct_parents=False).astype(np.uint32)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        stream = torch.cuda.current_stream().cuda_stream
        dp = torch.from_numpy(pairs.view(np.int32)).cuda()
        ref = torch.empty((pairs.shape[0], 2), dtype=torch.float64, device="cuda")
        w.eval_pairs_device(dp.data_ptr(), pairs.shape[0], ref.data_ptr(), stream)
        w.sync(stream)
        expected = ref.cpu().numpy()
        lib = L.load()
        for call in range(2):
            out = torch.full((pairs.shape[0], 2), float("nan"), dtype=torch.float64, device="cuda")
            st = lib.nw_eval_hs_pairs_noalloc(w._ctx, ctypes.c_void_p(dp.data_ptr()), pairs.shape[0],
                                              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
            assert st == 0, (call, lib.nw_last_error(w._ctx))
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got)), call
            assert np.max(np.abs(got - expected)) <= ATOL, call


def test_noalloc_rejects_requests_above_its_limit():
    torch = pytest.importorskip("torch")
    system = sy.make_system(8, 3, 3, 2, 20, seed=4)
    basis = sy.sd_basis(8, 3, 3, 2)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        w.build().set_basis(basis)
        dp = torch.zeros(16, dtype=torch.int32, device="cuda")
        out = torch.zeros(16, dtype=torch.float64, device="cuda")
        with pytest.raises(L.NwError) as e:
            w.eval_pairs_noalloc(dp.data_ptr(), L.NOALLOC_MAX_PAIRS + 1, out.data_ptr())
        assert e.value.status == 4
        # still usable afterwards
        w.eval_pairs_noalloc(dp.data_ptr(), 8, out.data_ptr())
        torch.cuda.synchronize()
        assert np.all(np.isfinite(out.cpu().numpy()))
