"""nw_eval_hs_pairs_noalloc: pair evaluation without device allocation.

Some callers cannot allocate device memory at the point where they evaluate matrix elements:
for example a host program whose own memory pool has already reserved nearly all of HBM, or
a tight loop (QMC spawning, an iterative solver) that cannot absorb cudaMalloc's implicit
device synchronisation or handle an allocation failure halfway through.  The allocation-free
entry point serves them by keeping its per-call scratch in one fixed device array that lives
in the library.

Each check uses a fresh context on which the allocation-free call runs first, so the
allocating path's grown buffers cannot stand in for the fixed array, and the device's free
memory is the same before and after two calls.  The second system has reference pairs with
zero-overlap orbitals, so the m > 0 evaluator and its work counter in the fixed array run too.

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


def _noalloc_twice_then_allocating(system, basis, pairs):
    """Two allocation-free calls on a fresh context (free device memory checked around them),
    then the allocating entry point on the same pairs; returns both calls' results and it."""
    torch = pytest.importorskip("torch")
    lib = L.load()
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        stream = torch.cuda.current_stream().cuda_stream
        dp = torch.from_numpy(pairs.view(np.int32)).cuda()
        outs = [torch.full((pairs.shape[0], 2), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
        ref = torch.empty((pairs.shape[0], 2), dtype=torch.float64, device="cuda")
        # first call on the device: looks up the fixed array's address (and loads the kernels)
        st = lib.nw_eval_hs_pairs_noalloc(w._ctx, ctypes.c_void_p(dp.data_ptr()), pairs.shape[0],
                                          ctypes.c_void_p(outs[0].data_ptr()), ctypes.c_void_p(stream))
        assert st == 0, lib.nw_last_error(w._ctx)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for call in (1, 2):
            st = lib.nw_eval_hs_pairs_noalloc(w._ctx, ctypes.c_void_p(dp.data_ptr()), pairs.shape[0],
                                              ctypes.c_void_p(outs[call].data_ptr()), ctypes.c_void_p(stream))
            assert st == 0, (call, lib.nw_last_error(w._ctx))
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, "the allocation-free calls changed the device's free memory"
        w.eval_pairs_device(dp.data_ptr(), pairs.shape[0], ref.data_ptr(), stream)
        w.sync(stream)
        return [o.cpu().numpy() for o in outs[1:]], ref.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 300_000, seed=77, distinct_parents=False).astype(np.uint32)
    got, expected = _noalloc_twice_then_allocating(system, basis, pairs)
    for call, g in enumerate(got):
        assert np.all(np.isfinite(g)), call
        assert np.max(np.abs(g - expected)) <= ATOL, call


def test_noalloc_zero_overlap_system_matches_on_two_calls():
    # two unordered reference pairs with zero-overlap orbitals (m_alpha = 1; m_beta = 2)
    system = sy.make_system(10, 3, 3, 3, 20, seed=5, k_scale=0.3, zero_pairs=[(0, 1, 1, 0), (1, 2, 0, 2)],
                            enuc=0.37)
    basis = sy.sd_basis(10, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 200_000, seed=78, distinct_parents=False).astype(np.uint32)
    par = basis["parent"].astype(np.int64)
    gp = par[pairs[:, 0]] * 3 + par[pairs[:, 1]]
    assert np.isin(gp, [1, 3, 5, 7]).sum() > 10_000  # the m > 0 evaluator has work
    got, expected = _noalloc_twice_then_allocating(system, basis, pairs)
    for call, g in enumerate(got):
        assert np.all(np.isfinite(g)), call
        assert np.max(np.abs(g - expected)) <= ATOL, call


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
