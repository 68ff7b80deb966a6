"""The Cholesky-route product of the two-electron tensors on tcgen05 (csrc/tc_gemm.cu) against
the FP64 product: t4[p][r][q][s] = sum_P U[P][pq] V[P][rs].

* NW_TRANSFORM_CHOL_INT8 (Ozaki slices on the int8 tensor cores, exact int32 sums): FP64-faithful,
  |T - T_fp64| <= 1e-13 * sum_P |U||V| (8 slices of 7 bits, rebuilt in FP64);
* NW_TRANSFORM_CHOL_BF16X6 (three BF16 pieces, six products in FP32): FP32-class, bounded by
  the FP32 accumulation over the 6 naux products, |T - T_fp64| <= 1e-4 * sum_P |U||V|
  (about 6 naux 2^-24 for naux = 256);
* NW_TRANSFORM_CHOL_FP64 (the FP64 tensor-core GEMM plus the index swap): to rounding.
Sizes cover partial tiles (n^2 not a multiple of the 128 x 64 tile, naux not a multiple of the
128-byte K tile) and the config-3 shape (n = 64, naux = 256).  Then whole builds: a Cholesky
context built with each transform gives (H, S) within the bar of its precision."""
import ctypes

import numpy as np
import pytest

import nociwick
from nociwick import lib as L
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu


def _product(mode, u, v, naux, n):
    torch = pytest.importorskip("torch")
    lib = L.load()
    du = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    dv = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    dt = torch.full((n ** 4,), float("nan"), dtype=torch.float64, device="cuda")
    st = lib.nw_transform_product(L.TRANSFORMS[mode], ctypes.c_void_p(du.data_ptr()), ctypes.c_void_p(dv.data_ptr()),
                                  naux, n, ctypes.c_void_p(dt.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, (mode, st)
    return dt.cpu().numpy().reshape(n, n, n, n)


@pytest.mark.parametrize("n,naux", [(5, 7), (12, 40), (30, 130), (64, 256)])
@pytest.mark.parametrize("mode,rel", [("chol_fp64", 1e-13), ("chol_int8", 1e-13), ("chol_bf16x6", 1e-4)])
def test_split_product_matches_fp64(n, naux, mode, rel):
    rng = np.random.default_rng(n * 100 + naux)
    # rows of very different magnitude exercise the per-row scaling of the integer slices
    u = rng.standard_normal((naux, n * n)) * np.exp(rng.uniform(-6, 6, n * n))[None, :]
    v = rng.standard_normal((naux, n * n)) * np.exp(rng.uniform(-6, 6, n * n))[None, :]
    got = _product(mode, u, v, naux, n)
    ref = (u.T @ v).reshape(n, n, n, n).transpose(0, 2, 1, 3)        # [p][q][r][s] -> [p][r][q][s]
    bound = (np.abs(u).T @ np.abs(v)).reshape(n, n, n, n).transpose(0, 2, 1, 3)
    assert np.all(np.isfinite(got))
    assert np.all(np.abs(got - ref) <= rel * bound + 1e-300)


@pytest.mark.parametrize("mode,atol", [("chol_fp64", 1e-11), ("chol_int8", 1e-11), ("chol_bf16x6", 1e-4)])
def test_cholesky_builds_match_full_tensor_build(mode, atol):
    system = sy.make_system(16, 3, 3, 3, 48, seed=12, k_scale=0.3, zero_pairs=[(0, 2, 1, 0)], enuc=0.1)
    basis = sy.sd_basis(16, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 40_000, seed=13, distinct_parents=False).astype(np.uint32)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        ref = w.build().set_basis(basis).eval_pairs(pairs)
    with nociwick.WicksShared(system.s, system.h, None, system.enuc, system.refs, chol=system.chol) as w:
        got = w.set_transform(mode).build().set_basis(basis).eval_pairs(pairs)
    err = np.max(np.abs(got - ref))
    assert np.all(np.isfinite(got))
    assert err <= atol * max(1.0, np.max(np.abs(ref))), err


def test_cholesky_transform_needs_factors():
    system = sy.make_system(8, 3, 3, 2, 20, seed=4)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        with pytest.raises(L.NwError) as e:
            w.set_transform("chol_int8")
        assert e.value.status == 5
