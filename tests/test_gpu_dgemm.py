"""The engine's FP64 tensor-core GEMM (nw_dgemm, csrc/dgemm.cu) against numpy FP64 products:
all four transpose combinations, edge tiles (sizes not multiples of the 64 x 64 x 16 tile),
shared (stride 0) and strided batches, alpha / beta, and the shapes the intermediate build
uses (the n x n^3 first quarter transform, batched n x n products, the M . G contraction).
The build's dense products all run on this kernel, so the whole-pipeline parity tests cover
it too; this file checks it in isolation.

Tolerance: FP64 products accumulate in FP64 on the tensor cores (DMMA), so the result differs
from numpy's only by summation order: |C - C_ref| <= 1e-13 * sum_k |A_ik B_kj|."""
import ctypes

import numpy as np
import pytest

from nociwick import lib as L

pytestmark = pytest.mark.gpu


def _gemm(ta, tb, a, b, m, n, k, alpha=1.0, beta=0.0, c=None, batch=1, sa=0, sb=0, sc=None):
    torch = pytest.importorskip("torch")
    lib = L.load()
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    db = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    if c is None:
        c = np.full((batch * m * n,), np.nan) if beta == 0.0 else np.zeros(batch * m * n)
    dc = torch.from_numpy(np.ascontiguousarray(c)).cuda()
    lda = m if ta else k
    ldb = k if tb else n
    sc = m * n if sc is None else sc
    st = lib.nw_dgemm(int(ta), int(tb), m, n, k, alpha, ctypes.c_void_p(da.data_ptr()), lda, sa,
                      ctypes.c_void_p(db.data_ptr()), ldb, sb, beta, ctypes.c_void_p(dc.data_ptr()), n, sc, batch,
                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, L.load().nw_status_string(st)
    torch.cuda.synchronize()
    return dc.cpu().numpy()


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (7, 5, 3), (64, 64, 16), (65, 130, 17), (30, 900, 30), (200, 33, 129)])
def test_dgemm_matches_numpy(ta, tb, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    a = rng.standard_normal((k, m) if ta else (m, k))
    b = rng.standard_normal((n, k) if tb else (k, n))
    opa = a.T if ta else a
    opb = b.T if tb else b
    got = _gemm(ta, tb, a, b, m, n, k).reshape(m, n)
    ref = opa @ opb
    bound = 1e-13 * (np.abs(opa) @ np.abs(opb)) + 1e-300
    assert np.all(np.abs(got - ref) <= bound)


def test_dgemm_batched_shared_operand_alpha_beta():
    rng = np.random.default_rng(5)
    m, n, k, batch = 40, 40, 40, 7
    a = rng.standard_normal((batch, m, k))
    b = rng.standard_normal((k, n))                    # shared across the batch (stride 0)
    c0 = rng.standard_normal((batch, m, n))
    got = _gemm(False, False, a.ravel(), b, m, n, k, alpha=0.5, beta=-2.0, c=c0.ravel(), batch=batch, sa=m * k,
                sb=0).reshape(batch, m, n)
    ref = 0.5 * (a @ b) - 2.0 * c0
    assert np.max(np.abs(got - ref)) <= 1e-12


def test_dgemm_build_shapes():
    """The four-index transform's first quarter (n x n^3 = A^T E) and the M . G^T contraction."""
    rng = np.random.default_rng(6)
    n = 30
    A = rng.standard_normal((n, n))
    E = rng.standard_normal((n, n ** 3))
    got = _gemm(True, False, A, E, n, n ** 3, n).reshape(n, n ** 3)
    ref = A.T @ E
    assert np.max(np.abs(got - ref)) <= 1e-12
    Mv = rng.standard_normal((12, n * n))
    G = rng.standard_normal((n * n, n * n))
    got = _gemm(False, True, Mv, G, 12, n * n, n * n).reshape(12, n * n)
    assert np.max(np.abs(got - Mv @ G.T)) <= 1e-11


def test_dgemm_rejects_bad_arguments():
    lib = L.load()
    assert lib.nw_dgemm(0, 0, 4, 4, 4, 1.0, None, 4, 0, None, 4, 0, 0.0, None, 4, 0, 1, None) == 1
    torch = pytest.importorskip("torch")
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    assert lib.nw_dgemm(0, 0, -1, 4, 4, 1.0, p, 4, 0, p, 4, 0, 0.0, p, 4, 0, 1, None) == 1
    assert lib.nw_dgemm(0, 0, 4, 4, 0, 1.0, p, 4, 0, p, 4, 0, 0.0, p, 4, 0, 1, None) == 1
