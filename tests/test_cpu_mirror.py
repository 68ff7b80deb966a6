"""CPU checks of the engine's device code (no GPU needed).

noci-rs_b200/csrc/wick_math.cuh holds every per-pair function the CUDA kernels call (record
unpacking, contraction labels, the m = 0 and m > 0 evaluators, the overlap evaluator, the
Jacobi SVD pairing and the layout formulas of the build).  tests/cpu_mirror compiles that same
header with g++; these tests run it against the FP64 oracle, so the kernels' index arithmetic
is checked on the CPU before any GPU time is spent.
"""
import numpy as np
import pytest

import mirror as MR
from nociwick import synthetic as sy
from oracle import wick_build as WB
from oracle.oracle import Oracle

TIGHT = 1e-12


@pytest.fixture(scope="module")
def setup():
    n, o = 8, 3
    system = sy.make_system(n, o, o, 3, 20, seed=1, k_scale=0.3, zero_pairs=[(0, 1, 1, 0), (1, 2, 0, 2)], enuc=0.37)
    orc = Oracle.from_system(system, tol=1e-8)
    basis = sy.sd_basis(n, o, o, 3, orders=(1, 2, 3, 4))
    return n, o, system, orc, basis, orc.oracle_basis(basis)


def test_record_unpacking(setup):
    import ctypes
    n, o, system, orc, basis, ob = setup
    k = basis.shape[0]
    par = np.empty(k, np.int32)
    ra = np.empty(k, np.int32)
    rb = np.empty(k, np.int32)
    ia = np.empty(k, np.uint64)
    ib = np.empty(k, np.uint64)
    ph = np.empty(k)
    MR.lib().mir_unpack(basis.ctypes.data_as(ctypes.c_void_p), k, MR.p(par, ctypes.c_int32),
                        MR.p(ra, ctypes.c_int32), MR.p(rb, ctypes.c_int32), MR.p(ia, ctypes.c_uint64),
                        MR.p(ib, ctypes.c_uint64), MR.p(ph, ctypes.c_double))
    assert np.array_equal(par, basis["parent"]) and np.array_equal(ra, basis["rank_a"])
    assert np.array_equal(rb, basis["rank_b"]) and np.array_equal(ph, basis["phase"])
    assert np.array_equal(ia, basis["idx_a"].copy().view(np.uint64).ravel())
    assert np.array_equal(ib, basis["idx_b"].copy().view(np.uint64).ravel())


def test_labels_register_and_runtime_paths_agree(setup):
    import ctypes
    n, o, system, orc, basis, ob = setup
    rng = np.random.default_rng(0)
    for _ in range(500):
        a, b = (int(v) for v in rng.integers(0, basis.shape[0], 2))
        for spin in (0, 1):
            rc, cc, rr, cr = (np.zeros(8, np.int32) for _ in range(4))
            L = MR.lib().mir_labels(basis.ctypes.data_as(ctypes.c_void_p), a, b, spin, o, n,
                                    MR.p(rc, ctypes.c_int32), MR.p(cc, ctypes.c_int32),
                                    MR.p(rr, ctypes.c_int32), MR.p(cr, ctypes.c_int32))
            assert np.all(rr[:L] >= 0) and np.all(rr[:L] < n) and np.all(cr[:L] >= 0) and np.all(cr[:L] < n)
            if L <= 4:
                assert np.array_equal(rc[:L], rr[:L]) and np.array_equal(cc[:L], cr[:L])


def test_far_same_parent_rule(setup):
    import ctypes
    n, o, system, orc, basis, ob = setup
    rng = np.random.default_rng(1)
    idx = np.nonzero(basis["parent"] == 2)[0]
    for _ in range(400):
        a, b = (int(v) for v in rng.choice(idx, 2))
        diff = bin(int(ob["occ_a"][a][0]) ^ int(ob["occ_a"][b][0])).count("1") + \
            bin(int(ob["occ_b"][a][0]) ^ int(ob["occ_b"][b][0])).count("1")
        assert MR.lib().mir_far_same_parent(basis.ctypes.data_as(ctypes.c_void_p), a, b) == int(diff > 4)


def test_fast_and_generic_evaluators_match_oracle(setup):
    n, o, system, orc, basis, ob = setup
    par = basis["parent"].astype(int)
    rng = np.random.default_rng(2)
    for x in range(3):
        for w in range(3):
            pid = x * 3 + w
            b = orc.builds[pid]
            ia = np.nonzero(par == x)[0]
            iw = np.nonzero(par == w)[0]
            pairs = np.stack([rng.choice(ia, 300), rng.choice(iw, 300)], 1)
            if b.aa.m == 0 and b.bb.m == 0:
                ref = np.array([orc.eval_wick(ob, int(p), int(q)) for p, q in pairs])
                h, s = MR.eval_fast(b, n, o, o, orc.enuc, basis, pairs)
                assert np.max(np.abs(h - ref[:, 0])) < TIGHT and np.max(np.abs(s - ref[:, 1])) < TIGHT
            else:
                for exact in (False, True):
                    ref = np.array([orc.eval_wick(ob, int(p), int(q), exact=exact) for p, q in pairs])
                    for dispatch in (False, True):   # runtime-size path; register twins up to rank 4
                        h, s = MR.eval_gen(orc, pid, n, o, o, basis, pairs, exact=exact, dispatch=dispatch)
                        assert np.max(np.abs(h - ref[:, 0])) < TIGHT and np.max(np.abs(s - ref[:, 1])) < TIGHT
                so = MR.eval_s_gen(orc, pid, n, o, o, basis, pairs)
                ref_s = np.array([orc.eval_overlap(ob, int(p), int(q)) for p, q in pairs])
                assert np.max(np.abs(so - ref_s)) < TIGHT


def test_build_layout_formulas(setup):
    """jas/jstored/ii index formulas of the GPU build, fed the four-quarter transform results
    in the [p][r][q][s] order the build produces."""
    n, o, system, orc, basis, ob = setup
    b = orc.builds[0]
    ss = b.aa
    td = WB.ao2mo(orc.eri, ss.cx[0], ss.xc[0], ss.cx[0], ss.xc[0]).transpose(0, 2, 1, 3).copy()
    te = WB.ao2mo(orc.eri, ss.cx[0], ss.cx[0], ss.xc[0], ss.xc[0]).transpose(0, 2, 1, 3).copy()
    j0 = ss.j[0].transpose(2, 3, 0, 1)
    assert np.max(np.abs(MR.layout(1, td, te) - j0)) < TIGHT
    assert np.max(np.abs(MR.layout(0, td, te) - (j0 - j0.transpose(0, 3, 2, 1)))) < TIGHT
    t4 = WB.ao2mo(orc.eri, b.aa.cx[0], b.aa.xc[0], b.bb.cx[0], b.bb.xc[0]).transpose(0, 2, 1, 3).copy()
    assert np.max(np.abs(MR.layout(2, t4) - b.ab.ii[(0, 0, 0, 0)])) < TIGHT


@pytest.mark.parametrize("nzero", [0, 1, 2, 3])
def test_jacobi_svd_and_canonical_gauge(nzero):
    rng = np.random.default_rng(10 + nzero)
    o = 7
    u0, _ = np.linalg.qr(rng.standard_normal((o, o)))
    v0, _ = np.linalg.qr(rng.standard_normal((o, o)))
    sv = np.sort(rng.random(o))[::-1] + 0.05
    if nzero:
        sv[o - nzero:] = 0.0
    a = u0 @ np.diag(sv) @ v0.T
    u, s, v, phase = MR.svd(a, 1e-8)
    un, sn, vnt = np.linalg.svd(a)
    un, vn, _ = WB.canonical_null_gauge(un, vnt.T, sn, 1e-8)
    assert np.max(np.abs(s - sn)) < 1e-13
    assert np.max(np.abs(u @ np.diag(s) @ v.T - a)) < 1e-13
    assert np.max(np.abs(u.T @ u - np.eye(o))) < 1e-13 and np.max(np.abs(v.T @ v - np.eye(o))) < 1e-13
    assert abs(phase - np.linalg.det(u) * np.linalg.det(v)) < 1e-12
    if nzero >= 1:
        z = slice(o - nzero, o)
        assert np.max(np.abs(u[:, z] - un[:, z])) < 1e-12 and np.max(np.abs(v[:, z] - vn[:, z])) < 1e-12


@pytest.mark.parametrize("cap", [1 << 23, 5000, 26])
def test_sort_keys_group_classes_and_bras(setup, cap):
    """pair_sort_key / sort_key_shift as classify_kernel uses them: fast-pair keys lie in their
    class's range [cls * nbucket, (cls + 1) * nbucket), keys of zero-overlap reference pairs
    after all of them grouped by the full (L_alpha, L_beta), every key below the planned count, the fast-class counters within the
    budget, and with shift 0 one key holds one (bra, ket reference) combination."""
    import ctypes
    n, o, system, orc, basis, ob = setup
    nref = 3
    # the two forced zero-overlap reference pairs of the fixture, both orders
    gen = {(0, 1), (1, 0), (1, 2), (2, 1)}
    fast = [(x, w) for x in range(nref) for w in range(nref) if (x, w) not in gen]
    slow = [(x, w) for x in range(nref) for w in range(nref) if (x, w) in gen]
    order = np.zeros(nref * nref, np.int32)
    for k, (x, w) in enumerate(fast + slow):
        order[x * nref + w] = k
    nfast = len(fast)
    pairs = sy.sample_pairs(basis, 20000, seed=5, distinct_parents=False).astype(np.uint32)
    keys = np.zeros(pairs.shape[0], np.uint32)
    nb, sh = np.zeros(1, np.uint32), np.zeros(1, np.int32)
    nkeys = MR.lib().mir_sort_keys(basis.ctypes.data_as(ctypes.c_void_p), basis.shape[0], nref, MR.p(order, ctypes.c_int32),
                                   nfast, MR.p(pairs, ctypes.c_uint32), pairs.shape[0], cap, MR.p(keys, ctypes.c_uint32),
                                   MR.p(nb, ctypes.c_uint32), MR.p(sh, ctypes.c_int32))
    nb, sh = int(nb[0]), int(sh[0])
    assert 26 * nb <= max(cap, 26) and nkeys == 26 * nb + 81 * len(slow)
    ra, rb = basis["rank_a"].astype(int), basis["rank_b"].astype(int)
    par = basis["parent"].astype(int)
    live = keys != 0xFFFFFFFF
    a, b = pairs[live, 0].astype(int), pairs[live, 1].astype(int)
    k = keys[live].astype(np.int64)
    assert np.all(k < nkeys)
    la, lb = ra[a] + ra[b], rb[a] + rb[b]
    cls = np.where((la <= 4) & (lb <= 4), la * 5 + lb, 25)
    isfast = order[par[a] * nref + par[b]] < nfast
    assert np.all(k[isfast] // nb == cls[isfast])
    assert np.all(k[~isfast] >= 26 * nb)
    assert np.all((k[~isfast] - 26 * nb) % 81 == (la * 9 + lb)[~isfast])
    if sh == 0:
        combo = a.astype(np.int64) * nref + par[b]
        for key in np.unique(k[isfast])[:500]:
            assert len(np.unique(combo[isfast][k[isfast] == key])) == 1
    # far same-parent pairs are exactly the skipped ones
    same = par[pairs[:, 0]] == par[pairs[:, 1]]
    assert np.all(same[~live])


def test_fock_evaluators_match_oracle(setup):
    """(F, S) device code (fast records and the m > 0 distribution sum) against the oracle's
    calculate_m_pair_wicks restatement, all contraction ranks up to 4 + 4."""
    n, o, system, orc, basis, ob = setup
    rng = np.random.default_rng(7)
    a = rng.normal(0.0, 0.3, (n, n))
    fa = 0.5 * (a + a.T) + system.h
    b = rng.normal(0.0, 0.3, (n, n))
    fb = 0.5 * (b + b.T) + system.h
    orc.set_fock(fa, fb)
    par = basis["parent"].astype(int)
    for x in range(3):
        for w in range(3):
            pid = x * 3 + w
            bld = orc.builds[pid]
            ia = np.nonzero(par == x)[0]
            iw = np.nonzero(par == w)[0]
            pairs = np.stack([rng.choice(ia, 300), rng.choice(iw, 300)], 1)
            if bld.aa.m == 0 and bld.bb.m == 0:
                _, f_ref, s_ref = orc.eval_m_pairs(ob, pairs, 0.0)
                f, s = MR.eval_fs_fast(orc, bld, pid, n, o, o, basis, pairs)
                assert np.max(np.abs(f - f_ref)) < TIGHT and np.max(np.abs(s - s_ref)) < TIGHT
            else:
                for exact in (False, True):
                    _, f_ref, s_ref = orc.eval_m_pairs(ob, pairs, 0.0, exact=exact)
                    for dispatch in (False, True):   # runtime-size path; register twins up to rank 4
                        f, s = MR.eval_fs_gen(orc, pid, n, o, o, basis, pairs, exact=exact, dispatch=dispatch)
                        assert np.max(np.abs(f - f_ref)) < TIGHT and np.max(np.abs(s - s_ref)) < TIGHT
