"""The lane-batched restatement of the reference's fixed-rank SIMD path (oracle/wick_binned.cpp,
the CPU baseline of bench.py) against the scalar generic evaluators of the oracle
(preparehamiltonianoverlap.rs:121-362 against :20304-20966): every (L_alpha, L_beta) bin with
L_alpha + L_beta <= 6, partial bins, the generic fallback (ranks > 4 per spin or L_alpha +
L_beta > 6), reference pairs with zero-overlap orbitals and the same-parent shortcuts."""
import numpy as np
import pytest

from nociwick import synthetic as sy
from oracle.oracle import Oracle

ATOL = 1e-11


def _lanes_available():
    import subprocess
    flags = open("/proc/cpuinfo").read() if __import__("os").path.exists("/proc/cpuinfo") else ""
    out = []
    if " avx512f" in flags and " avx512dq" in flags:
        out.append(8)
    if " avx2" in flags and " fma" in flags:
        out.append(4)
    return out


def _pairs_per_bin(basis, per_bin, seed):
    """per_bin random pairs (any parents) for every (L_alpha, L_beta) with L_alpha + L_beta <= 8
    that the basis can form, plus a uniform draw: all 28 bins, partial bins and the fallback."""
    rng = np.random.default_rng(seed)
    ra, rb = basis["rank_a"].astype(int), basis["rank_b"].astype(int)
    groups = {}
    for i, k in enumerate(zip(ra.tolist(), rb.tolist())):
        groups.setdefault(k, []).append(i)
    groups = {k: np.array(v) for k, v in groups.items()}
    out = [sy.sample_pairs(basis, 5000, seed=seed, distinct_parents=False)]
    for la in range(9):
        for lb in range(9 - la):
            combos = [(kx, kw) for kx in groups for kw in groups if kx[0] + kw[0] == la and kx[1] + kw[1] == lb]
            if not combos:
                continue
            for t in range(per_bin):
                kx, kw = combos[rng.integers(len(combos))]
                out.append(np.array([[rng.choice(groups[kx]), rng.choice(groups[kw])]]))
    return np.concatenate(out).astype(np.int64)


@pytest.mark.parametrize("lanes", [8, 4])
def test_binned_matches_scalar_oracle_all_bins(lanes):
    if lanes not in _lanes_available():
        pytest.skip(f"host lacks the {lanes}-lane instruction set")
    # up to quadruples: L = 6 per spin in the bins, L_alpha + L_beta > 6 in the generic fallback;
    # zero-overlap reference pairs take the generic m > 0 path
    system = sy.make_system(10, 4, 4, 3, 20, seed=9, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.4)
    basis = sy.sd_basis(10, 4, 4, 3, orders=(1, 2, 3, 4))
    pairs = _pairs_per_bin(basis, per_bin=60, seed=3)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    h0, s0 = orc.eval_pairs(ob, pairs, nthreads=4)
    h1, s1, used = orc.eval_pairs_binned(ob, pairs, nthreads=4, lanes=lanes)
    assert used == lanes
    la = basis["rank_a"][pairs[:, 0]].astype(int) + basis["rank_a"][pairs[:, 1]]
    lb = basis["rank_b"][pairs[:, 0]].astype(int) + basis["rank_b"][pairs[:, 1]]
    assert len(set(zip(la[la + lb <= 6].tolist(), lb[la + lb <= 6].tolist()))) == 28  # every bin is used
    assert (la + lb > 6).any()                                                        # and the fallback
    assert np.max(np.abs(h1 - h0)) <= ATOL * max(1.0, np.max(np.abs(h0)))
    assert np.max(np.abs(s1 - s0)) <= ATOL


def test_binned_default_width_matches_on_config2_sample():
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 100_000, seed=12345)
    orc = Oracle.from_system(system, tol=1e-8, with_mo_cache=False)
    ob = orc.oracle_basis(basis)
    h0, s0 = orc.eval_pairs(ob, pairs, nthreads=4)
    h1, s1, used = orc.eval_pairs_binned(ob, pairs, nthreads=4)
    assert used in (4, 8)
    assert np.max(np.abs(h1 - h0)) <= 1e-12 * max(1.0, np.max(np.abs(h0)))
    assert np.max(np.abs(s1 - s0)) <= 1e-13
