"""The CPU restatement of the NOCI-QMC propagation (oracle/qmc.py) estimates what it must:
one cycle's change is an unbiased estimate of -dt [(H - E_s S) N - E^I N], checked against the
dense H and S of the oracle over many independent cycles (per determinant, 6 standard errors).
The GPU propagation is checked the same way in test_gpu_qmc.py."""
import numpy as np
import pytest

from nociwick import synthetic as sy
from oracle.oracle import Oracle
from oracle.qmc import OracleQmc


@pytest.mark.parametrize("prop,ident", [("unshifted", 0.0), ("shifted", 1.0)])
def test_oracle_cycle_is_unbiased(prop, ident):
    system = sy.make_system(6, 2, 2, 2, 16, seed=3, k_scale=0.3)
    basis = sy.sd_basis(6, 2, 2, 2)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    nd = basis.shape[0]
    pairs = np.array([(a, b) for a in range(nd) for b in range(nd)])
    h, s = orc.eval_pairs(ob, pairs)
    h, s = h.reshape(nd, nd), s.reshape(nd, nd)
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    c0 = np.zeros(nd)
    c0[refs] = 1.0
    es, dt = -1.1, 0.004
    q = OracleQmc(orc, ob, c0, refs, dt=dt, sampling_cutoff=0.5, spawn_cutoff=0.05, initial_shift=es,
                  propagator=prop, seed=5)
    rng = np.random.default_rng(2)
    q.pop = rng.normal(0.0, 2.0, nd) * (rng.random(nd) < 0.4)
    k = 1500
    d = np.array([q.cycle_delta() for _ in range(k)])
    expected = -dt * ((h - es * s) @ q.pop - ident * es * q.pop)
    mean, se = d.mean(axis=0), d.std(axis=0, ddof=1) / np.sqrt(k)
    live = se > 0
    assert np.all(np.abs(mean[~live] - expected[~live]) <= 1e-12)
    assert (np.abs(mean[live] - expected[live]) / se[live]).max() < 6.0
