"""GPU learned spawning proposal (nw_qmc_harvest / train_proposal / set_generator and the MLP
entry points) against the numpy restatement in oracle/proposal.py.

The proposal has no counterpart in noci-rs (its generators are uniform, heat-bath and
overlap-weighted, src/input/qmc.rs:10); what must hold is what any generator of
propagate_iteration (src/stochastic/metric.rs:378-473) must satisfy:

* the network's loss and gradient, and the bin probabilities of the proposal table, equal the
  restatement's on the same parameters (BF16 weights, FP32 accumulation vs FP64: rtol 1e-3);
* training on harvested attempts lowers the weighted cross entropy;
* one cycle's population change under the learned mixture is still an unbiased estimate of
  -dt (H - E_s S) N, per determinant within 6 standard errors;
* the trained proposal lowers the second moment sum_l (H - E_s S)_lg^2 / pgen(l | g) of the
  spawned amplitude below the uniform generator's, which is what it is trained for.
"""
import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy
from oracle import proposal as PR

pytestmark = pytest.mark.gpu

NMO, NREF = 8, 2


def _setup(seed=3):
    system = sy.make_system(NMO, 2, 2, NREF, 20, seed=seed, k_scale=0.3)
    basis = sy.sd_basis(NMO, 2, 2, NREF)
    w = nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build()
    w.set_basis(basis)
    h, s = w.build_hs_matrix()
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    return w, basis, h, s, refs


def _qmc(w, basis, refs, es, **kw):
    c0 = np.zeros(basis.shape[0])
    c0[refs] = 1.0
    args = dict(dt=0.004, initial_population=100.0, sampling_cutoff=0.5, spawn_cutoff=0.0, initial_shift=es,
                propagator="unshifted", seed=11)
    args.update(kw)
    return nociwick.Qmc(w, c0, refs, **args)


def _rows(rng, basis, det_bin, sizes, n):
    parents = rng.integers(0, basis.shape[0], n)
    mask = PR.valid_mask(det_bin, sizes, parents)
    tb = np.array([rng.choice(np.nonzero(mask[i])[0]) for i in range(n)])
    return parents, tb, mask


def test_loss_and_gradient_match_oracle():
    w, basis, h, s, refs = _setup()
    det_bin, sizes = PR.bins(basis, NREF)
    with w, _qmc(w, basis, refs, -1.0) as q:
        din, nbin, npar = q.proposal_dims()
        assert nbin == NREF * PR.RANK_BINS and din == 32
        rng = np.random.default_rng(1)
        params = q.mlp_params().astype(np.float32)
        params[din * 128:din * 128 + 128] = rng.normal(0.0, 0.2, 128)     # nonzero biases
        q.set_mlp_params(params)
        parents, tb, mask = _rows(rng, basis, det_bin, sizes, 300)
        wt = rng.uniform(0.05, 3.0, 300).astype(np.float32)
        loss, g = q.mlp_loss_grad(parents, tb, wt)
    x = PR.features(basis, parents, NREF, NMO, din)
    lo, go = PR.loss_grad(params, x, mask, tb, wt.astype(np.float64), din, nbin)
    assert abs(loss - lo) <= 1e-4 * abs(lo), (loss, lo)
    assert np.abs(g - go).max() <= 1e-3 * np.abs(go).max(), np.abs(g - go).max() / np.abs(go).max()


def test_proposal_table_matches_oracle():
    w, basis, h, s, refs = _setup()
    det_bin, sizes = PR.bins(basis, NREF)
    with w, _qmc(w, basis, refs, -1.0) as q:
        din, nbin, npar = q.proposal_dims()
        params = (q.mlp_params() * 2.0).astype(np.float32)   # sharper distributions than the initial ones
        q.set_mlp_params(params)
        dets = np.array([0, 1, 17, 60, basis.shape[0] // 2, basis.shape[0] - 1])
        got = np.array([q.proposal_probs(int(d)) for d in dets])
    x = PR.features(basis, dets, NREF, NMO, din)
    _, _, z = PR.forward(params, x, din, nbin)
    mask = PR.valid_mask(det_bin, sizes, dets)
    ref = PR.probs(z, mask)
    assert np.all(got[~mask] == 0.0)
    assert np.allclose(got.sum(axis=1), 1.0, atol=1e-6)
    assert np.abs(got - ref).max() <= 1e-5 + 1e-3 * ref.max()


def test_training_and_learned_generator():
    w, basis, h, s, refs = _setup()
    nd = basis.shape[0]
    det_bin, sizes = PR.bins(basis, NREF)
    es, dt = -1.3, 0.004
    with w:
        e0 = w.general_evp(h, s, project=True, tol=1e-8)[0][0]
        with _qmc(w, basis, refs, e0, initial_population=2000.0, target_population=2e4, shift_damping=0.05,
                  ncycles=10, max_attempts=4_000_000) as q:
            with pytest.raises(nociwick.NwError):
                q.set_generator(True, 0.1)                 # nothing trained yet
            q.harvest(True)
            q.run(20)
            q.harvest(False)
            rep = q.train_proposal(epochs=8, batch=2048, lr=2e-3, seed=5)
            assert rep["samples"] > 10_000 and rep["steps"] > 0
            assert rep["loss_last"] < 0.8 * rep["loss_first"], rep

            # second moment of the spawned amplitude, per parent, learned vs uniform
            pop = q.populations()
            k_mat = h - e0 * s
            occ = np.nonzero(pop)[0]
            m2_l = m2_u = 0.0
            for g in occ:
                pb = q.proposal_probs(int(g))
                lam = np.delete(np.arange(nd), g)
                size = sizes[det_bin[lam]] - (det_bin[lam] == det_bin[g])
                pgen = 0.1 / (nd - 1) + 0.9 * pb[det_bin[lam]] / size
                assert np.all(pgen > 0)
                m2_l += abs(pop[g]) * np.sum(k_mat[lam, g] ** 2 / pgen)
                m2_u += abs(pop[g]) * (nd - 1) * np.sum(k_mat[lam, g] ** 2)
            print("second moment learned / uniform:", m2_l / m2_u)
            assert m2_l < 0.9 * m2_u, (m2_l, m2_u)

            # unbiased one-cycle change under the learned mixture
            q.set_generator(True, 0.1)
            rng = np.random.default_rng(5)
            pop = rng.normal(0.0, 3.0, nd) * (rng.random(nd) < 0.3)
            q.set_shift(es)
            q.set_populations(pop)
            k = 3000
            d = np.array([q.cycle_delta(c) for c in range(k)])
    expected = -dt * (h - es * s) @ pop
    mean = d.mean(axis=0)
    se = d.std(axis=0, ddof=1) / np.sqrt(k)
    live = se > 0
    assert np.all(np.abs(mean[~live] - expected[~live]) <= 1e-12)
    z = np.abs(mean[live] - expected[live]) / se[live]
    assert z.max() < 6.0, z.max()


def test_invalid_training_rows_are_rejected():
    w, basis, h, s, refs = _setup()
    det_bin, sizes = PR.bins(basis, NREF)
    empty = int(np.nonzero(sizes == 0)[0][0])            # e.g. rank (4, 4): no determinant there
    with w, _qmc(w, basis, refs, -1.0) as q:
        with pytest.raises(nociwick.NwError):
            q.mlp_loss_grad([0], [empty], [1.0])
        with pytest.raises(nociwick.NwError):
            q.mlp_loss_grad([0], [det_bin[1]], [float("nan")])
        with pytest.raises(nociwick.NwError):
            q.train_proposal()                            # nothing harvested


def test_learned_run_converges_to_noci_ground_state():
    """A full run with shift control under the learned mixture estimates the same energy as the
    uniform generator: the lowest eigenvalue of H c = E S c, within its blocked error bar."""
    w, basis, h, s, refs = _setup()
    nd = basis.shape[0]
    with w:
        e0 = w.general_evp(h, s, project=True, tol=1e-8)[0][0]
        er, cr = w.general_evp(h[np.ix_(refs, refs)], s[np.ix_(refs, refs)], project=True, tol=1e-8)
        c0 = np.zeros(nd)
        c0[refs] = cr[:, 0]
        e_ref0 = h[refs[0], refs[0]] / s[refs[0], refs[0]]
        with nociwick.Qmc(w, c0, refs, dt=0.004, initial_population=500.0, target_population=3e5,
                          shift_damping=0.05, initial_shift=e_ref0, ncycles=10, propagator="unshifted",
                          seed=77, max_attempts=20_000_000) as q:
            q.run(200)
            q.harvest(True)
            q.run(2)
            q.harvest(False)
            q.train_proposal(epochs=4, batch=4096, lr=1e-3, seed=3)
            q.set_generator(True, 0.1)
            rep = q.run(600)
    tail = rep[100:]
    eproj = tail["eproj_num"] / tail["eproj_den"]
    blocks = eproj[: (len(eproj) // 25) * 25].reshape(-1, 25).mean(axis=1)
    mean = tail["eproj_num"].sum() / tail["eproj_den"].sum()
    err = blocks.std(ddof=1) / np.sqrt(len(blocks))
    print("learned run: E_proj", mean, "+-", err, "E0", e0)
    assert abs(mean - e0) < 5 * err + 5e-4, (mean, e0, err)
    assert abs(tail["shift"].mean() - e0) < 0.05
