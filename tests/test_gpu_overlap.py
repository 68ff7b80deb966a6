"""Overlap action y += S x over the resident basis (nw_apply_overlap_device) and the
direct-overlap NOCI-QMC propagator built on it (qmc_step of src/stochastic/metric.rs:766-1087).

* The action equals the engine's own overlap matrix (nw_build_hs_matrix, itself checked against
  the oracle) times x, and the oracle's restatement of the spin-factorised contraction
  (oracle/overlap_action.py), on systems with and without zero-overlap reference pairs, with a
  duplicated determinant, with a record whose phase is not the canonical one and through
  quadruple excitations in one spin.
* Direct overlap: the populations start at S c_0 scaled to the initial 1-norm; one report of one
  cycle changes them by exactly S times that cycle's change; they stay in the range of S on an
  overcomplete basis; the mean over independent runs follows the deterministic recursion; and a
  run at a fixed shift tracks the deterministic projected energy on its way to the lowest root.
"""
import numpy as np
import pytest

import nociwick
from nociwick import synthetic as sy
from oracle.overlap_action import OverlapFactorisation

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _apply(w, x, y0=None):
    dx = torch.from_numpy(np.ascontiguousarray(x, np.float64)).cuda()
    dy = torch.from_numpy(np.zeros_like(x) if y0 is None else np.array(y0, np.float64)).cuda()
    w.apply_overlap_device(dx.data_ptr(), dy.data_ptr(), _stream())
    w.sync(_stream())
    return dy.cpu().numpy()


@pytest.mark.parametrize("zero_pairs", [(), ((0, 1, 1, 0), (1, 2, 0, 2))])
def test_overlap_action_matches_overlap_matrix(zero_pairs):
    system = sy.make_system(10, 3, 2, 3, 16, seed=4, k_scale=0.3, zero_pairs=list(zero_pairs))
    basis = sy.sd_basis(10, 3, 2, 3)
    rng = np.random.default_rng(9)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        _, s = w.build_hs_matrix()
        x = rng.standard_normal(basis.shape[0]) * (rng.random(basis.shape[0]) < 0.5)
        y0 = rng.standard_normal(basis.shape[0])
        y = _apply(w, x, y0)
        y2 = _apply(w, x)          # second call reuses the factor tables
    ref = y0 + s @ x
    scale = np.abs(s).max() * np.abs(x).sum()
    assert np.abs(y - ref).max() <= 1e-13 * scale, np.abs(y - ref).max() / scale
    f = OverlapFactorisation(system.s, system.refs, 3, 2, basis)
    assert np.abs(y2 - f.apply(x)).max() <= 1e-13 * scale


def test_overlap_action_duplicates_and_phases():
    """A duplicated determinant (overlap 1 with its twin) and a record whose phase is the
    negative of its canonical excitation phase (its row and column of S change sign)."""
    system = sy.make_system(8, 2, 2, 3, 12, seed=6, k_scale=0.3)
    basis = sy.sd_basis(8, 2, 2, 3)
    basis = np.concatenate([basis, basis[[5, 140]]])
    basis["phase"][7] *= -1.0
    rng = np.random.default_rng(2)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        _, s = w.build_hs_matrix()
        x = rng.standard_normal(basis.shape[0])
        y = _apply(w, x)
    assert abs(s[5, basis.shape[0] - 2] - 1.0) < 1e-14
    scale = np.abs(s).max() * np.abs(x).sum()
    assert np.abs(y - s @ x).max() <= 1e-13 * scale


def test_overlap_action_needs_a_basis():
    system = sy.make_system(6, 2, 2, 2, 10, seed=1)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs) as w:
        x = torch.zeros(4, dtype=torch.float64, device="cuda")
        with pytest.raises(nociwick.NwError) as e:
            w.apply_overlap_device(x.data_ptr(), x.data_ptr(), _stream())
        assert e.value.status == 5


def _setup(seed=3, zero_pairs=()):
    # 2 references, n = 8, 2 + 2 electrons: the 186 singles and doubles are linearly dependent
    # (S has 18 null directions)
    system = sy.make_system(8, 2, 2, 2, 20, seed=seed, k_scale=0.3, zero_pairs=list(zero_pairs))
    basis = sy.sd_basis(8, 2, 2, 2)
    w = nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8).build()
    w.set_basis(basis)
    h, s = w.build_hs_matrix()
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0]
    return w, basis, h, s, refs


@pytest.mark.parametrize("zero_pairs", [(), ((0, 1, 1, 0),)])
def test_direct_overlap_start_and_one_report(zero_pairs):
    w, basis, h, s, refs = _setup(zero_pairs=zero_pairs)
    nd = basis.shape[0]
    c0 = np.zeros(nd)
    c0[refs] = [0.8, 0.6]
    with w, nociwick.Qmc(w, c0, refs, dt=0.004, initial_population=300.0, target_population=1e5,
                         sampling_cutoff=0.5, spawn_cutoff=0.05, initial_shift=-5.2, ncycles=1,
                         propagator="direct-overlap", seed=7) as q:
        n0 = q.populations()
        sc0 = s @ c0
        assert np.abs(n0 - 300.0 * sc0 / np.abs(sc0).sum()).max() <= 1e-12 * np.abs(n0).max()
        for k in range(3):
            before = q.populations()
            d = q.cycle_delta(k)
            rep = q.run(1)
            after = q.populations()
            scale = np.abs(s).max() * np.abs(d).sum()
            assert np.abs((after - before) - s @ d).max() <= 1e-12 * scale
            assert np.abs(d).max() > 0
            assert abs(rep["nw"][0] - np.abs(after).sum()) <= 1e-9 * rep["nw"][0]


def test_direct_overlap_stays_in_the_range_of_s():
    """On the overcomplete basis the null-space part of N stays at rounding level, while the
    signed-walker propagator's change, Delta itself, has a null-space part of its own size."""
    w, basis, h, s, refs = _setup()
    nd = basis.shape[0]
    ev, vec = np.linalg.eigh(s)
    null = vec[:, ev < 1e-10 * ev.max()]
    assert null.shape[1] >= 10
    c0 = np.zeros(nd)
    c0[refs] = 1.0
    with w, nociwick.Qmc(w, c0, refs, dt=0.004, initial_population=500.0, target_population=1e5,
                         sampling_cutoff=0.5, spawn_cutoff=0.05, initial_shift=-5.2, ncycles=5,
                         propagator="direct-overlap", seed=3, update_cutoff=0.02) as q:
        d = q.cycle_delta(0)
        q.run(60)
        n = q.populations()
    assert np.linalg.norm(null.T @ d) > 1e-3 * np.linalg.norm(d)
    assert np.linalg.norm(null.T @ n) <= 1e-10 * np.linalg.norm(n), np.linalg.norm(null.T @ n) / np.linalg.norm(n)


def _deterministic(h, s, n0, dt, es, steps):
    """The expectation of the direct-overlap recursion with a fixed shift:
    N_{k+1} = N_k - dt S (H - es S) N_k."""
    a = np.eye(h.shape[0]) - dt * s @ (h - es * s)
    out = [n0]
    for _ in range(steps):
        out.append(a @ out[-1])
    return np.array(out)


def test_direct_overlap_report_is_unbiased():
    """With a fixed shift (no damping) the report map is linear in expectation, so the mean of
    N_k over independent runs is the deterministic iterate (I - dt S (H - E S))^k N_0, here after
    30 one-cycle reports with FRI sampling, spawn rounding and FRI-compressed updates."""
    w, basis, h, s, refs = _setup(zero_pairs=((0, 1, 1, 0),))
    nd = basis.shape[0]
    c0 = np.zeros(nd)
    c0[refs] = [0.8, 0.6]
    es, dt, k, runs = -3.0, 0.004, 30, 48
    out = []
    with w:
        for seed in range(runs):
            with nociwick.Qmc(w, c0, refs, dt=dt, initial_population=400.0, target_population=1e6,
                              sampling_cutoff=0.5, spawn_cutoff=0.05, shift_damping=0.0, initial_shift=es,
                              ncycles=1, propagator="direct-overlap", seed=100 + seed, update_cutoff=0.05,
                              max_attempts=1_000_000) as q:
                n0 = q.populations()
                q.run(k)
                out.append(q.populations())
    out = np.array(out)
    expected = _deterministic(h, s, n0, dt, es, k)[-1]
    mean = out.mean(axis=0)
    se = out.std(axis=0, ddof=1) / np.sqrt(runs)
    live = se > 1e-12 * np.abs(expected).max()
    z = np.abs(mean[live] - expected[live]) / se[live]
    assert z.max() < 6.0, z.max()
    if (~live).any():
        assert np.abs(mean[~live] - expected[~live]).max() <= 1e-9 * np.abs(expected).max()


def test_direct_overlap_run_approaches_ground_state():
    """A run at a fixed shift E_0 follows the deterministic direct-overlap iteration, whose
    projected energy approaches the lowest root of H c = E S c (S-preconditioned, so modes of
    small overlap eigenvalue relax slowly: 1.6 mEh above E_0 on average over cycles 3000-7000
    at dt = 0.02 on this system): the run's projected energy over those cycles equals the
    deterministic one within its blocked error bar."""
    w, basis, h, s, refs = _setup()
    nd = basis.shape[0]
    with w:
        e, c = w.general_evp(h, s, project=True, tol=1e-8)
        e0 = e[0]
        er, cr = w.general_evp(h[np.ix_(refs, refs)], s[np.ix_(refs, refs)], project=True, tol=1e-8)
        c0 = np.zeros(nd)
        c0[refs] = cr[:, 0]
        dt, ncyc, nrep = 0.02, 1, 7000
        with nociwick.Qmc(w, c0, refs, dt=dt, initial_population=2000.0, target_population=1e6,
                          sampling_cutoff=0.5, spawn_cutoff=0.05, shift_damping=0.0, initial_shift=e0,
                          ncycles=ncyc, propagator="direct-overlap", seed=2025, max_attempts=20_000_000) as q:
            n0 = q.populations()
            rep = q.run(nrep)
    assert np.all(np.isfinite(rep["nw"]))
    det = _deterministic(h, s, n0, dt * ncyc, e0, nrep)[1:]   # one report of one cycle per step
    ref_row = c0 @ h, c0 @ s
    tail = slice(3000, nrep)
    e_det = (det[tail] @ ref_row[0]).sum() / (det[tail] @ ref_row[1]).sum()
    assert 0.0 < e_det - e0 < 5e-3, e_det - e0
    eproj = rep["eproj_num"][tail] / rep["eproj_den"][tail]
    blocks = eproj[: (len(eproj) // 200) * 200].reshape(-1, 200).mean(axis=1)
    mean = rep["eproj_num"][tail].sum() / rep["eproj_den"][tail].sum()
    err = blocks.std(ddof=1) / np.sqrt(len(blocks))
    assert abs(mean - e_det) < 5 * err + 5e-4, (mean, e_det, e0, err)


def test_overlap_action_single_parent_and_missing_parent():
    """One reference (only the orthonormal same-parent block) and a basis in which a middle
    reference has no determinants (empty parent blocks on both sides of the contraction)."""
    rng = np.random.default_rng(5)
    one = sy.make_system(8, 2, 2, 1, 12, seed=2, k_scale=0.3)
    b1 = sy.sd_basis(8, 2, 2, 1)
    with nociwick.WicksShared(one.s, one.h, one.eri, one.enuc, one.refs, tol=1e-8) as w:
        w.build().set_basis(b1)
        x = rng.standard_normal(b1.shape[0])
        y = _apply(w, x)
    assert np.abs(y - x).max() <= 1e-15 * np.abs(x).max()
    three = sy.make_system(8, 2, 2, 3, 12, seed=9, k_scale=0.3)
    b3 = sy.sd_basis(8, 2, 2, 3)
    b3 = b3[b3["parent"] != 1]
    with nociwick.WicksShared(three.s, three.h, three.eri, three.enuc, three.refs, tol=1e-8) as w:
        w.build().set_basis(b3)
        _, s = w.build_hs_matrix()
        x = rng.standard_normal(b3.shape[0])
        y = _apply(w, x)
    assert np.abs(y - s @ x).max() <= 1e-13 * np.abs(s).max() * np.abs(x).sum()


@pytest.mark.parametrize("nocc", [6, 9])
def test_overlap_action_more_occupied_orbitals(nocc):
    """Single-spin determinants of 6 and 9 occupied orbitals (the factor kernel's larger LU
    scratch variants), singles and doubles of three references."""
    n = nocc + 5
    system = sy.make_system(n, nocc, nocc, 3, 16, seed=nocc, k_scale=0.2)
    basis = sy.sd_basis(n, nocc, nocc, 3)
    rng = np.random.default_rng(nocc)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        _, s = w.build_hs_matrix()
        x = rng.standard_normal(basis.shape[0])
        y = _apply(w, x)
    scale = np.abs(s).max() * np.abs(x).sum()
    assert np.abs(y - s @ x).max() <= 1e-12 * scale, np.abs(y - s @ x).max() / scale


def test_overlap_action_through_quadruple_excitations():
    """Singles to quadruples of two references with 4 alpha and 3 beta electrons (single-spin
    strings of rank 3 and 4): the action equals the engine's S times x and the oracle's
    factorised contraction."""
    system = sy.make_system(8, 4, 3, 2, 12, seed=12, k_scale=0.3)
    basis = sy.sd_basis(8, 4, 3, 2, orders=(1, 2, 3, 4))
    rng = np.random.default_rng(13)
    with nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-8) as w:
        w.build().set_basis(basis)
        _, s = w.build_hs_matrix()
        x = rng.standard_normal(basis.shape[0])
        y = _apply(w, x)
    scale = np.abs(s).max() * np.abs(x).sum()
    assert np.abs(y - s @ x).max() <= 1e-13 * scale, np.abs(y - s @ x).max() / scale
    f = OverlapFactorisation(system.s, system.refs, 4, 3, basis)
    assert np.abs(y - f.apply(x)).max() <= 1e-13 * scale
