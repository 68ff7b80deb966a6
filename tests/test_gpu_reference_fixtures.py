"""The reference's own energy fixtures through the GPU engine (see tests/test_reference_fixtures.py
for the CPU/oracle run and tests/golden/make_reference_fixtures.py for how the fixtures' AO
data and SCF states are rebuilt): reference-space NOCI energies from nw_build_hs_matrix +
nw_general_evp, NOCI-PT2 and selected-NOCI energies from the selected-NOCI driver on the
engine (every matrix element, M and GMRES on the GPU), against the reference's stored
energies."""
import numpy as np
import pytest

import nociwick
import reffix
from nociwick import snoci as sn
from nociwick import synthetic as sy

pytestmark = pytest.mark.gpu

NAMES = reffix.names()


def _engine(system):
    return nociwick.WicksShared(system.s, system.h, system.eri, system.enuc, system.refs, tol=1e-12).build()


@pytest.mark.parametrize("name", [n for n in NAMES if not n.startswith("QMC_")])
def test_reference_noci_energy(name):
    system, meta = reffix.load(name)
    st, _ = sn.reference_states(len(system.refs), system.nocc_a, system.nocc_b)
    with _engine(system) as w:
        w.set_basis(sn.to_nw_dets(st))
        e, _ = sn.solve_current_space(w, st.shape[0], 1e-12)
    assert abs(e - meta["expected"]["reference_noci_energy"]) < 1e-8, (e, meta["expected"])


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith("DET_")])
def test_deterministic_noci_energy(name):
    system, meta = reffix.load(name)
    basis = sy.sd_basis(system.nmo, system.nocc_a, system.nocc_b, len(system.refs), orders=(1, 2),
                        include_refs=True)
    with _engine(system) as w:
        w.set_basis(basis)
        h, s = w.build_hs_matrix()
        e, _ = w.general_evp(h, s, project=True, tol=1e-12)
    assert abs(e[0] - meta["expected"]["deterministic_noci_energy"]) < 1e-8, (e[0], meta["expected"])


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith(("PT2_", "SNOCI_"))])
def test_pt2_and_snoci_energies(name):
    system, meta = reffix.load(name)
    expected = meta["expected_wicks"] or meta["expected"]
    with _engine(system) as w:
        res = sn.snoci(w, system, reffix.snoci_options(meta))
    if name.startswith("PT2_"):
        it = res.iterations[0]
        assert it.gmres["converged"]
        assert abs(it.ecurrent + it.ept2 - expected["noci_pt2_energy"]) < 1e-8, (it.ecurrent + it.ept2, expected)
    else:
        assert abs(res.energy - expected["snoci_energy"]) < 1e-8, (res.energy, expected)


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith("QMC_") and "_TRAJECTORY_" in n])
def test_qmc_trajectory_bounds(name):
    """The reference's DDS-u2 and direct-overlap trajectory fixtures (tests/qmc.rs:195-243,
    487-545): a short NOCI-QMC run with the fixture's qmc / prop blocks (uniform generator, 80
    one-cycle reports from 200 walkers towards 500) must give at least min_samples projected energies, all finite
    and inside [min_energy, max_energy], spanning at least min_energy_span and ending at least
    min_final_drop below the first.  The engine's random stream is Philox, not the reference's
    SmallRng, so its trajectory for seed 1 is a different sample of the same process; with a few
    hundred walkers a single trajectory's end-to-end drop is of the order of its noise.  So every
    one of 8 independent trajectories (seeds 1..8) must satisfy the window, and the span and the
    final drop are required of their mean trajectory."""
    system, meta = reffix.load(name)
    opt, exp = meta["qmc"], meta["expected"]
    basis = sy.sd_basis(system.nmo, system.nocc_a, system.nocc_b, len(system.refs), orders=tuple(meta["orders"]),
                        include_refs=True)
    refs = np.nonzero((basis["rank_a"] == 0) & (basis["rank_b"] == 0))[0].astype(np.uint32)
    runs = []
    with _engine(system) as w:
        w.set_basis(basis)
        hr, sr = w.build_hs_matrix(refs, refs)
        er, cr = w.general_evp(hr, sr, project=True, tol=1e-12)
        c0 = np.zeros(basis.shape[0])
        c0[refs] = cr[:, 0]
        for seed in range(opt["seed"], opt["seed"] + 8):
            with nociwick.Qmc(w, c0, refs, dt=opt["dt"], initial_population=opt["initial_population"],
                              target_population=opt["target_population"], sampling_cutoff=opt["sampling_cutoff"],
                              spawn_cutoff=opt["spawn_cutoff"], initial_shift=float(er[0]), ncycles=opt["ncycles"],
                              propagator=opt["propagator"], seed=seed) as q:
                rep = q.run(opt["nreports"])
            runs.append(rep["eproj_num"] / rep["eproj_den"])
    for e in runs:
        assert e.shape[0] >= exp["min_samples"]
        assert np.all(np.isfinite(e))
        assert np.all((e >= exp["min_energy"]) & (e <= exp["max_energy"])), (e.min(), e.max())
    mean = np.mean(runs, axis=0)
    assert mean.max() - mean.min() >= exp["min_energy_span"], mean
    assert mean[0] - mean[-1] >= exp["min_final_drop"], (mean[0], mean[-1], [e[0] - e[-1] for e in runs])
