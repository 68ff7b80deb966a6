"""The reference's own energy fixtures (noci-rs tests/fixtures/*/expected.json), reproduced on
the CPU through the oracle.  The fixtures' AO data and SCF states are rebuilt from first
principles by tests/golden/make_reference_fixtures.py (their SCF energies match the stored
ones to 2e-14 Eh); here the oracle's matrix elements give

* the reference-space NOCI energy (calculate_noci_energy: H, S over the SCF states, GEVP with
  the positive-subspace projection), to 1e-8 Eh (measured: 5e-15 to 2e-9; the NOCI energy is
  first order in the reference orbitals, which the reference's own SCF converges to
  e_tol = 1e-12 only, hence LiH's 2e-9); square H4 includes zero-overlap (m = 1 per spin)
  reference pairs, i.e. the distribution-sum evaluator;
* the deterministic NOCI-QMC energy (tests/deterministic.rs: converged propagation in the
  singles-and-doubles basis of the references) as the lowest GEVP root over that basis, to
  1e-8 Eh (F2: 300 determinants, excited-excited pairs across references);
* the NOCI-PT2 energy E_current + E_PT2 of one snoci_step (tests/pt2.rs:31-84) and the
  selected-NOCI energy after the fixture's SNOCI iterations (tests/snoci.rs:33-79), through
  the selected-NOCI driver nociwick.snoci run on the dense oracle engine (oracle/engine.py),
  to 1e-8 Eh.

This pins the oracle, and with the GPU parity tests the engine, against numbers produced by
the reference itself.
"""
import numpy as np
import pytest

import reffix
from nociwick import snoci as sn
from nociwick import synthetic as sy
from oracle import linalg as LA
from oracle.engine import DenseEngine
from oracle.oracle import Oracle

REF_NOCI = [n for n in reffix.names() if not n.startswith("QMC_")]
DET = [n for n in reffix.names() if n.startswith("DET_")]
PT2 = [n for n in reffix.names() if n.startswith("PT2_")]
SNOCI = [n for n in reffix.names() if n.startswith("SNOCI_")]


def reference_noci(system, tol=1e-12):
    nref = len(system.refs)
    basis = sy.sd_basis(system.nmo, system.nocc_a, system.nocc_b, nref, orders=(1,), include_refs=True)
    basis = basis[(basis["rank_a"] == 0) & (basis["rank_b"] == 0)]
    orc = Oracle.from_system(system, tol=tol)
    ob = orc.oracle_basis(basis)
    pairs = np.array([(i, j) for i in range(nref) for j in range(nref)])
    h, s = orc.eval_pairs(ob, pairs)
    e, _ = LA.general_evp(h.reshape(nref, nref), s.reshape(nref, nref), True, tol)
    return float(e[0])


@pytest.mark.parametrize("name", REF_NOCI)
def test_reference_noci_energy(name):
    system, meta = reffix.load(name)
    assert np.allclose(sorted(meta["scf_energies"]), sorted(meta["expected"]["scf_energies"]), atol=1e-12)
    e = reference_noci(system)
    assert abs(e - meta["expected"]["reference_noci_energy"]) < 1e-8, (e, meta["expected"])


@pytest.mark.parametrize("name", DET)
def test_deterministic_noci_energy(name):
    """The deterministic NOCI-QMC energy of tests/deterministic.rs: its propagation in the
    singles-and-doubles basis of the references (references included) converges to the lowest
    root of H c = E S c over that basis."""
    system, meta = reffix.load(name)
    basis = sy.sd_basis(system.nmo, system.nocc_a, system.nocc_b, len(system.refs), orders=(1, 2),
                        include_refs=True)
    with DenseEngine(system, tol=1e-12) as eng:
        eng.set_basis(basis)
        h, s = eng.build_hs_matrix()
        e, _ = eng.general_evp(h, s, True, 1e-12)
    assert abs(e[0] - meta["expected"]["deterministic_noci_energy"]) < 1e-8, (e[0], meta["expected"])


@pytest.mark.parametrize("name", PT2)
def test_noci_pt2_energy(name):
    system, meta = reffix.load(name)
    opts = reffix.snoci_options(meta)
    with DenseEngine(system, tol=1e-12) as eng:
        res = sn.snoci(eng, system, opts)
    it = res.iterations[0]
    assert abs(it.ecurrent - meta["expected"]["reference_noci_energy"]) < 1e-10
    assert abs(it.ecurrent + it.ept2 - meta["expected"]["noci_pt2_energy"]) < 1e-8, (it.ecurrent + it.ept2, meta)


@pytest.mark.parametrize("name", SNOCI)
def test_snoci_energy(name):
    """Against the Wick-path twin of the fixture (the reference runs each SNOCI input through
    its naive and its Wick paths; for H4 they select different determinants, and the engine
    restates the Wick path)."""
    system, meta = reffix.load(name)
    expected = meta["expected_wicks"] or meta["expected"]
    opts = reffix.snoci_options(meta)
    with DenseEngine(system, tol=1e-12) as eng:
        res = sn.snoci(eng, system, opts)
    assert abs(res.iterations[0].ecurrent - expected["reference_noci_energy"]) < 1e-10
    assert abs(res.energy - expected["snoci_energy"]) < 1e-8, (res.energy, expected, res.stop,
                                                            [i.ecurrent for i in res.iterations])
