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


@pytest.mark.parametrize("name", NAMES)
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
