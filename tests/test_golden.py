"""Committed golden fixtures (tests/golden/, generated by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from nociwick import synthetic as sy
from oracle.oracle import Oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def tiny_system(g):
    refs = [(g["ca"][i], 3, g["cb"][i], 3) for i in range(g["ca"].shape[0])]
    return sy.System(nmo=6, nocc_a=2, nocc_b=2, s=g["s"], h=g["h"], eri=g["eri"], chol=np.zeros((1, 6, 6)),
                     enuc=float(g["enuc"]), refs=refs)


@pytest.fixture(scope="module")
def tiny():
    return np.load(os.path.join(GOLD, "tiny_zero_overlap.npz"))


def test_fixture_fock_values_pin_exact_convention(tiny):
    """The brute-force Fock-space values stored with the fixture equal the exact convention."""
    n = tiny["fock_hs"].shape[0]
    assert np.max(np.abs(tiny["fock_hs"][:, 0] - tiny["h_exact"][:n])) < 1e-12
    assert np.max(np.abs(tiny["fock_hs"][:, 1] - tiny["s_exact"][:n])) < 1e-12


def test_oracle_reproduces_tiny_fixture(tiny):
    system = tiny_system(tiny)
    orc = Oracle.from_system(system, tol=float(tiny["tol"]))
    ob = orc.oracle_basis(tiny["basis"])
    h, s = orc.eval_pairs(ob, tiny["pairs"])
    he, se = orc.eval_pairs(ob, tiny["pairs"], exact=True)
    assert np.max(np.abs(h - tiny["h_ref"])) < 1e-12 and np.max(np.abs(s - tiny["s_ref"])) < 1e-12
    assert np.max(np.abs(he - tiny["h_exact"])) < 1e-12 and np.max(np.abs(se - tiny["s_exact"])) < 1e-12


def test_oracle_reproduces_config2_fixture():
    g = np.load(os.path.join(GOLD, "config2_sample.npz"))
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    orc = Oracle.from_system(system, tol=1e-8, with_mo_cache=False)
    h, s = orc.eval_pairs(orc.oracle_basis(basis), g["pairs"])
    assert np.max(np.abs(h - g["h"])) < 1e-11 and np.max(np.abs(s - g["s"])) < 1e-11
