"""Loader of tests/golden/reference_fixtures.npz (made by tests/golden/make_reference_fixtures.py
from the reference's energy fixtures): the rebuilt AO data and SCF states of each fixture as a
synthetic.System, its expected energies and the options of its input."""
import json
import os

import numpy as np

from nociwick import snoci as sn
from nociwick import synthetic as sy

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures.npz")


def names():
    with np.load(PATH) as z:
        return sorted(json.loads(bytes(z["meta"]).decode()).keys())


def load(name):
    with np.load(PATH) as z:
        meta = json.loads(bytes(z["meta"]).decode())[name]
        s, h, eri = z[f"{name}/s"], z[f"{name}/h"], z[f"{name}/eri"]
        ca, cb = z[f"{name}/ca"], z[f"{name}/cb"]
    n, no = s.shape[0], meta["nocc"]
    occ = (1 << no) - 1
    refs = [(ca[r], occ, cb[r], occ) for r in range(ca.shape[0])]
    system = sy.System(nmo=n, nocc_a=no, nocc_b=no, s=s, h=h, eri=eri, chol=np.zeros((1, n, n)),
                       enuc=float(meta["enuc"]), refs=refs)
    return system, meta


def snoci_options(meta) -> "sn.SnociOptions":
    """SnociOptions of a fixture's input: its excitation orders and snoci block on top of the
    reference defaults (sigma 1e-6, tol 1e-8, max_add 1, max_dim 100, Woodbury), with the
    1e-12 zero tolerance of the reference's fixture tests (tests/snoci.rs:58)."""
    b = meta["snoci"]
    return sn.SnociOptions(max_iter=b["max_iter"], max_add=b.get("max_add", 1), sigma=1e-6, tol=1e-8, max_dim=100,
                           lin_tol=1e-12, orders=tuple(meta["orders"]), gmres_max_iter=b["gmres_max_iter"],
                           gmres_restart=b["restart"],
                           gmres_res_tol=b["res_tol"], preconditioner="woodbury")
