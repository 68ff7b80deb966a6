"""Generate the golden fixtures in tests/golden/ (run from the repository root).

tiny_zero_overlap.npz  - n = 6, 2 + 2 electrons, 3 references, one alpha zero-overlap pair:
                         the AO data and orbitals themselves, 300 determinant pairs (same-parent
                         pairs included) with the oracle's (H, S) in the reference and exact
                         conventions, and 40 of them evaluated by brute force in Fock space.
config2_sample.npz     - the n = 30 stand-in workload of bench.py: a checksum of its generated
                         AO data and orbitals, 3000 of its pairs, and the oracle's (H, S).

Values come from the FP64 oracle (oracle/) and the brute-force Fock-space evaluator; they
freeze the oracle's behaviour so that later changes to either the oracle or the engine are
caught against fixed numbers.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "noci-rs_b200"))

from nociwick import synthetic as sy  # noqa: E402
from oracle.fockspace import FockSpace, hs_element  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def system_digest(system) -> str:
    h = hashlib.sha256()
    for a in (system.s, system.h, system.eri):
        h.update(np.ascontiguousarray(a).tobytes())
    for ca, oa, cb, ob in system.refs:
        h.update(np.ascontiguousarray(ca).tobytes())
        h.update(np.ascontiguousarray(cb).tobytes())
        h.update(f"{oa},{ob}".encode())
    return h.hexdigest()


def tiny():
    system = sy.make_system(6, 2, 2, 3, 12, seed=21, k_scale=0.3, zero_pairs=[(0, 1, 1, 0)], enuc=0.53)
    basis = sy.sd_basis(6, 2, 2, 3)
    pairs = sy.sample_pairs(basis, 300, seed=22, distinct_parents=False)
    orc = Oracle.from_system(system, tol=1e-8)
    ob = orc.oracle_basis(basis)
    h_ref, s_ref = orc.eval_pairs(ob, pairs)
    h_ex, s_ex = orc.eval_pairs(ob, pairs, exact=True)
    fs = FockSpace(6, 2, 2)
    fock = np.array([hs_element(fs, orc.h, orc.eri, orc.enuc, orc.det_orbitals(ob, int(a)),
                                orc.det_orbitals(ob, int(b))) for a, b in pairs[:40]])
    np.savez_compressed(os.path.join(OUT, "tiny_zero_overlap.npz"), s=system.s, h=system.h, eri=system.eri,
                        enuc=system.enuc, ca=np.stack([r[0] for r in system.refs]),
                        cb=np.stack([r[2] for r in system.refs]), nocc=np.array([2, 2]), basis=basis, pairs=pairs,
                        h_ref=h_ref, s_ref=s_ref, h_exact=h_ex, s_exact=s_ex, fock_hs=fock, tol=1e-8)


def config2():
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 3000, seed=12345)
    orc = Oracle.from_system(system, tol=1e-8, with_mo_cache=False)
    h, s = orc.eval_pairs(orc.oracle_basis(basis), pairs)
    np.savez_compressed(os.path.join(OUT, "config2_sample.npz"), digest=system_digest(system), pairs=pairs,
                        h=h, s=s)


if __name__ == "__main__":
    tiny()
    config2()
    print("wrote", sorted(f for f in os.listdir(OUT) if f.endswith(".npz")))
