"""Why the engine keeps every stored intermediate in FP64 (the 1e-9 Eh element bar).

In the stored-intermediate formulation the evaluator's work is gathers of precomputed
intermediates; the only way a lower precision reduces its bytes is to store them narrower.
With every intermediate of the oracle rounded to FP32 (halving the stored bytes), the
Hamiltonian elements of the bench workload's pairs move by up to 4e-8 Eh (rms ~1e-9), above
the 1e-9 Eh bar, so no FP32 storage class is admissible; the two-electron tensors alone are at
most 46 % of a pair's algorithmic bytes (La = Lb = 2), which bounds what a partial narrowing
could gain to 1.3x.  The measurement is repeated here so the numbers can be checked.
"""
import numpy as np

from nociwick import synthetic as sy
from oracle.oracle import Oracle


def test_fp32_intermediates_exceed_the_element_bar():
    system = sy.config2_system()
    basis = sy.sd_basis(30, 3, 3, 3)
    pairs = sy.sample_pairs(basis, 20000, seed=7)
    orc = Oracle.from_system(system, tol=1e-8, with_mo_cache=False)
    ob = orc.oracle_basis(basis)
    h64, s64 = orc.eval_pairs(ob, pairs)
    slab = orc.slab.copy()
    orc.slab = slab.astype(np.float32).astype(np.float64)
    h32, s32 = orc.eval_pairs(ob, pairs)
    orc.slab = slab
    dh = np.abs(h32 - h64)
    print("FP32 intermediates: max |dH|", dh.max(), "rms", np.sqrt(np.mean(dh ** 2)), "max |dS|", np.abs(s32 - s64).max())
    assert dh.max() > 1e-8          # well above the 1e-9 Eh bar
    assert np.sqrt(np.mean(dh ** 2)) > 5e-10
