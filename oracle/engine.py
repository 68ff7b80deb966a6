"""Dense CPU stand-in for the engine surface the selected-NOCI driver uses (test
infrastructure only): the same methods as nociwick.WicksShared -- set_basis, build_hs_matrix,
build_fs_matrix, general_evp, update_fock, pt2 -- backed by the FP64 oracle's matrix elements
(oracle/oracle.py: the restated Wick path with the same-parent Slater-Condon dispatch of
src/noci/hs.rs), the restated general_evp (oracle/linalg.py, src/maths/linalg.rs:180-256) and
the CPU GMRES with the reference preconditioners (oracle/pt2.py, src/snoci/gmres.rs,
src/snoci/types.rs).  Driving nociwick.snoci.snoci with it gives a CPU run of the whole SNOCI
loop to compare with the GPU run and with the reference's stored energies.
"""
from __future__ import annotations

import numpy as np

from . import linalg as LA
from . import pt2 as PT
from .oracle import Oracle


class DensePt2:
    """M = F - E0 S over the candidates as a dense matrix, its product and GMRES on M^Omega."""

    def __init__(self, engine: "DenseEngine", cand, e0: float):
        cand = np.asarray(cand, dtype=np.int64)
        f, s = engine.build_fs_matrix(cand, cand, symmetric=True)
        self.m = f - e0 * s

    def apply_m(self, x):
        return self.m @ np.asarray(x, dtype=np.float64)

    def solve(self, e0, s_a0, s_0a, f_a0, f_0a, rhs, max_iter=100, restart=200, res_tol=1e-8,
              preconditioner="woodbury"):
        p = {"e0": e0, "s_a0": np.asarray(s_a0), "s_0a": np.asarray(s_0a), "f_a0": np.asarray(f_a0),
             "f_0a": np.asarray(f_0a)}
        pre = PT.preconditioner(np.diag(self.m).copy(), p, preconditioner)
        x, res, it, conv = PT.gmres(lambda z: PT.apply_omega(self.m, p, z), pre, np.asarray(rhs, dtype=np.float64),
                                    max_iter=max_iter, restart=restart, res_tol=res_tol)
        return x, {"residual_rms": float(res), "iterations": int(it), "converged": bool(conv)}

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class DenseEngine:
    def __init__(self, system, tol: float = 1e-8):
        self.orc = Oracle.from_system(system, tol=tol)
        self.ob = None
        self.n = 0

    def set_basis(self, dets: np.ndarray):
        self.ob = self.orc.oracle_basis(dets)
        self.n = dets.shape[0]
        return self

    def _pairs(self, left, right):
        left = np.arange(self.n) if left is None else np.asarray(left, dtype=np.int64)
        right = left if right is None else np.asarray(right, dtype=np.int64)
        pairs = np.stack(np.meshgrid(left, right, indexing="ij"), axis=-1).reshape(-1, 2)
        return left.shape[0], right.shape[0], pairs

    def build_hs_matrix(self, left=None, right=None, symmetric: bool = True):
        nl, nr, pairs = self._pairs(left, right)
        h, s = self.orc.eval_pairs(self.ob, pairs)
        return h.reshape(nl, nr), s.reshape(nl, nr)

    def build_fs_matrix(self, left=None, right=None, symmetric: bool = True):
        nl, nr, pairs = self._pairs(left, right)
        _, f, s = self.orc.eval_m_pairs(self.ob, pairs, 0.0)
        return f.reshape(nl, nr), s.reshape(nl, nr)

    def general_evp(self, h, s, project: bool = True, tol: float = 1e-8):
        return LA.general_evp(h, s, project, tol)

    def update_fock(self, fa, fb):
        self.orc.set_fock(fa, fb)
        return self

    def pt2(self, cand, e0: float, matrix_free: bool = False) -> DensePt2:
        # the dense oracle forms M itself either way; matrix_free only selects the GPU storage mode
        return DensePt2(self, cand, e0)

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
