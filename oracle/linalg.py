"""CPU restatement of the generalised eigensolve of noci-rs (src/maths/linalg.rs:180-256).

Test infrastructure only: the GPU path (nw_general_evp) is checked against it.  numpy's eigh
calls LAPACK's symmetric eigensolver on the lower triangle, as ndarray-linalg's
``eigh_into(UPLO::Lower)`` does in the reference (hermitian_eigh, linalg.rs:283-292).
"""
from __future__ import annotations

import numpy as np


def hermitian_eigh(a: np.ndarray):
    """hermitian_eigh(a, UPLO::Lower): ascending eigenvalues, eigenvectors as columns."""
    return np.linalg.eigh(a, UPLO="L")


def positive_subspace(s: np.ndarray, tol: float):
    """positive_subspace (linalg.rs:180-201): eigenpairs of s with eigenvalue > tol."""
    lam, vec = hermitian_eigh(s)
    pos = lam > tol
    return lam[pos], vec[:, pos]


def loewdin_x(s: np.ndarray, project: bool, tol: float) -> np.ndarray:
    """loewdin_x (linalg.rs:203-228): U_+ diag(lambda_+^-1/2), or U diag(lambda^-1/2) U^T."""
    if project:
        vals, vecs = positive_subspace(s, tol)
        return vecs @ np.diag(1.0 / np.sqrt(vals))
    vals, vecs = hermitian_eigh(s)
    return vecs @ np.diag(1.0 / np.sqrt(vals)) @ vecs.T


def general_evp(h: np.ndarray, s: np.ndarray, project: bool, tol: float):
    """general_evp (linalg.rs:230-256): H C = S C e via X^T H X."""
    x = loewdin_x(s, project, tol)
    ht = x.T @ h @ x
    eps, u = hermitian_eigh(ht)
    return eps, x @ u
