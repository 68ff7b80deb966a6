"""CPU checks of the NOCI-PT2 restatement (oracle/pt2.py): the Woodbury preconditioner is the
exact inverse of diag(M) plus the rank-2 projection terms (Preconditioner::new/apply,
src/snoci/types.rs:161-288), and GMRES (src/snoci/gmres.rs) reaches the dense solution."""
import numpy as np

from oracle import pt2 as PT


def _problem(n=60, seed=0):
    rng = np.random.default_rng(seed)
    a = rng.normal(0, 0.1, (n, n))
    m = 0.5 * (a + a.T) + np.diag(rng.uniform(1.0, 3.0, n))
    p = {"e0": -1.3, "s_a0": rng.normal(0, 0.1, n), "f_a0": rng.normal(0, 0.1, n)}
    p["s_0a"], p["f_0a"] = p["s_a0"].copy(), p["f_a0"].copy()
    return m, p, rng.normal(0, 1, n)


def test_woodbury_is_exact_inverse_of_diagonal_plus_projection():
    m, p, v = _problem()
    d = np.diag(np.diag(m))
    u0 = -p["f_a0"] + 2 * p["e0"] * p["s_a0"]
    u1 = -p["s_a0"]
    full = d + np.outer(u0, p["s_0a"]) + np.outer(u1, p["f_0a"])
    pre = PT.preconditioner(np.diag(m), p, "woodbury")
    assert np.allclose(pre(v), np.linalg.solve(full, v), atol=1e-12)
    # the projected operator is M plus the same rank-2 terms
    a = np.array([PT.apply_omega(m, p, e) for e in np.eye(m.shape[0])]).T
    assert np.allclose(a, m + np.outer(u0, p["s_0a"]) + np.outer(u1, p["f_0a"]), atol=1e-13)


def test_gmres_reaches_dense_solution():
    m, p, b = _problem(seed=3)
    a = np.array([PT.apply_omega(m, p, e) for e in np.eye(m.shape[0])]).T
    for kind in ("woodbury", "diag"):
        pre = PT.preconditioner(np.diag(m), p, kind)
        x, res, it, conv = PT.gmres(lambda z: PT.apply_omega(m, p, z), pre, b, max_iter=100, restart=7, res_tol=1e-12)
        assert conv and res <= 1e-12
        assert np.allclose(x, np.linalg.solve(a, b), atol=1e-10)
