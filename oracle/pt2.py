"""CPU restatement of the NOCI-PT2 / SNOCI linear solve of noci-rs (test infrastructure only).

* projected operator  apply_omega_m + apply_projection_correction (src/snoci/operators.rs:696-955)
* preconditioners     Preconditioner::new / apply, Diag and Woodbury (src/snoci/types.rs:138-288)
* GMRES               gmres / run_arnoldi_cycle with two modified Gram-Schmidt passes, Givens
                      rotations, back substitution and true-residual restarts (src/snoci/gmres.rs)
for real states and no imaginary shift, on a dense M = F - E0 S.
"""
from __future__ import annotations

import numpy as np

SMALL = 1e-14


def apply_omega(m, p, x):
    """M^Omega x = M x - f_a0 (s_0a.x) - s_a0 (f_0a.x) + 2 E0 s_a0 (s_0a.x)."""
    sx, fx = p["s_0a"] @ x, p["f_0a"] @ x
    return m @ x - p["f_a0"] * sx - p["s_a0"] * fx + 2.0 * p["e0"] * p["s_a0"] * sx


def preconditioner(m_diag, p, kind):
    """apply(v) of the reference preconditioner ("diag" or "woodbury")."""
    if kind == "diag":
        d = m_diag - p["f_a0"] * p["s_0a"] - p["s_a0"] * p["f_0a"] + 2.0 * p["e0"] * p["s_a0"] * p["s_0a"]
    else:
        d = m_diag.copy()
    dmax = np.abs(d).max() if d.size else 0.0
    dfloor = max(1e-12 * dmax, 1e-14)
    dinv = np.where(np.abs(d) > dfloor, 1.0 / np.where(d == 0, 1.0, d), d / (dfloor * dfloor))
    if kind == "diag":
        return lambda v: v * dinv
    u0 = -p["f_a0"] + 2.0 * p["e0"] * p["s_a0"]
    u1 = -p["s_a0"]
    v0, v1 = p["s_0a"], p["f_0a"]
    z0, z1 = dinv * u0, dinv * u1
    c00, c01 = 1.0 + v0 @ z0, v0 @ z1
    c10, c11 = v1 @ z0, 1.0 + v1 @ z1
    det = c00 * c11 - c01 * c10
    if abs(det) <= 1e-14:
        return lambda v: v * dinv
    w00, w01, w10, w11 = c11 / det, -c01 / det, -c10 / det, c00 / det

    def apply(v):
        y = v * dinv
        t0, t1 = v0 @ y, v1 @ y
        return y - z0 * (w00 * t0 + w01 * t1) - z1 * (w10 * t0 + w11 * t1)
    return apply


def gmres(apply, precond, b, max_iter=100, restart=200, res_tol=1e-8):
    """Returns (x, residual_rms, iterations, converged)."""
    n = b.size
    x = np.zeros(n)
    rms = np.sqrt(n)
    r = b - apply(x)
    res = np.linalg.norm(r) / rms
    if res <= res_tol:
        return x, res, 0, True
    total = 0
    while total < max_iter:
        beta = np.linalg.norm(r)
        if beta <= SMALL:
            return x, beta / rms, total, beta / rms <= res_tol
        inner = min(restart, max_iter - total)
        q = [r / beta]
        h = np.zeros((inner + 1, inner))
        cs, sn = np.zeros(inner), np.zeros(inner)
        g = np.zeros(inner + 1)
        g[0] = beta
        kfinal = 0
        for k in range(inner):
            w = apply(precond(q[k]))
            for _ in range(2):
                for j in range(k + 1):
                    hjk = q[j] @ w
                    h[j, k] += hjk
                    w = w - hjk * q[j]
            hn = np.linalg.norm(w)
            h[k + 1, k] = hn
            if hn > SMALL:
                q.append(w / hn)
            for j in range(k):
                t = cs[j] * h[j, k] + sn[j] * h[j + 1, k]
                h[j + 1, k] = -sn[j] * h[j, k] + cs[j] * h[j + 1, k]
                h[j, k] = t
            a_, b_ = h[k, k], h[k + 1, k]
            den = np.hypot(a_, b_)
            cs[k], sn[k] = (a_ / den, b_ / den) if den > SMALL else (1.0, 0.0)
            h[k, k] = cs[k] * a_ + sn[k] * b_
            h[k + 1, k] = 0.0
            g[k + 1] = -sn[k] * g[k]
            g[k] = cs[k] * g[k]
            kfinal = k + 1
            if abs(g[k + 1]) / rms <= res_tol or hn <= SMALL:
                break
        y = np.zeros(kfinal)
        for i in range(kfinal - 1, -1, -1):
            s = g[i] - h[i, i + 1:kfinal] @ y[i + 1:kfinal]
            y[i] = s / h[i, i] if abs(h[i, i]) > SMALL else 0.0
        for j in range(kfinal):
            x = x + y[j] * precond(q[j])
        total += kfinal
        r = b - apply(x)
        res = np.linalg.norm(r) / rms
        if res <= res_tol:
            return x, res, total, True
    return x, res, total, res <= res_tol
