"""CPU restatement of the NOCI-QMC signed-walker propagation of noci-rs (test and baseline
infrastructure only).

Follows qmc_step of src/stochastic/walkers.rs:101-441 for the uniform excitation generator:
per cycle sample_populations (FRI with the sampling cutoff, metric.rs:579-673), the diagonal
change (state.rs:653-667), ceil|n| uniform spawning attempts per occupied determinant
(state.rs:681-726), (H, S) of every canonicalised attempt through the Wick path
(resolve_batched_spawning, state.rs:537-615, here the oracle's C++ evaluator), FRI rounding of
the spawned amplitude with the spawn cutoff; after ncycles the accumulated change is added to
the populations and the shift is updated (update_shift, metric.rs:729-751).  The random numbers
are numpy's (the reference's SmallRng stream is not reproduced); comparisons are statistical.

The direct-overlap propagator (qmc_step of src/stochastic/metric.rs:766-1087) runs the same cycles
with no identity shift, starts from N_0 = S c_0 scaled to the initial 1-norm (init.rs:32-83) and
applies each report's accumulated change through the overlap, N += S Phi_c(Delta), with the update
cutoff c of fri_population_updates (metric.rs:701-718, :1030) -- so N stays in the range of S.
"""
from __future__ import annotations

import numpy as np

PROPAGATORS = {"unshifted": 0, "shifted": 1, "doubly-shifted": 2, "difference-doubly-shifted-u1": 3,
               "difference-doubly-shifted-u2": 4, "direct-overlap": 5}


def fri(x: np.ndarray, c: float, u: np.ndarray) -> np.ndarray:
    """Phi_c (fri, metric.rs:675-699), vectorised with uniforms u."""
    if c <= 0.0:
        return x.copy()
    ax = np.abs(x)
    small = (x != 0.0) & (ax < c)
    out = x.copy()
    out[small] = np.where(u[small] < ax[small] / c, np.copysign(c, x[small]), 0.0)
    return out


class OracleQmc:
    def __init__(self, orc, obasis, c0, ref_idx, dt, initial_population=100.0, target_population=1e5,
                 sampling_cutoff=0.0, spawn_cutoff=0.0, shift_damping=5e-4, initial_shift=0.0, ncycles=10,
                 propagator="unshifted", seed=1, nthreads=0, update_cutoff=0.0, overlap=None):
        self.orc, self.ob = orc, obasis
        self.n = obasis.shape[0]
        self.dt, self.target = dt, target_population
        self.c1, self.c2 = sampling_cutoff, spawn_cutoff
        self.damping, self.ncycles = shift_damping, ncycles
        self.prop = PROPAGATORS[propagator]
        self.shift = initial_shift
        self.nthreads = nthreads
        self.rng = np.random.default_rng(seed)
        g = np.arange(self.n)
        h, s = orc.eval_pairs(obasis, np.stack([g, g], 1), nthreads=nthreads)
        self.diag = np.stack([h, s], 1)
        self.refhs = np.zeros((self.n, 2))
        self.isref = np.zeros(self.n, bool)
        for i in ref_idx:
            self.isref[i] = True
            if c0[i] != 0.0:
                hi, si = orc.eval_pairs(obasis, np.stack([np.full(self.n, i), g], 1), nthreads=nthreads)
                self.refhs += c0[i] * np.stack([hi, si], 1)
        c0 = np.asarray(c0, float)
        self.c_update, self.overlap = update_cutoff, overlap
        if self.prop == 5:
            if overlap is None:
                raise ValueError("the direct-overlap propagator needs the overlap action S x")
            c0 = overlap(c0)
        self.pop = initial_population / np.abs(c0).sum() * c0
        self.nw_prev = np.abs(self.pop).sum()
        self.reached = False
        self.attempts = 0

    def identity_shift(self):
        return self.shift if self.prop in (1, 2) else 0.0

    def cycle_delta(self):
        """One cycle's population change from the current populations (not applied)."""
        n, rng = self.n, self.rng
        sampled = fri(self.pop, self.c1, rng.random(n))
        delta = -self.dt * (self.diag[:, 0] - self.shift * self.diag[:, 1] - self.identity_shift()) * sampled
        na = np.where(sampled != 0.0, np.maximum(1.0, np.ceil(np.abs(sampled))), 0.0).astype(np.int64)
        parents = np.repeat(np.arange(n), na)
        self.attempts += parents.size
        if parents.size:
            amp = sampled[parents] / na[parents]
            lam = rng.integers(0, n - 1, parents.size)
            lam += lam >= parents
            pairs = np.stack([np.minimum(lam, parents), np.maximum(lam, parents)], 1)
            h, s = self.orc.eval_pairs(self.ob, pairs, nthreads=self.nthreads)
            raw = -self.dt * (h - self.shift * s) * amp * (n - 1)
            dn = fri(raw, self.c2, rng.random(raw.size))
            np.add.at(delta, lam, dn)
        self.last_sampled = sampled
        return delta

    def report(self):
        """One report block: ncycles cycles, population update, statistics and shift."""
        self.attempts = 0
        delta = np.zeros(self.n)
        for _ in range(self.ncycles):
            delta += self.cycle_delta()
        if self.prop == 5:
            self.pop += self.overlap(fri(delta, self.c_update, self.rng.random(self.n)))
        else:
            self.pop += delta
        a = np.abs(self.pop)
        nw = a.sum()
        if not self.reached and nw >= self.target:
            self.reached = True
        if self.reached:
            self.shift -= (self.damping / (self.dt * self.ncycles)) * np.log(nw / self.nw_prev)
        self.nw_prev = nw
        return {"shift": self.shift, "eproj_num": float(self.pop @ self.refhs[:, 0]),
                "eproj_den": float(self.pop @ self.refhs[:, 1]), "nw": nw, "nref": a[self.isref].sum(),
                "nattempts": self.attempts}
