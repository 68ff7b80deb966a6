"""Selected NOCI with NOCI-PT2 selection (snoci_step of noci-rs) on the B200 engine.

The host logic follows the reference step by step; every matrix element, the packed
candidate matrix M = F - E0 S, its mat-vec and GMRES run on the GPU through the C ABI:

* ``generate_excited_basis``  src/basis/excitation.rs:276-372 (labels, phases, parent-relative
  excitations of already excited determinants);
* ``CandidatePool``           src/snoci/candidate.rs:12-80;
* ``noci_density``            src/noci/naive.rs:231-276 with build_s_pair / pair_density
  (naive.rs:34-230): Loewdin-paired co-densities, the one-zero rule;
* ``fock``                    src/scf/kernels.rs:46-90;
* ``snoci_step``              src/snoci/step.rs:178-550 with solve_current_space,
  build_snoci_projection, build_candidate_v, build_omega_v and select_candidates
  (src/snoci/operators.rs:77-205, 991-1030, 1064-1083).

Determinant states are kept as a structured array (parent, alpha / beta occupation masks, the
total excitation masks from the parent reference, phase) plus a parallel list of labels.  A
label is the tuple (label of the generating state, total excitation masks), which compares
equal exactly when the reference's label strings ``"{generating label} {excitation}"`` do.

The optional learned screener (``LearnedScreen``, passed to ``snoci``) keeps only the
candidates an MLP ranks highest before M is built; the exhaustive screen stays the default and
the referee of its error.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from itertools import combinations
from typing import List, Optional, Sequence

import numpy as np

from .synthetic import NW_DET_DTYPE

STATE_DTYPE = np.dtype([("parent", "<u4"), ("oa", "<u8"), ("ob", "<u8"), ("ha", "<u8"), ("pa", "<u8"),
                        ("hb", "<u8"), ("pb", "<u8"), ("phase", "<f8")])
MAX_RANK = 4  # holes (and particles) per spin that an nw_det record holds


def _bits(mask: int) -> List[int]:
    return [i for i in range(64) if (mask >> i) & 1]


def _popcount(a: np.ndarray) -> np.ndarray:
    return np.bitwise_count(a.astype(np.uint64)).astype(np.int64)


def phase_bits(occ: np.ndarray, holes: np.ndarray, parts: np.ndarray, nmo: int) -> np.ndarray:
    """excitation_phase_bits (src/basis/excitation.rs:110-146), vectorised over masks: remove
    the holes from the highest down, then add the particles from the lowest up, counting the
    occupied orbitals below each; the last particle is counted but not added."""
    occ = occ.astype(np.uint64).copy()
    holes = holes.astype(np.uint64)
    parts = parts.astype(np.uint64)
    odd = np.zeros(occ.shape, np.int64)
    one = np.uint64(1)
    for b in range(nmo - 1, -1, -1):
        bit = one << np.uint64(b)
        sel = (holes & bit) != 0
        if sel.any():
            below = occ & (bit - one)
            odd ^= np.where(sel, _popcount(below) & 1, 0)
            occ = np.where(sel, occ & ~bit, occ)
    top = np.zeros(occ.shape, np.int64) - 1
    for b in range(nmo):
        top = np.where((parts >> np.uint64(b)) & one != 0, b, top)
    for b in range(nmo):
        bit = one << np.uint64(b)
        sel = (parts & bit) != 0
        if sel.any():
            below = occ & (bit - one)
            odd ^= np.where(sel, _popcount(below) & 1, 0)
            occ = np.where(sel & (top != b), occ | bit, occ)
    return np.where(odd & 1, -1.0, 1.0)


def _combo_masks(orbitals: Sequence[int], k: int) -> np.ndarray:
    """Masks of all k-subsets of `orbitals` in itertools (lexicographic) order."""
    if k == 0:
        return np.zeros(1, np.uint64)
    return np.array([sum(1 << o for o in c) for c in combinations(orbitals, k)], dtype=np.uint64)


def reference_states(nref: int, nocc_a: int, nocc_b: int):
    """The aufbau reference determinants (states, labels)."""
    st = np.zeros(nref, STATE_DTYPE)
    st["parent"] = np.arange(nref)
    st["oa"] = (1 << nocc_a) - 1
    st["ob"] = (1 << nocc_b) - 1
    st["phase"] = 1.0
    return st, [f"REF{r}" for r in range(nref)]


def generate_excited_basis(states: np.ndarray, labels: Sequence, nmo: int, orders: Sequence[int] = (1, 2),
                           include_refs: bool = False):
    """All excitations of the given orders on each state, expressed relative to the state's
    parent reference (generate_excited_basis, src/basis/excitation.rs:276-372)."""
    out, out_labels = [], []
    full = (1 << nmo) - 1
    for st, lab in zip(states, labels):
        oa, ob = int(st["oa"]), int(st["ob"])
        if include_refs:
            out.append(np.array([st], STATE_DTYPE))
            out_labels.append(lab)
        par_a = (oa & ~int(st["pa"])) | int(st["ha"])
        par_b = (ob & ~int(st["pb"])) | int(st["hb"])
        occ_a, vir_a = _bits(oa), _bits(full & ~oa)
        occ_b, vir_b = _bits(ob), _bits(full & ~ob)
        for k in sorted(set(orders)):
            for ka in range(k + 1):
                kb = k - ka
                if ka > len(occ_a) or ka > len(vir_a) or kb > len(occ_b) or kb > len(vir_b):
                    continue
                ha, pa = _combo_masks(occ_a, ka), _combo_masks(vir_a, ka)
                hb, pb = _combo_masks(occ_b, kb), _combo_masks(vir_b, kb)
                # loop order of the reference: alpha holes, alpha particles, beta holes, beta particles
                a_rem = np.repeat(ha, len(pa))
                a_add = np.tile(pa, len(ha))
                b_rem = np.repeat(hb, len(pb))
                b_add = np.tile(pb, len(hb))
                na, nb = len(a_rem), len(b_rem)
                new_a = (np.uint64(oa) & ~a_rem) | a_add
                new_b = (np.uint64(ob) & ~b_rem) | b_add
                blk = np.zeros(na * nb, STATE_DTYPE)
                blk["parent"] = st["parent"]
                blk["oa"] = np.repeat(new_a, nb)
                blk["ob"] = np.tile(new_b, na)
                pa_mask, pb_mask = np.uint64(par_a), np.uint64(par_b)
                blk["ha"] = pa_mask & ~blk["oa"]
                blk["pa"] = blk["oa"] & ~pa_mask
                blk["hb"] = pb_mask & ~blk["ob"]
                blk["pb"] = blk["ob"] & ~pb_mask
                ph_a = phase_bits(np.full(na, par_a, np.uint64), blk["ha"][::nb], blk["pa"][::nb], nmo)
                ph_b = phase_bits(np.full(nb, par_b, np.uint64), blk["hb"][:nb], blk["pb"][:nb], nmo)
                blk["phase"] = np.repeat(ph_a, nb) * np.tile(ph_b, na)
                out.append(blk)
                out_labels.extend((lab, int(x["ha"]), int(x["pa"]), int(x["hb"]), int(x["pb"])) for x in blk)
    if not out:
        return np.zeros(0, STATE_DTYPE), []
    return np.concatenate(out), out_labels


class CandidatePool:
    """Candidate determinants of the current selected space (src/snoci/candidate.rs)."""

    def __init__(self, selected: np.ndarray, labels: Sequence, nmo: int, orders: Sequence[int] = (1, 2)):
        self.nmo, self.orders = nmo, tuple(orders)
        self.states, self.labels = generate_excited_basis(selected, labels, nmo, orders, include_refs=False)

    def remove_selected(self, selected_labels: Sequence):
        drop = set(selected_labels)
        keep = np.array([lab not in drop for lab in self.labels], bool)
        self.states = self.states[keep]
        self.labels = [lab for lab, k in zip(self.labels, keep) if k]

    def update(self, selected_labels: Sequence, new_states: np.ndarray, new_labels: Sequence):
        if len(new_labels) == 0:
            return
        self.remove_selected(new_labels)
        cand, cand_labels = generate_excited_basis(new_states, new_labels, self.nmo, self.orders, include_refs=False)
        existing = set(selected_labels) | set(self.labels)
        keep = np.array([lab not in existing for lab in cand_labels], bool)
        self.states = np.concatenate([self.states, cand[keep]])
        self.labels += [lab for lab, k in zip(cand_labels, keep) if k]


def to_nw_dets(states: np.ndarray) -> np.ndarray:
    """nw_det records (parent, ranks, first four holes / particles ascending, phase)."""
    out = np.zeros(states.shape[0], NW_DET_DTYPE)
    out["parent"] = states["parent"]
    out["phase"] = states["phase"]
    for spin in ("a", "b"):
        h, p = states["h" + spin], states["p" + spin]
        rank = _popcount(h)
        if rank.size and (rank.max() > MAX_RANK or not np.array_equal(rank, _popcount(p))):
            raise ValueError("determinant with more than four holes per spin: beyond the nw_det record")
        idx = np.zeros((states.shape[0], 8), np.uint8)
        nh = np.zeros(states.shape[0], np.int64)
        npt = np.zeros(states.shape[0], np.int64)
        one = np.uint64(1)
        for b in range(64):
            hb = ((h >> np.uint64(b)) & one) != 0
            pb = ((p >> np.uint64(b)) & one) != 0
            if hb.any():
                r = np.nonzero(hb)[0]
                idx[r, nh[r]] = b
                nh[r] += 1
            if pb.any():
                r = np.nonzero(pb)[0]
                idx[r, 4 + npt[r]] = b
                npt[r] += 1
        out["rank_" + spin] = rank
        out["idx_" + spin] = idx
    return out


def _occ_columns(c: np.ndarray, mask: int) -> np.ndarray:
    return c[:, [i for i in range(c.shape[1]) if (mask >> i) & 1]]


def noci_density(system, states: np.ndarray, coeffs: np.ndarray, tol: float, phases: bool = True):
    """Alpha and beta AO densities of a NOCI state (noci_density, src/noci/naive.rs:231): per
    ordered pair of determinants (occupied columns in ascending order) the occupied overlap
    C_x^T S C_w = U s V^T is paired; with no zero singular value the co-density is
    phase * s_red * sum_i C_w v_i u_i^T C_x^T / s_i, with one zero it is
    phase * s_red * (C_w v_k)(C_x u_k)^T, with more it vanishes; the other spin enters through
    its full overlap.

    With ``phases`` (the reference, naive.rs:262) each pair is also weighted by the product of
    the two determinants' excitation phases.  The engine's matrix elements are between the
    canonically ordered determinants, so that is the density of sum_i phase_i c_i |Phi_i>;
    ``phases=False`` gives the density of sum_i c_i |Phi_i> itself.  Both agree while every
    selected determinant has phase +1 (the references, the first SNOCI iteration)."""
    n = system.s.shape[0]
    m = states.shape[0]
    occ = {"a": [], "b": []}
    for st in states:
        ca, _, cb, _ = system.refs[int(st["parent"])]
        occ["a"].append(_occ_columns(ca, int(st["oa"])))
        occ["b"].append(_occ_columns(cb, int(st["ob"])))
    ii, jj = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    res = {}
    for spin in ("a", "b"):
        cl = np.stack([occ[spin][i] for i in ii])          # bra x
        cg = np.stack([occ[spin][j] for j in jj])          # ket w
        sij = np.einsum("pmi,mn,pnj->pij", cl, system.s, cg)
        u, sv, vt = np.linalg.svd(sij)
        v = np.transpose(vt, (0, 2, 1))
        phase = np.linalg.det(u) * np.linalg.det(v)
        zero = np.abs(sv) <= tol
        nz = zero.sum(axis=1)
        s_red = np.prod(np.where(zero, 1.0, sv), axis=1)
        s_full = np.where(nz == 0, phase * np.prod(sv, axis=1), 0.0)
        lt = np.einsum("pmi,pij->pmj", cl, u)
        gt = np.einsum("pmi,pij->pmj", cg, v)
        w = np.where(zero, 0.0, 1.0 / np.where(zero, 1.0, sv))      # no zeros: 1 / s_i
        w = np.where((nz == 1)[:, None], zero.astype(float), w)     # one zero: that column only
        w = np.where((nz >= 2)[:, None], 0.0, w)
        res[spin] = (s_full, (phase * s_red)[:, None] * w, lt, gt)
    det_phase = states["phase"][ii] * states["phase"][jj] if phases else np.ones(ii.shape[0])
    cij = coeffs[ii] * coeffs[jj] * det_phase
    da = np.einsum("pmi,pi,pni->mn", res["a"][3], (cij * res["b"][0])[:, None] * res["a"][1], res["a"][2])
    db = np.einsum("pmi,pi,pni->mn", res["b"][3], (cij * res["a"][0])[:, None] * res["b"][1], res["b"][2])
    return da, db


def fock(h: np.ndarray, eri: np.ndarray, da: np.ndarray, db: np.ndarray):
    """F_s = h + J[D_a + D_b] - K[D_s] with J_pq = sum_rs D_rs (pq|rs), K_pq = sum_rs D_rs (pr|qs)
    (src/scf/kernels.rs:46-90)."""
    j = np.einsum("pqrs,rs->pq", eri, da + db)
    return h + j - np.einsum("prqs,rs->pq", eri, da), h + j - np.einsum("prqs,rs->pq", eri, db)


def select_candidates(scores: np.ndarray, sigma: float, max_add: int) -> np.ndarray:
    """Indices of the highest-scoring candidates above sigma, by decreasing score, stable for
    ties (select_candidates, src/snoci/operators.rs:1064-1083)."""
    idx = np.nonzero(scores > sigma)[0]
    order = idx[np.argsort(-scores[idx], kind="stable")]
    return order[:max_add]


@dataclass
class SnociOptions:
    """The snoci input block fields the step reads (src/input/snoci.rs)."""
    max_iter: int = 10
    max_dim: int = 100
    max_add: int = 10
    sigma: float = 1e-6
    tol: float = 1e-8               # |E_PT2| convergence
    lin_tol: float = 1e-8           # zero-overlap / projection tolerance
    orders: Sequence[int] = (1, 2)
    gmres_max_iter: int = 100
    gmres_restart: int = 30
    gmres_res_tol: float = 1e-8
    preconditioner: str = "woodbury"
    density_phases: bool = True     # reference density convention (see noci_density)
    keep_fraction: float = 0.25     # learned screener: share of the pool kept for PT2
    min_keep: int = 64
    audit: bool = False             # screened iterations also score the whole pool (the referee)
    packed_m_max_bytes: float = 120e9   # above this the candidate M is applied matrix-free


@dataclass
class SnociIteration:
    it: int
    nselected: int
    npool: int
    nscored: int
    ecurrent: float
    e0: float
    ept2: float
    gmres: dict
    selected: int
    seconds: float
    screened: bool
    recall: Optional[float] = None        # audit: exhaustive top picks found among the kept
    best_kept: Optional[bool] = None       # audit: the exhaustive best candidate was kept
    same_selection: Optional[bool] = None  # audit: the screened step selected the same set


@dataclass
class SnociResult:
    energy: float
    ept2: float
    coeffs: np.ndarray
    states: np.ndarray
    labels: list
    iterations: List[SnociIteration] = field(default_factory=list)
    stop: str = ""
    added: list = field(default_factory=list)   # labels selected by the last iteration


def solve_current_space(wicks, m: int, tol: float):
    """H, S over the first m resident determinants and the lowest GEVP root
    (solve_current_space, src/snoci/operators.rs:77-97)."""
    cur = np.arange(m, dtype=np.uint32)
    hcur, scur = wicks.build_hs_matrix(cur, cur)
    evals, cvecs = wicks.general_evp(hcur, scur, project=True, tol=tol)
    return float(evals[0]), cvecs[:, 0]


def pt2_scores(wicks, m: int, cand: np.ndarray, c: np.ndarray, ecurrent: float, opts: SnociOptions):
    """One NOCI-PT2 solve over the candidates `cand` (resident indices) against the current
    space (the first m resident determinants, coefficients c), after update_fock:
    E0 = c^T F c, the projection contractions s_a0 = S_ai c, f_a0 = F_ai c (real states, so the
    transposed contractions are equal), V^Omega = H_ai c - E_current s_a0, GMRES on
    M^Omega a = -V^Omega, E_PT2 = a.M^Omega a + 2 a.V^Omega and the scores |a_a V_a^Omega|
    (src/snoci/step.rs:265-441).  A candidate M larger than opts.packed_m_max_bytes is applied
    matrix-free (apply_candidate_m without a cached matrix).  Returns (scores, E_PT2, E0, GMRES
    info)."""
    cur = np.arange(m, dtype=np.uint32)
    cand = np.ascontiguousarray(cand, dtype=np.uint32)
    h_ai, s_ai = wicks.build_hs_matrix(cand, cur, symmetric=False)
    f_ii, _ = wicks.build_fs_matrix(cur, cur)
    f_ai, _ = wicks.build_fs_matrix(cand, cur, symmetric=False)
    e0 = float(c @ f_ii @ c)
    s_a0 = s_ai @ c
    f_a0 = f_ai @ c
    v_omega = h_ai @ c - ecurrent * s_a0
    matrix_free = 8.0 * cand.shape[0] * (cand.shape[0] + 1) / 2 > opts.packed_m_max_bytes
    with wicks.pt2(cand, e0, matrix_free=matrix_free) as pt:
        amp, info = pt.solve(e0, s_a0, s_a0, f_a0, f_a0, -v_omega, max_iter=opts.gmres_max_iter,
                             restart=opts.gmres_restart, res_tol=opts.gmres_res_tol,
                             preconditioner=opts.preconditioner)
        sx, fx = float(s_a0 @ amp), float(f_a0 @ amp)
        ma = pt.apply_m(amp) - f_a0 * sx - s_a0 * fx + 2.0 * e0 * s_a0 * sx
    ept2 = float(amp @ ma + 2.0 * (amp @ v_omega))
    return np.abs(amp * v_omega), ept2, e0, info


def snoci(wicks, system, opts: SnociOptions, screener=None, log=None) -> SnociResult:
    """Iterate snoci_step (src/snoci/step.rs:178-550) from the reference space.  ``wicks`` is a
    built WicksShared of the system's references; its resident basis is replaced each
    iteration by the selected space followed by the candidate pool.  ``log``, if given, is
    called with a short progress message at each stage."""
    say = log if log is not None else (lambda msg: None)
    nmo = system.nmo
    sel, sel_labels = reference_states(system.nref, system.nocc_a, system.nocc_b)
    pool: Optional[CandidatePool] = None
    result = None
    for it in range(opts.max_iter):
        t0 = time.perf_counter()
        if pool is None:
            pool = CandidatePool(sel, sel_labels, nmo, opts.orders)
        m = sel.shape[0]
        wicks.set_basis(to_nw_dets(np.concatenate([sel, pool.states])))
        ecurrent, c = solve_current_space(wicks, m, opts.lin_tol)
        if pool.states.shape[0] == 0:
            return SnociResult(ecurrent, 0.0, c, sel, sel_labels, [] if result is None else result.iterations,
                               "empty candidate pool")
        # generalised Fock of the current NOCI density
        da, db = noci_density(system, sel, c, opts.lin_tol, opts.density_phases)
        fa, fb = fock(system.h, system.eri, da, db)
        wicks.update_fock(fa, fb)
        npool = pool.states.shape[0]
        cand_all = np.arange(m, m + npool, dtype=np.uint32)
        screened = screener is not None and screener.ready
        if screened:
            keep = screener.keep(cand_all, opts, pool.states)
        else:
            keep = np.arange(npool)
        cand = cand_all[keep]
        say(f"iteration {it}: selected {m}, pool {npool}, scoring {cand.shape[0]}, E_current {ecurrent:.10f}, "
            f"{time.perf_counter() - t0:.1f} s")
        kept_scores, ept2, e0, info = pt2_scores(wicks, m, cand, c, ecurrent, opts)
        say(f"iteration {it}: E_PT2 {ept2:.10f}, GMRES {info}, {time.perf_counter() - t0:.1f} s")
        scores = np.zeros(npool)
        scores[keep] = kept_scores
        if screener is not None:
            screener.learn(cand, kept_scores, pool.states[keep])
        remaining = max(opts.max_dim - m, 0)
        chosen = select_candidates(scores, opts.sigma, min(opts.max_add, remaining)) if remaining else np.zeros(0, int)
        seconds = time.perf_counter() - t0
        recall = best = same = None
        if screened and opts.audit:
            exact, _, _, _ = pt2_scores(wicks, m, cand_all, c, ecurrent, opts)
            top = select_candidates(exact, opts.sigma, min(opts.max_add, remaining)) if remaining else chosen
            recall = float(np.isin(top, keep).mean()) if top.size else 1.0
            best = bool(np.isin(top[:1], keep).all())
            same = set(top.tolist()) == set(chosen.tolist())
        rec = SnociIteration(it, m, npool, int(cand.shape[0]), ecurrent, e0, ept2, info, int(chosen.shape[0]),
                             seconds, screened, recall, best, same)
        result = SnociResult(ecurrent, ept2, c, sel, sel_labels,
                             ([] if result is None else result.iterations) + [rec],
                             added=[pool.labels[i] for i in chosen])
        if remaining == 0:
            result.stop = "max_dim"
            return result
        if chosen.shape[0] == 0:
            result.stop = "sigma"
            return result
        if abs(ept2) < opts.tol:
            result.stop = "tol"
            return result
        new_states = pool.states[chosen]
        new_labels = [pool.labels[i] for i in chosen]
        sel = np.concatenate([sel, new_states])
        sel_labels = sel_labels + new_labels
        pool.update(sel_labels, new_states, new_labels)
    # maximum iteration reached: the state of the last iteration (its current-space energy,
    # before that iteration's selections), as snoci_step returns final_state (step.rs:525-549)
    if result is not None:
        result.stop = "max_iter"
        return result
    wicks.set_basis(to_nw_dets(sel))
    energy, c = solve_current_space(wicks, sel.shape[0], opts.lin_tol)
    return SnociResult(energy, 0.0, c, sel, sel_labels, [], "max_iter")


def _excitation_class(states: np.ndarray) -> np.ndarray:
    """(parent, rank_a, rank_b) of each state as one integer."""
    return (states["parent"].astype(np.int64) * 64 + _popcount(states["ha"]) * 8 + _popcount(states["hb"]))


class LearnedScreen:
    """Learned screening policy for ``snoci``: the first iteration scores the whole pool
    (exhaustive) and trains the GPU screener (``lib.Screen``) on log10 of the scores; later
    iterations score exactly (M and GMRES) only
      * candidates of every excitation class (parent, rank_a, rank_b) with fewer than
        ``min_class`` exactly scored examples so far -- all of them, or a seeded random
        ``explore_per_class`` of a large class (new classes appear as the selected space grows:
        excitations of selected determinants reach triples and quadruples), and
      * the candidates the screener ranks highest, up to ``keep_fraction`` of the pool (at
        least ``min_keep``),
    and fine-tune the screener on them.  Selection still uses the exact scores."""

    def __init__(self, wicks, epochs: int = 40, finetune_epochs: int = 10, batch: int = 1024, lr: float = 2e-3,
                 floor: float = 1e-14, seed: int = 17, min_class: int = 32, explore_per_class: int = 256):
        from .lib import Screen
        self.net = Screen(wicks, seed)
        self.epochs, self.finetune_epochs, self.batch, self.lr, self.floor = epochs, finetune_epochs, batch, lr, floor
        self.min_class = min_class
        self.explore_per_class = explore_per_class
        self.rng = np.random.default_rng(seed)
        self.clip: Optional[float] = None   # targets below the first set's median are clipped to it
        self.seen: dict = {}
        self.ready = False
        self.reports: List[dict] = []

    def keep(self, cand_all: np.ndarray, opts: SnociOptions, states: np.ndarray) -> np.ndarray:
        cls = _excitation_class(states)
        explore = np.zeros(cls.shape[0], bool)
        for c in np.unique(cls):
            if self.seen.get(int(c), 0) >= self.min_class:
                continue
            members = np.nonzero(cls == c)[0]
            if members.shape[0] > self.explore_per_class:
                members = self.rng.choice(members, self.explore_per_class, replace=False)
            explore[members] = True
        pred = self.net.predict(cand_all)
        pred[explore] = np.inf
        nkeep = min(cand_all.shape[0], max(opts.min_keep, int(np.ceil(opts.keep_fraction * cand_all.shape[0]))))
        nkeep = max(nkeep, int(explore.sum()))
        return np.sort(np.argsort(-pred, kind="stable")[:nkeep])

    def learn(self, cand: np.ndarray, scores: np.ndarray, states: np.ndarray):
        for c, k in zip(*np.unique(_excitation_class(states), return_counts=True)):
            self.seen[int(c)] = self.seen.get(int(c), 0) + int(k)
        target = np.log10(np.maximum(scores, self.floor))
        if self.clip is None:
            self.clip = float(np.median(target))
        # only the ranking of the upper half matters for selection: the negligible tail is
        # flattened so the fit spends its capacity there
        target = np.maximum(target, self.clip)
        rep = self.net.train(cand, target, epochs=self.finetune_epochs if self.ready else self.epochs,
                             batch=min(self.batch, max(1, cand.shape[0])), lr=self.lr, seed=len(self.reports) + 1)
        self.reports.append(rep)
        self.ready = True

    def close(self):
        self.net.close()
