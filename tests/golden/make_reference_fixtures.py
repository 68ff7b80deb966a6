"""Regenerate tests/golden/reference_fixtures.npz from the reference's own energy fixtures.

noci-rs tests its NOCI, NOCI-PT2 and selected-NOCI paths against energies stored in
``tests/fixtures/<NAME>/expected.json``; their integrals come from PySCF and their reference
determinants from the project's SCF, neither of which exists here.  For the fixtures whose
molecules carry only s and p functions this script rebuilds both from first principles:

* integrals over contracted cartesian s and p Gaussians by the McMurchie-Davidson scheme
  (Hermite expansion coefficients, Hermite Coulomb integrals over the Boys function), the
  basis data of PySCF's STO-3G, 3-21G and 6-31G files for H, Li and F, contracted functions
  normalised, coordinates in Bohr with 1 Bohr = 0.52917721092 Angstrom;
* the states of each fixture's ``states.mom`` list as the reference builds them
  (src/basis/bias.rs): the density guess is half the (lowest) RHF density per spin, each atom's AO
  block scaled by 1 +- pol following the spin or spatial bias pattern, then unrestricted SCF
  (Roothaan steps with DIIS) to 1e-13 Eh.

The SCF energies of every state must equal the fixture's ``scf_energies`` (sorted) to 1e-9 Eh,
which pins both the integrals and the states; the script refuses to write otherwise.  The
archive holds, per fixture, the AO data, the reference orbitals, the expected energies (of the
fixture and, where the reference has one, of its ``_WICKS`` twin, which runs the same input
through the Wick path) and the options of the fixture's input (excitation orders, snoci
block).  Tests read only the archive.

Run from the repository root, naming the reference checkout's fixture directory:
    python tests/golden/make_reference_fixtures.py <noci-rs checkout>/tests/fixtures
"""
import json
import os
from math import exp, pi, sqrt

import numpy as np
from scipy.special import gamma, gammainc

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.npz")
BOHR = 0.52917721092

# Shells per element: (angular momentum, exponents, contraction coefficients), as in PySCF's
# basis files (STO-3G: H and F; 3-21G: H; 6-31G: H and Li).
STO3G = {
    "H": [(0, [3.42525091, 0.62391373, 0.16885540], [0.15432897, 0.53532814, 0.44463454])],
    "F": [(0, [166.6791300, 30.3608120, 8.2168207], [0.15432897, 0.53532814, 0.44463454]),
          (0, [6.4648032, 1.5022812, 0.4885885], [-0.09996723, 0.39951283, 0.70011547]),
          (1, [6.4648032, 1.5022812, 0.4885885], [0.15591627, 0.60768372, 0.39195739])],
    "Li": [(0, [16.1195750, 2.9362007, 0.7946505], [0.15432897, 0.53532814, 0.44463454]),
           (0, [0.6362897, 0.1478601, 0.0480887], [-0.09996723, 0.39951283, 0.70011547]),
           (1, [0.6362897, 0.1478601, 0.0480887], [0.15591627, 0.60768372, 0.39195739])],
}
B321G = {"H": [(0, [5.4471780, 0.8245470], [0.1562850, 0.9046910]), (0, [0.1831920], [1.0])]}
B631G = {
    "H": [(0, [18.7311370, 2.8253937, 0.6401217], [0.03349460, 0.23472695, 0.81375733]),
          (0, [0.1612778], [1.0])],
    "Li": [(0, [642.4189200, 96.7985150, 22.0911210, 6.2010703, 1.9351177, 0.6367358],
            [0.0021426, 0.0162089, 0.0773156, 0.2457860, 0.4701890, 0.3454708]),
           (0, [2.3249184, 0.6324306, 0.0790534], [-0.0350917, -0.1912328, 1.0839878]),
           (1, [2.3249184, 0.6324306, 0.0790534], [0.0089415, 0.1410095, 0.9453637]),
           (0, [0.0359620], [1.0]), (1, [0.0359620], [1.0])],
}
BASIS = {"STO-3G": STO3G, "3-21G": B321G, "6-31G": B631G}
CHARGE = {"H": 1, "Li": 3, "F": 9}


def boys(n, t):
    """F_n(t) = int_0^1 u^(2n) exp(-t u^2) du, by the incomplete gamma function."""
    if t < 1e-12:
        return 1.0 / (2 * n + 1) - t / (2 * n + 3)
    return gamma(n + 0.5) * gammainc(n + 0.5, t) / (2.0 * t ** (n + 0.5))


def hermite_e(i, j, t, qx, a, b):
    """McMurchie-Davidson expansion coefficient E_t^{ij} of a 1-D Gaussian product."""
    p, mu = a + b, a * b / (a + b)
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return exp(-mu * qx * qx)
    if j == 0:
        return (hermite_e(i - 1, j, t - 1, qx, a, b) / (2 * p) - mu * qx / a * hermite_e(i - 1, j, t, qx, a, b)
                + (t + 1) * hermite_e(i - 1, j, t + 1, qx, a, b))
    return (hermite_e(i, j - 1, t - 1, qx, a, b) / (2 * p) + mu * qx / b * hermite_e(i, j - 1, t, qx, a, b)
            + (t + 1) * hermite_e(i, j - 1, t + 1, qx, a, b))


def hermite_r(t, u, v, n, p, pc):
    """Hermite Coulomb integral R^n_{tuv} for exponent p and separation vector pc."""
    if t == u == v == 0:
        return (-2.0 * p) ** n * boys(n, p * float(pc @ pc))
    if t == u == 0:
        r = pc[2] * hermite_r(t, u, v - 1, n + 1, p, pc)
        return r + ((v - 1) * hermite_r(t, u, v - 2, n + 1, p, pc) if v > 1 else 0.0)
    if t == 0:
        r = pc[1] * hermite_r(t, u - 1, v, n + 1, p, pc)
        return r + ((u - 1) * hermite_r(t, u - 2, v, n + 1, p, pc) if u > 1 else 0.0)
    r = pc[0] * hermite_r(t - 1, u, v, n + 1, p, pc)
    return r + ((t - 1) * hermite_r(t - 2, u, v, n + 1, p, pc) if t > 1 else 0.0)


def _e3(la, lb, A, B, a, b):
    return [[hermite_e(la[k], lb[k], t, A[k] - B[k], a, b) for t in range(la[k] + lb[k] + 1)] for k in range(3)]


def overlap_p(a, la, A, b, lb, B):
    e = _e3(la, lb, A, B, a, b)
    return e[0][0] * e[1][0] * e[2][0] * (pi / (a + b)) ** 1.5


def kinetic_p(a, la, A, b, lb, B):
    def ov(l):
        return overlap_p(a, la, A, b, l, B) if min(l) >= 0 else 0.0
    l, m, n = lb
    return (b * (2 * (l + m + n) + 3) * ov(lb)
            - 2 * b * b * (ov((l + 2, m, n)) + ov((l, m + 2, n)) + ov((l, m, n + 2)))
            - 0.5 * (l * (l - 1) * ov((l - 2, m, n)) + m * (m - 1) * ov((l, m - 2, n)) + n * (n - 1) * ov((l, m, n - 2))))


def nuclear_p(a, la, A, b, lb, B, C):
    p = a + b
    pc = (a * A + b * B) / p - C
    e = _e3(la, lb, A, B, a, b)
    v = 0.0
    for t, ex in enumerate(e[0]):
        for u, ey in enumerate(e[1]):
            for w, ez in enumerate(e[2]):
                v += ex * ey * ez * hermite_r(t, u, w, 0, p, pc)
    return 2 * pi / p * v


def eri_p(a, la, A, b, lb, B, c, lc, C, d, ld, D):
    p, q = a + b, c + d
    alpha = p * q / (p + q)
    pq = (a * A + b * B) / p - (c * C + d * D) / q
    e1, e2 = _e3(la, lb, A, B, a, b), _e3(lc, ld, C, D, c, d)
    v = 0.0
    for t, x1 in enumerate(e1[0]):
        for u, y1 in enumerate(e1[1]):
            for w, z1 in enumerate(e1[2]):
                f1 = x1 * y1 * z1
                if f1 == 0.0:
                    continue
                for t2, x2 in enumerate(e2[0]):
                    for u2, y2 in enumerate(e2[1]):
                        for w2, z2 in enumerate(e2[2]):
                            v += f1 * x2 * y2 * z2 * (-1) ** (t2 + u2 + w2) * hermite_r(t + t2, u + u2, w + w2, 0, alpha, pq)
    return 2 * pi ** 2.5 / (p * q * sqrt(p + q)) * v


def _prim_norm(a, l):
    def dfact(k):
        return 1 if k <= 0 else k * dfact(k - 2)
    return (2 * a / pi) ** 0.75 * (4 * a) ** (sum(l) / 2) / sqrt(dfact(2 * l[0] - 1) * dfact(2 * l[1] - 1) * dfact(2 * l[2] - 1))


def basis_functions(atoms, basis):
    """Contracted cartesian functions (centre, (lx, ly, lz), exponents, normalised coefficients)
    and the AO indices of each atom; p shells in the order x, y, z."""
    fns, atomao = [], []
    for el, centre in atoms:
        atomao.append([])
        for l, ex, co in basis[el]:
            for lv in ([(0, 0, 0)] if l == 0 else [(1, 0, 0), (0, 1, 0), (0, 0, 1)]):
                ex_ = np.array(ex, float)
                c = np.array(co, float) * np.array([_prim_norm(x, lv) for x in ex_])
                norm = sum(c[i] * c[j] * overlap_p(ex_[i], lv, centre, ex_[j], lv, centre)
                           for i in range(len(ex_)) for j in range(len(ex_)))
                atomao[-1].append(len(fns))
                fns.append((centre, lv, ex_, c / sqrt(norm)))
    return fns, atomao


def integrals(atoms_ang, basis):
    """(S, h, eri, E_nuc, AO indices per atom) for atoms [(element, (x, y, z) in Angstrom)]."""
    atoms = [(el, np.array(xyz, float) / BOHR) for el, xyz in atoms_ang]
    fns, atomao = basis_functions(atoms, basis)
    n = len(fns)
    s, t, v = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    for i, (A, la, ea, ca) in enumerate(fns):
        for j, (B, lb, eb, cb) in enumerate(fns):
            for a, xa in zip(ea, ca):
                for b, xb in zip(eb, cb):
                    s[i, j] += xa * xb * overlap_p(a, la, A, b, lb, B)
                    t[i, j] += xa * xb * kinetic_p(a, la, A, b, lb, B)
                    for el, C in atoms:
                        v[i, j] -= CHARGE[el] * xa * xb * nuclear_p(a, la, A, b, lb, B, C)
    eri = np.zeros((n, n, n, n))
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if i * (i + 1) // 2 + j < k * (k + 1) // 2 + l:
                        continue
                    (A, la, ea, ca), (B, lb, eb, cb) = fns[i], fns[j]
                    (C, lc, ec, cc), (D, ld, ed, cd) = fns[k], fns[l]
                    val = 0.0
                    for a, x1 in zip(ea, ca):
                        for b, x2 in zip(eb, cb):
                            for c, x3 in zip(ec, cc):
                                for d, x4 in zip(ed, cd):
                                    val += x1 * x2 * x3 * x4 * eri_p(a, la, A, b, lb, B, c, lc, C, d, ld, D)
                    for (w, x, y, z) in ((i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k),
                                         (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i)):
                        eri[w, x, y, z] = val
    enuc = sum(CHARGE[atoms[a][0]] * CHARGE[atoms[b][0]] / np.linalg.norm(atoms[a][1] - atoms[b][1])
               for a in range(len(atoms)) for b in range(a))
    return s, t + v, eri, enuc, atomao


def uhf(s, h, eri, enuc, na, nb, da, db, maxit=20000):
    """Unrestricted SCF from densities (da, db): Roothaan steps with DIIS on FDS - SDF."""
    w, u = np.linalg.eigh(s)
    x = u @ np.diag(w ** -0.5) @ u.T
    hist_f, hist_e = [], []
    e_old = None
    for _ in range(maxit):
        j = np.einsum("pqrs,rs->pq", eri, da + db)
        fa = h + j - np.einsum("prqs,rs->pq", eri, da)
        fb = h + j - np.einsum("prqs,rs->pq", eri, db)
        e = 0.5 * np.sum((da + db) * h) + 0.5 * np.sum(da * fa) + 0.5 * np.sum(db * fb) + enuc
        err = np.concatenate([(fa @ da @ s - s @ da @ fa).ravel(), (fb @ db @ s - s @ db @ fb).ravel()])
        if e_old is not None and abs(e - e_old) < 1e-15 and np.abs(err).max() < 1e-13:
            break
        e_old = e
        hist_f.append((fa, fb))
        hist_e.append(err)
        hist_f, hist_e = hist_f[-8:], hist_e[-8:]
        m = len(hist_e)
        if m > 1:
            bmat = -np.ones((m + 1, m + 1))
            bmat[m, m] = 0.0
            for a in range(m):
                for b in range(m):
                    bmat[a, b] = hist_e[a] @ hist_e[b]
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            coef = np.linalg.lstsq(bmat, rhs, rcond=None)[0][:m]
            fa = sum(c * f[0] for c, f in zip(coef, hist_f))
            fb = sum(c * f[1] for c, f in zip(coef, hist_f))
        ca = x @ np.linalg.eigh(x.T @ fa @ x)[1]
        cb = x @ np.linalg.eigh(x.T @ fb @ x)[1]
        da = ca[:, :na] @ ca[:, :na].T
        db = cb[:, :nb] @ cb[:, :nb].T
    j = np.einsum("pqrs,rs->pq", eri, da + db)
    fa = h + j - np.einsum("prqs,rs->pq", eri, da)
    fb = h + j - np.einsum("prqs,rs->pq", eri, db)
    ca = x @ np.linalg.eigh(x.T @ fa @ x)[1]
    cb = x @ np.linalg.eigh(x.T @ fb @ x)[1]
    e = 0.5 * np.sum((da + db) * h) + 0.5 * np.sum(da * fa) + 0.5 * np.sum(db * fb) + enuc
    return e, ca, cb


def scale_blocks(d, atomao, pattern, pol, sign):
    d = d.copy()
    for a, sg in enumerate(pattern):
        if sg == 0:
            continue
        f = 1.0 + pol if sg * sign > 0 else 1.0 - pol
        idx = atomao[a]
        d[np.ix_(idx, idx)] *= f
    return d


def lowest_rhf(s, h, eri, enuc, nocc):
    """The lowest RHF solution found from the core guess and from the core-guess solution's
    occupations with one occupied orbital swapped for the lowest virtual (a core guess can
    converge to an excited RHF determinant, e.g. F2 with its single virtual orbital)."""
    zero = np.zeros_like(s)
    best = uhf(s, h, eri, enuc, nocc, nocc, zero, zero)
    w, u = np.linalg.eigh(s)
    x = u @ np.diag(w ** -0.5) @ u.T
    d = best[1][:, :nocc] @ best[1][:, :nocc].T
    f = h + np.einsum("pqrs,rs->pq", eri, 2 * d) - np.einsum("prqs,rs->pq", eri, d)
    c = x @ np.linalg.eigh(x.T @ f @ x)[1]
    if nocc < s.shape[0]:
        for k in range(nocc):
            occ = [i for i in range(nocc + 1) if i != k]
            dg = c[:, occ] @ c[:, occ].T
            cand = uhf(s, h, eri, enuc, nocc, nocc, dg, dg)
            if cand[0] < best[0] - 1e-10:
                best = cand
    return best


def states_for(s, h, eri, enuc, atomao, nelec, recipes):
    na = nb = nelec // 2
    _, ca, _ = lowest_rhf(s, h, eri, enuc, na)
    dm = ca[:, :na] @ ca[:, :na].T * 2.0     # RHF density (both spins)
    out = []
    for rec in recipes:
        if "image_of" in rec:
            # the symmetry image of an earlier state: AO permutation of a point-group operation
            src, perm = rec["image_of"]
            p = np.zeros((len(perm), len(perm)))
            for i, j in enumerate(perm):
                p[j, i] = 1.0
            e, ca_, cb_ = out[src]
            out.append((e, p @ ca_, p @ cb_))
            continue
        da, db = 0.5 * dm, 0.5 * dm
        if "spin" in rec:
            pat, pol = rec["spin"]
            da = scale_blocks(da, atomao, pat, pol, +1)
            db = scale_blocks(db, atomao, pat, pol, -1)
        if "spatial" in rec:
            pat, pol = rec["spatial"]
            da = scale_blocks(da, atomao, pat, pol, +1)
            db = scale_blocks(db, atomao, pat, pol, +1)
        out.append(uhf(s, h, eri, enuc, na, nb, da, db))
    return out


def chain(r, offsets, elements=None):
    elements = elements or ["H"] * len(offsets)
    return [(el, (0.0, 0.0, o * r)) for el, o in zip(elements, offsets)]


def square(a):
    h_ = a / 2
    return [("H", (-h_, -h_, 0.0)), ("H", (-h_, h_, 0.0)), ("H", (h_, -h_, 0.0)), ("H", (h_, h_, 0.0))]


H2_STATES = [{"label": "RHF (0, 0)"}, {"label": "UHF (1, -1)", "spin": ((1, -1), 0.75)},
             {"label": "UHF (-1, 1)", "spin": ((-1, 1), 0.75)}]
H4_CHAIN_STATES = [{"label": "RHF (0, 0)"}, {"label": "UHF (1, -1)", "spin": ((1, -1, 1, -1), 0.75)},
                   {"label": "UHF (-1, 1)", "spin": ((-1, 1, -1, 1), 0.75)}]
# Square H4: the RHF HOMO pair is degenerate by symmetry.  The reference's two spatially biased
# RHF states start from PySCF's RHF density, whose choice inside the pair is not reproducible
# here; they converge to the two members (the occupied e orbital along x or along y), which
# map onto each other under the 90 degree rotation of the square (atoms 0->2, 1->0, 2->3, 3->1
# for the order of the input), so the second is built as the image of the first.
H4_SQUARE_STATES = [{"label": "RHF (1, 1, -1, -1)", "spatial": ((1, 1, -1, -1), 1e-2)},
                    {"label": "RHF (1, -1, 1, -1)", "image_of": (0, (2, 0, 3, 1))},
                    {"label": "UHF (1, 1, -1, -1)", "spin": ((1, 1, -1, -1), 0.75)},
                    {"label": "UHF (-1, -1, 1, 1)", "spin": ((-1, -1, 1, 1), 0.75)}]
LIH_STATES = [{"label": "RHF (0, 0)", "noci": False}, {"label": "UHF (1, -1)", "spin": ((1, -1), 0.75)},
              {"label": "UHF (-1, 1)", "spin": ((-1, 1), 0.75)}]
GMRES_128 = {"gmres_max_iter": 128, "restart": 64, "res_tol": 1e-10}
GMRES_512 = {"gmres_max_iter": 512, "restart": 64, "res_tol": 1e-10}

# name: (basis, geometry, states, excitation orders, snoci block) -- from each input.lua
FIXTURES = {
    "REF_NOCI_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, None, None),
    "REF_NOCI_H4_STO-3G_1_75": ("STO-3G", square(1.75), H4_SQUARE_STATES, None, None),
    "REF_NOCI_F2_STO-3G_1_75": ("STO-3G", chain(1.75, (-0.5, 0.5), ["F", "F"]), H2_STATES, None, None),
    "REF_NOCI_LiH_6-31G_2_8": ("6-31G", chain(2.8, (-0.5, 0.5), ["Li", "H"]), LIH_STATES, None, None),
    "DET_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2), None),
    "DET_F2_sto-3g_1_75": ("STO-3G", chain(1.75, (-0.5, 0.5), ["F", "F"]), H2_STATES, (1, 2), None),
    "PT2_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2), {"max_iter": 1, **GMRES_128}),
    "PT2_H2_3-21G_1_5": ("3-21G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2), {"max_iter": 1, **GMRES_128}),
    "SNOCI_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2),
                            {"max_iter": 5, "max_add": 1, **GMRES_128}),
    "SNOCI_H2_3-21G_1_5": ("3-21G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2),
                           {"max_iter": 5, "max_add": 1, **GMRES_128}),
    "SNOCI_H4_STO-3G_1_5": ("STO-3G", chain(1.5, (-1.5, -0.5, 0.5, 1.5)), H4_CHAIN_STATES, (2,),
                            {"max_iter": 2, "max_add": 1, **GMRES_512}),
    "QMC_LiH_STO-3G_2_8_TRAJECTORY_DDS2": ("STO-3G", chain(2.8, (-0.5, 0.5), ["Li", "H"]), LIH_STATES, (1, 2), None),
    "QMC_LiH_6-31G_2_8_TRAJECTORY_DDS2": ("6-31G", chain(2.8, (-0.5, 0.5), ["Li", "H"]), LIH_STATES, (1, 2), None),
    "QMC_LiH_STO-3G_2_8_TRAJECTORY_DIRECT_OVERLAP": ("STO-3G", chain(2.8, (-0.5, 0.5), ["Li", "H"]), LIH_STATES,
                                                     (1, 2), None),
    "QMC_LiH_6-31G_2_8_TRAJECTORY_DIRECT_OVERLAP": ("6-31G", chain(2.8, (-0.5, 0.5), ["Li", "H"]), LIH_STATES,
                                                    (1, 2), None),
}

# qmc / prop blocks of the QMC trajectory fixtures' inputs (their expected.json stores only
# trajectory bounds: an energy window, a minimum number of report energies, span and drop)
QMC_OPTIONS = {
    name: {"dt": dt, "propagator": prop, "initial_population": 200,
           "target_population": 500, "ncycles": 1, "nreports": 80, "sampling_cutoff": 1.0, "spawn_cutoff": 0.25,
           "excitation_gen": "uniform", "seed": 1}
    for name, prop, dt in (("QMC_LiH_STO-3G_2_8_TRAJECTORY_DDS2", "difference-doubly-shifted-u2", 1e-2),
                           ("QMC_LiH_6-31G_2_8_TRAJECTORY_DDS2", "difference-doubly-shifted-u2", 1e-3),
                           ("QMC_LiH_STO-3G_2_8_TRAJECTORY_DIRECT_OVERLAP", "direct-overlap", 1e-2),
                           ("QMC_LiH_6-31G_2_8_TRAJECTORY_DIRECT_OVERLAP", "direct-overlap", 1e-3))
}


def main(ref_dir: str):
    arrays, meta = {}, {}
    for name, (basis, geom, recipes, orders, snoci) in FIXTURES.items():
        with open(os.path.join(ref_dir, name, "expected.json")) as f:
            expected = json.load(f)
        wicks_path = os.path.join(ref_dir, name + "_WICKS", "expected.json")
        expected_wicks = None
        if os.path.exists(wicks_path):
            with open(wicks_path) as f:
                expected_wicks = json.load(f)
        s, h, eri, enuc, atomao = integrals(geom, BASIS[basis])
        nelec = sum(CHARGE[el] for el, _ in geom)
        states = states_for(s, h, eri, enuc, atomao, nelec, recipes)
        energies = sorted(e for e, _, _ in states)
        if "scf_energies" in expected:
            ref = sorted(expected["scf_energies"])
            dev = max(abs(a - b) for a, b in zip(energies, ref))
            print(f"{name}: SCF energies {energies} vs {ref}: max dev {dev:.2e}")
            if dev > 1e-9:
                raise SystemExit(f"{name}: SCF states do not reproduce the fixture's SCF energies")
        else:
            # trajectory fixtures store no SCF energies: the 6-31G one has the molecule and states
            # of REF_NOCI_LiH_6-31G_2_8 (pinned above); the STO-3G one is not pinned
            print(f"{name}: SCF energies {energies} (the fixture stores none)")
        arrays[f"{name}/s"] = s
        arrays[f"{name}/h"] = h
        arrays[f"{name}/eri"] = eri
        noci = [r.get("noci", True) for r in recipes]
        arrays[f"{name}/ca"] = np.stack([ca for (_, ca, _), k in zip(states, noci) if k])
        arrays[f"{name}/cb"] = np.stack([cb for (_, _, cb), k in zip(states, noci) if k])
        meta[name] = {"basis": basis, "enuc": enuc, "nocc": nelec // 2,
                      "labels": [r["label"] for r, k in zip(recipes, noci) if k],
                      "scf_energies": [e for e, _, _ in states], "expected": expected,
                      "expected_wicks": expected_wicks,
                      "orders": list(orders) if orders else None, "snoci": snoci,
                      "qmc": QMC_OPTIONS.get(name)}
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("fixtures", help="tests/fixtures directory of a noci-rs checkout")
    main(ap.parse_args().fixtures)
