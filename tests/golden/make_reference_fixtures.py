"""Regenerate tests/golden/reference_fixtures.npz from the reference's own energy fixtures.

noci-rs tests its NOCI, NOCI-PT2 and selected-NOCI paths against energies stored in
``tests/fixtures/<NAME>/expected.json``; their integrals come from PySCF and their reference
determinants from the project's SCF, neither of which exists here.  For the fixtures whose
molecules carry only s functions (hydrogen chains in STO-3G and 3-21G) this script rebuilds
both from first principles:

* integrals over contracted s Gaussians in closed form (overlap, kinetic, nuclear attraction
  and electron repulsion with the Boys function F0), basis data of the published STO-3G and
  3-21G hydrogen sets, contracted functions normalised, coordinates in Bohr with
  1 Bohr = 0.52917721092 Angstrom;
* the states of each fixture's ``states.mom`` list as the reference builds them
  (src/basis/bias.rs): the density guess is half the RHF density per spin, each atom's AO
  block scaled by 1 +- pol following the spin or spatial bias pattern, then unrestricted SCF
  (Roothaan steps with DIIS) to 1e-13 Eh.

The SCF energies of every state must equal the fixture's ``scf_energies`` (sorted) to 1e-9 Eh,
which pins both the integrals and the states; the script refuses to write otherwise.  The
archive holds, per fixture, the AO data, the reference orbitals, the expected energies (of the
fixture and, where the reference has one, of its ``_WICKS`` twin, which runs the same input
through the Wick path) and the options of the fixture's input (excitation orders, snoci
block).  Tests read only the archive.

Run from the repository root with the reference checked out at /root/reference:
    python tests/golden/make_reference_fixtures.py
"""
import json
import os
from math import erf, exp, pi, sqrt

import numpy as np

REF = "/root/reference/tests/fixtures"
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.npz")
BOHR = 0.52917721092

STO3G_H = [[(3.42525091, 0.15432897), (0.62391373, 0.53532814), (0.16885540, 0.44463454)]]
B321G_H = [[(5.4471780, 0.1562850), (0.8245470, 0.9046910)], [(0.1831920, 1.0)]]
BASIS = {"STO-3G": STO3G_H, "3-21G": B321G_H}


def boys0(t):
    return 1.0 - t / 3.0 if t < 1e-12 else 0.5 * sqrt(pi / t) * erf(sqrt(t))


def contracted(shell):
    ex = np.array([a for a, _ in shell])
    c = np.array([d for _, d in shell]) * (2.0 * ex / pi) ** 0.75
    norm = sum(c[i] * c[j] * (pi / (ex[i] + ex[j])) ** 1.5 for i in range(len(ex)) for j in range(len(ex)))
    return ex, c / sqrt(norm)


def integrals(atoms_ang, basis):
    """(S, h, eri, E_nuc, AO indices per atom) for hydrogen atoms at the given positions."""
    centres = [np.array(a) / BOHR for a in atoms_ang]
    fns, atomao = [], []
    for ia, centre in enumerate(centres):
        atomao.append([])
        for shell in basis:
            atomao[-1].append(len(fns))
            fns.append((centre,) + contracted(shell))
    n = len(fns)
    s, t, v = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    for i, (a_c, a_e, a_k) in enumerate(fns):
        for j, (b_c, b_e, b_k) in enumerate(fns):
            ab2 = float(np.dot(a_c - b_c, a_c - b_c))
            for a, ka in zip(a_e, a_k):
                for b, kb in zip(b_e, b_k):
                    p, mu = a + b, a * b / (a + b)
                    pc = (a * a_c + b * b_c) / p
                    ov = (pi / p) ** 1.5 * exp(-mu * ab2)
                    s[i, j] += ka * kb * ov
                    t[i, j] += ka * kb * mu * (3.0 - 2.0 * mu * ab2) * ov
                    for c in centres:
                        v[i, j] -= ka * kb * 2.0 * pi / p * exp(-mu * ab2) * boys0(p * float(np.dot(pc - c, pc - c)))
    eri = np.zeros((n, n, n, n))
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if i * (i + 1) // 2 + j < k * (k + 1) // 2 + l:
                        continue
                    val = 0.0
                    (A, ea, ka_), (B, eb, kb_) = fns[i], fns[j]
                    (C, ec, kc_), (D, ed, kd_) = fns[k], fns[l]
                    for a, x1 in zip(ea, ka_):
                        for b, x2 in zip(eb, kb_):
                            p = a + b
                            P = (a * A + b * B) / p
                            kab = exp(-a * b / p * float(np.dot(A - B, A - B)))
                            for c, x3 in zip(ec, kc_):
                                for d, x4 in zip(ed, kd_):
                                    q = c + d
                                    Q = (c * C + d * D) / q
                                    kcd = exp(-c * d / q * float(np.dot(C - D, C - D)))
                                    val += (x1 * x2 * x3 * x4 * 2.0 * pi ** 2.5 / (p * q * sqrt(p + q)) * kab * kcd
                                            * boys0(p * q / (p + q) * float(np.dot(P - Q, P - Q))))
                    for (w, x, y, z) in ((i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k),
                                         (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i)):
                        eri[w, x, y, z] = val
    enuc = sum(1.0 / np.linalg.norm(centres[a] - centres[b]) for a in range(len(centres)) for b in range(a))
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


def states_for(s, h, eri, enuc, atomao, nelec, recipes):
    na = nb = nelec // 2
    e_rhf, ca, _ = uhf(s, h, eri, enuc, na, nb, *(2 * [np.zeros_like(s)]))
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


def chain(r, offsets):
    return [(0.0, 0.0, o * r) for o in offsets]


def square(a):
    h_ = a / 2
    return [(-h_, -h_, 0.0), (-h_, h_, 0.0), (h_, -h_, 0.0), (h_, h_, 0.0)]


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
GMRES_128 = {"gmres_max_iter": 128, "restart": 64, "res_tol": 1e-10}
GMRES_512 = {"gmres_max_iter": 512, "restart": 64, "res_tol": 1e-10}

# name: (basis, geometry, states, excitation orders, snoci block) -- from each input.lua
FIXTURES = {
    "REF_NOCI_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, None, None),
    "REF_NOCI_H4_STO-3G_1_75": ("STO-3G", square(1.75), H4_SQUARE_STATES, None, None),
    "PT2_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2), {"max_iter": 1, **GMRES_128}),
    "PT2_H2_3-21G_1_5": ("3-21G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2), {"max_iter": 1, **GMRES_128}),
    "SNOCI_H2_STO-3G_1_5": ("STO-3G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2),
                            {"max_iter": 5, "max_add": 1, **GMRES_128}),
    "SNOCI_H2_3-21G_1_5": ("3-21G", chain(1.5, (-0.5, 0.5)), H2_STATES, (1, 2),
                           {"max_iter": 5, "max_add": 1, **GMRES_128}),
    "SNOCI_H4_STO-3G_1_5": ("STO-3G", chain(1.5, (-1.5, -0.5, 0.5, 1.5)), H4_CHAIN_STATES, (2,),
                            {"max_iter": 2, "max_add": 1, **GMRES_512}),
}


def main():
    arrays, meta = {}, {}
    for name, (basis, geom, recipes, orders, snoci) in FIXTURES.items():
        with open(os.path.join(REF, name, "expected.json")) as f:
            expected = json.load(f)
        wicks_path = os.path.join(REF, name + "_WICKS", "expected.json")
        expected_wicks = None
        if os.path.exists(wicks_path):
            with open(wicks_path) as f:
                expected_wicks = json.load(f)
        s, h, eri, enuc, atomao = integrals(geom, BASIS[basis])
        nelec = len(geom)
        states = states_for(s, h, eri, enuc, atomao, nelec, recipes)
        energies = sorted(e for e, _, _ in states)
        ref = sorted(expected["scf_energies"])
        dev = max(abs(a - b) for a, b in zip(energies, ref))
        print(f"{name}: SCF energies {energies} vs {ref}: max dev {dev:.2e}")
        if dev > 1e-9:
            raise SystemExit(f"{name}: SCF states do not reproduce the fixture's SCF energies")
        arrays[f"{name}/s"] = s
        arrays[f"{name}/h"] = h
        arrays[f"{name}/eri"] = eri
        arrays[f"{name}/ca"] = np.stack([ca for _, ca, _ in states])
        arrays[f"{name}/cb"] = np.stack([cb for _, _, cb in states])
        meta[name] = {"basis": basis, "enuc": enuc, "nocc": nelec // 2, "labels": [r["label"] for r in recipes],
                      "scf_energies": [e for e, _, _ in states], "expected": expected,
                      "expected_wicks": expected_wicks,
                      "orders": list(orders) if orders else None, "snoci": snoci}
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
