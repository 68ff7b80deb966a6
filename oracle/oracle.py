"""CPU oracle (test infrastructure only): Python driver for the FP64 restatement of noci-rs.

Packs the per-reference-pair intermediates built by ``wick_build`` into the slab orders of
src/nonorthogonalwicks/layout.rs and calls the C++ evaluators of ``wick_eval.cpp`` through
ctypes.  Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py may
use this module; the product library under noci-rs_b200/ never imports or links it.

Parity status: pinned against reference-produced numbers.  The reference's own energy
fixtures (tests/fixtures/*/expected.json of noci-rs: reference-space NOCI, deterministic
SD-space, NOCI-PT2 and selected-NOCI energies of H2, H4, LiH and F2) are reproduced from
integrals and SCF states rebuilt by tests/golden/make_reference_fixtures.py
(tests/test_reference_fixtures.py); the oracle is also cross-checked against an independent
generalised Slater-Condon path and a brute-force Fock-space evaluation.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import naive as _naive
from . import wick_build as _wb

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libwick_oracle.so")
_lib = None

KMAXL = 8
ORACLE_DET_DTYPE = np.dtype({
    "names": ["parent", "rank_a", "rank_b", "holes_a", "parts_a", "holes_b", "parts_b",
              "occ_a", "occ_b", "pha", "phb"],
    "formats": ["<i4", "<i4", "<i4", ("u1", (KMAXL,)), ("u1", (KMAXL,)), ("u1", (KMAXL,)),
                ("u1", (KMAXL,)), ("<u8", (2,)), ("<u8", (2,)), "<f8", "<f8"],
    "offsets": [0, 4, 8, 12, 20, 28, 36, 48, 64, 80, 88],
    "itemsize": 96,
})


def build_lib() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build_lib()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        i64p = ctypes.POINTER(ctypes.c_int64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.orc_layout.argtypes = [ctypes.c_int]
        L.orc_layout.restype = ctypes.c_int
        L.orc_eval_pairs.argtypes = [dp, i64p, dp, i32p, ctypes.c_int, ctypes.c_void_p, i64p,
                                     ctypes.c_int64, ctypes.c_double, ctypes.c_double, i64p, i32p,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_eval_pairs.restype = ctypes.c_int
        L.orc_eval_pairs_binned.argtypes = [dp, i64p, dp, i32p, ctypes.c_int, ctypes.c_void_p, i64p,
                                            ctypes.c_int64, ctypes.c_double, ctypes.c_double, i64p, i32p,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_eval_pairs_binned.restype = ctypes.c_int
        L.orc_eval_wick.argtypes = [dp, i64p, dp, i32p, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_int64, ctypes.c_int64, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, dp, dp]
        L.orc_eval_wick.restype = ctypes.c_int
        L.orc_eval_overlap.argtypes = [dp, i64p, dp, i32p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_int64, ctypes.c_int64, dp]
        L.orc_eval_overlap.restype = ctypes.c_int
        L.orc_eval_m_pairs.argtypes = [dp, i64p, dp, i32p, ctypes.c_int, ctypes.c_void_p, i64p, ctypes.c_int64,
                                       dp, i64p, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp, dp]
        L.orc_eval_m_pairs.restype = ctypes.c_int
        assert L.orc_layout(3) == ORACLE_DET_DTYPE.itemsize, "oracle Det layout mismatch"
        _lib = L
    return _lib


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class _SlabWriter:
    def __init__(self):
        self.chunks: List[np.ndarray] = []
        self.size = 0

    def put(self, arr: Optional[np.ndarray]) -> int:
        if arr is None:
            return -1
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        off = self.size
        self.chunks.append(a)
        self.size += a.size
        return off

    def finish(self) -> np.ndarray:
        if not self.chunks:
            return np.zeros(1)
        return np.concatenate(self.chunks)


def pack_pairs(builds: Sequence[_wb.PairBuild], nmo: int, writer: Optional[_SlabWriter] = None):
    """Pack pair builds into (slab, offs, vals, ints) in the reference storage orders."""
    lay = lib()
    noff, nval, nint = lay.orc_layout(0), lay.orc_layout(1), lay.orc_layout(2)
    w = writer or _SlabWriter()
    npair = len(builds)
    offs = np.full((npair, noff), -1, np.int64)
    vals = np.zeros((npair, nval))
    ints = np.zeros((npair, nint), np.int32)
    for p, b in enumerate(builds):
        ints[p, 4] = nmo
        if b is None:  # not built (Oracle.create with only_pairs): offsets stay -1
            continue
        k = 0
        for s, (ss, hcol0) in enumerate(((b.aa, b.hcol0_a), (b.bb, b.hcol0_b))):
            for i in range(2):
                offs[p, k] = w.put(ss.x[i]); k += 1
            for i in range(2):
                offs[p, k] = w.put(ss.y[i]); k += 1
            for i in range(2):
                for j in range(2):
                    offs[p, k] = w.put(ss.fh[i][j].T); k += 1
            for i in range(2):
                for j in range(2):
                    for l in range(2):
                        offs[p, k] = w.put(ss.v[i][j][l].T); k += 1
            offs[p, k] = w.put(None if hcol0 is None else hcol0.T); k += 1
            for slot in range(10):
                t = ss.j.get(slot)
                offs[p, k] = w.put(None if t is None else t.transpose(2, 3, 0, 1)); k += 1
            v = vals[p, s * 7:(s + 1) * 7]
            v[0] = ss.phase
            v[1] = ss.tilde_s_prod
            v[2:4] = ss.f0h
            v[4:7] = ss.v0
            ints[p, 2 * s] = ss.m
            ints[p, 2 * s + 1] = ss.nocc
        for a in range(2):
            for bb in range(2):
                for c in range(2):
                    offs[p, k] = w.put(b.ab.vab[a][bb][c].T); k += 1
        for a in range(2):
            for bb in range(2):
                for c in range(2):
                    offs[p, k] = w.put(b.ab.vba[a][bb][c].T); k += 1
        for a in range(2):
            for bb in range(2):
                for c in range(2):
                    for d in range(2):
                        offs[p, k] = w.put(b.ab.ii.get((a, bb, c, d))); k += 1
        vals[p, 14:18] = np.array(b.ab.vab0).ravel()
        vals[p, 18:22] = np.array(b.ab.vba0).ravel()
    return w, offs, vals, ints


def to_oracle_dets(basis: np.ndarray, ref_occs: Sequence[Tuple[int, int]]) -> np.ndarray:
    """Convert nw_det records (ranks <= 4) into the oracle's determinant records."""
    n = basis.shape[0]
    out = np.zeros(n, ORACLE_DET_DTYPE)
    out["parent"] = basis["parent"].astype(np.int32)
    ra = basis["rank_a"].astype(np.int32)
    rb = basis["rank_b"].astype(np.int32)
    out["rank_a"] = ra
    out["rank_b"] = rb
    out["holes_a"][:, :4] = basis["idx_a"][:, :4]
    out["parts_a"][:, :4] = basis["idx_a"][:, 4:]
    out["holes_b"][:, :4] = basis["idx_b"][:, :4]
    out["parts_b"][:, :4] = basis["idx_b"][:, 4:]
    for k in range(4):
        for col in ("holes_a", "parts_a"):
            out[col][ra <= k, k] = 0
        for col in ("holes_b", "parts_b"):
            out[col][rb <= k, k] = 0
    # occupation masks: parent occupation with holes removed and particles added
    occ = np.array([[oa, ob] for (oa, ob) in ref_occs], dtype=object)
    par = out["parent"]
    for spin, (rk, hcol, pcol, field) in enumerate(((ra, "holes_a", "parts_a", "occ_a"),
                                                    (rb, "holes_b", "parts_b", "occ_b"))):
        lo = np.array([int(occ[p][spin]) & 0xFFFFFFFFFFFFFFFF for p in range(len(ref_occs))],
                      dtype=np.uint64)[par]
        hi = np.array([int(occ[p][spin]) >> 64 for p in range(len(ref_occs))], dtype=np.uint64)[par]
        for k in range(4):
            has = rk > k
            hidx = out[hcol][:, k].astype(np.uint64)
            pidx = out[pcol][:, k].astype(np.uint64)
            one = np.uint64(1)
            hl = np.where(has & (hidx < 64), one << (hidx % np.uint64(64)), np.uint64(0))
            hh = np.where(has & (hidx >= 64), one << (hidx % np.uint64(64)), np.uint64(0))
            pl = np.where(has & (pidx < 64), one << (pidx % np.uint64(64)), np.uint64(0))
            ph = np.where(has & (pidx >= 64), one << (pidx % np.uint64(64)), np.uint64(0))
            lo = (lo & ~hl) | pl
            hi = (hi & ~hh) | ph
        out[field][:, 0] = lo
        out[field][:, 1] = hi
    # The nw_det record stores the product of both spin phases; the oracle keeps it in pha.
    out["pha"] = basis["phase"]
    out["phb"] = 1.0
    return out


@dataclass
class Oracle:
    """FP64 oracle for one system: AO data, references, and all nref^2 pair intermediates."""

    s: np.ndarray
    h: np.ndarray
    eri: np.ndarray
    enuc: float
    refs: list
    tol: float
    builds: list
    slab: np.ndarray
    offs: np.ndarray
    vals: np.ndarray
    ints: np.ndarray
    mo_offs: Optional[np.ndarray]
    mo_orth: Optional[np.ndarray]
    nmo: int

    @classmethod
    def from_system(cls, sysm, tol: float = 1e-8, with_mo_cache: bool = True, null_gauge=None,
                    only_pairs=None):
        return cls.create(sysm.s, sysm.h, sysm.eri, sysm.enuc, sysm.refs, tol, with_mo_cache,
                          null_gauge, only_pairs)

    @classmethod
    def create(cls, s, h, eri, enuc, refs, tol=1e-8, with_mo_cache=True, null_gauge=None,
               only_pairs=None):
        """With ``only_pairs`` (ordered-pair indices x * nref + w) only those reference pairs
        are built; requests may then only name determinants of those parent pairs."""
        builds = _wb.build_all(s, h, eri, refs, tol, null_gauge, only=only_pairs)
        nmo = refs[0][0].shape[1]
        w, offs, vals, ints = pack_pairs(builds, nmo)
        mo_offs = mo_orth = None
        if with_mo_cache:
            asym = _naive.antisymmetrise(eri)
            mo_offs = np.zeros((len(refs), 5), np.int64)
            mo_orth = np.zeros(len(refs), np.int32)
            for i, (ca, _, cb, _) in enumerate(refs):
                c = _naive.build_mo_cache(s, h, eri, asym, ca, cb, tol)
                mo_offs[i] = [w.put(c.ha), w.put(c.hb), w.put(c.eri_aa_asym), w.put(c.eri_bb_asym),
                              w.put(c.eri_ab_coul)]
                mo_orth[i] = 1 if c.orthogonal else 0
        slab = w.finish()
        return cls(s=s, h=h, eri=eri, enuc=enuc, refs=refs, tol=tol, builds=builds, slab=slab,
                   offs=offs, vals=vals, ints=ints, mo_offs=mo_offs, mo_orth=mo_orth, nmo=nmo)

    @property
    def nref(self) -> int:
        return len(self.refs)

    def ref_occs(self):
        return [(r[1], r[3]) for r in self.refs]

    def oracle_basis(self, basis: np.ndarray) -> np.ndarray:
        return to_oracle_dets(basis, self.ref_occs())

    def eval_pairs(self, obasis: np.ndarray, pairs: np.ndarray, nthreads: int = 0,
                   exact: bool = False):
        """(H, S) for pairs, with the same-parent dispatch of calculate_hs_pairs_wicks_batched."""
        L = lib()
        pairs = np.ascontiguousarray(pairs, dtype=np.int64)
        n = pairs.shape[0]
        h = np.empty(n)
        s = np.empty(n)
        mo_offs = self.mo_offs if self.mo_offs is not None else np.zeros(1, np.int64)
        mo_orth = self.mo_orth if self.mo_orth is not None else np.zeros(1, np.int32)
        L.orc_eval_pairs(_ptr(self.slab, ctypes.c_double), _ptr(self.offs, ctypes.c_int64),
                         _ptr(self.vals, ctypes.c_double), _ptr(self.ints, ctypes.c_int32),
                         self.nref, obasis.ctypes.data_as(ctypes.c_void_p),
                         _ptr(pairs, ctypes.c_int64), n, self.enuc, self.tol,
                         _ptr(mo_offs, ctypes.c_int64) if self.mo_offs is not None else None,
                         _ptr(mo_orth, ctypes.c_int32) if self.mo_orth is not None else None,
                         self.nmo, nthreads, 1 if exact else 0, _ptr(h, ctypes.c_double),
                         _ptr(s, ctypes.c_double))
        return h, s

    def eval_pairs_binned(self, obasis: np.ndarray, pairs: np.ndarray, nthreads: int = 0, lanes: int = 0,
                          exact: bool = False):
        """(H, S) for pairs by the reference's own CPU path: dynamic chunks of requests over the
        threads, each through calculate_hs_pairs_wicks_batched with the 28 (L_alpha, L_beta)
        bins flushed through lane-batched fixed-rank kernels (8 lanes AVX-512, 4 lanes AVX2;
        lanes = 0 picks the widest the host has).  Returns (h, s, lanes used)."""
        L = lib()
        pairs = np.ascontiguousarray(pairs, dtype=np.int64)
        n = pairs.shape[0]
        h = np.empty(n)
        s = np.empty(n)
        mo_offs = self.mo_offs if self.mo_offs is not None else np.zeros(1, np.int64)
        mo_orth = self.mo_orth if self.mo_orth is not None else np.zeros(1, np.int32)
        used = L.orc_eval_pairs_binned(
            _ptr(self.slab, ctypes.c_double), _ptr(self.offs, ctypes.c_int64), _ptr(self.vals, ctypes.c_double),
            _ptr(self.ints, ctypes.c_int32), self.nref, obasis.ctypes.data_as(ctypes.c_void_p),
            _ptr(pairs, ctypes.c_int64), n, self.enuc, self.tol,
            _ptr(mo_offs, ctypes.c_int64) if self.mo_offs is not None else None,
            _ptr(mo_orth, ctypes.c_int32) if self.mo_orth is not None else None,
            self.nmo, nthreads, 1 if exact else 0, lanes, _ptr(h, ctypes.c_double), _ptr(s, ctypes.c_double))
        if used < 0:
            raise RuntimeError(f"lane-batched CPU path: {lanes} lanes not supported on this host")
        return h, s, used

    def eval_wick(self, obasis: np.ndarray, a: int, b: int, exact: bool = False):
        L = lib()
        h = ctypes.c_double()
        s = ctypes.c_double()
        L.orc_eval_wick(_ptr(self.slab, ctypes.c_double), _ptr(self.offs, ctypes.c_int64),
                        _ptr(self.vals, ctypes.c_double), _ptr(self.ints, ctypes.c_int32),
                        self.nref, obasis.ctypes.data_as(ctypes.c_void_p), a, b, self.enuc,
                        self.tol, 1 if exact else 0, ctypes.byref(h), ctypes.byref(s))
        return h.value, s.value

    def eval_overlap(self, obasis: np.ndarray, a: int, b: int) -> float:
        L = lib()
        s = ctypes.c_double()
        L.orc_eval_overlap(_ptr(self.slab, ctypes.c_double), _ptr(self.offs, ctypes.c_int64),
                           _ptr(self.vals, ctypes.c_double), _ptr(self.ints, ctypes.c_int32),
                           self.nref, obasis.ctypes.data_as(ctypes.c_void_p), a, b,
                           ctypes.byref(s))
        return s.value

    def set_fock(self, fa: np.ndarray, fb: np.ndarray):
        """update_wicks_fock (src/noci/wicks.rs:290-330): Fock intermediates of every pair."""
        w = _SlabWriter()
        npair = len(self.builds)
        foffs = np.zeros((npair, 2, 4), np.int64)
        fvals = np.zeros((npair, 2, 2))
        for p in range(npair):
            x, wref = divmod(p, self.nref)
            rx, rw = self.refs[x], self.refs[wref]
            for sp, fock in enumerate((fa, fb)):
                cx, ox = (rx[0], rx[1]) if sp == 0 else (rx[2], rx[3])
                cw, ow = (rw[0], rw[1]) if sp == 0 else (rw[2], rw[3])
                f0, ff = _wb.construct_f(self.s, fock, cx, ox, cw, ow, self.tol)
                fvals[p, sp] = f0
                for k in range(4):
                    foffs[p, sp, k] = w.put(ff[k >> 1][k & 1].T)
        self.fslab, self.foffs, self.fvals = w.finish(), foffs, fvals
        return self

    def eval_m_pairs(self, obasis: np.ndarray, pairs: np.ndarray, e0: float, exact: bool = False):
        """(M, F, S) per pair with M = F - E0 S (calculate_m_pair_wicks, src/noci/m.rs:160-197)."""
        L = lib()
        pairs = np.ascontiguousarray(pairs, dtype=np.int64)
        n = pairs.shape[0]
        m, f, s = np.empty(n), np.empty(n), np.empty(n)
        L.orc_eval_m_pairs(_ptr(self.slab, ctypes.c_double), _ptr(self.offs, ctypes.c_int64),
                           _ptr(self.vals, ctypes.c_double), _ptr(self.ints, ctypes.c_int32), self.nref,
                           obasis.ctypes.data_as(ctypes.c_void_p), _ptr(pairs, ctypes.c_int64), n,
                           _ptr(self.fslab, ctypes.c_double), _ptr(self.foffs, ctypes.c_int64),
                           _ptr(self.fvals, ctypes.c_double), e0, self.tol, 1 if exact else 0,
                           _ptr(m, ctypes.c_double), _ptr(f, ctypes.c_double), _ptr(s, ctypes.c_double))
        return m, f, s

    def naive_m(self, obasis: np.ndarray, a: int, b: int, fa, fb, e0: float):
        """calculate_m_pair_naive (src/noci/m.rs:106-130) between canonical determinants."""
        ca_x, oa_x, cb_x, ob_x = self.det_orbitals(obasis, a)
        ca_w, oa_w, cb_w, ob_w = self.det_orbitals(obasis, b)
        pa = _naive.build_s_pair(_wb.occ_coeffs(ca_x, oa_x), _wb.occ_coeffs(ca_w, oa_w), self.s, self.tol)
        pb = _naive.build_s_pair(_wb.occ_coeffs(cb_x, ob_x), _wb.occ_coeffs(cb_w, ob_w), self.s, self.tol)
        s = pa.s * pb.s
        f = pb.s * _naive.one_electron(fa, pa) + pa.s * _naive.one_electron(fb, pb)
        return f - e0 * s, f, s

    def det_orbitals(self, obasis: np.ndarray, i: int):
        """Orbital coefficients and integer occupation masks of determinant i (naive path)."""
        d = obasis[i]
        ca, _, cb, _ = self.refs[int(d["parent"])]
        oa = int(d["occ_a"][0]) | (int(d["occ_a"][1]) << 64)
        ob = int(d["occ_b"][0]) | (int(d["occ_b"][1]) << 64)
        return ca, oa, cb, ob

    def naive(self, obasis: np.ndarray, a: int, b: int):
        """calculate_hs_pair_naive between canonically ordered determinants a and b."""
        asym = getattr(self, "_asym", None)
        if asym is None:
            asym = _naive.antisymmetrise(self.eri)
            self._asym = asym
        ca_x, oa_x, cb_x, ob_x = self.det_orbitals(obasis, a)
        ca_w, oa_w, cb_w, ob_w = self.det_orbitals(obasis, b)
        return _naive.hs_pair_naive(self.s, self.h, self.eri, asym, self.enuc, ca_x, oa_x, cb_x,
                                    ob_x, ca_w, oa_w, cb_w, ob_w, self.tol)
