"""ctypes driver for the test-only CPU build of the engine's per-pair device code."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpu_mirror")
_PATH = os.path.join(_HERE, "_build", "libwick_mirror.so")
_lib = None

D = ctypes.POINTER(ctypes.c_double)
I64 = ctypes.POINTER(ctypes.c_int64)
I32 = ctypes.POINTER(ctypes.c_int32)
U32 = ctypes.POINTER(ctypes.c_uint32)
U64 = ctypes.POINTER(ctypes.c_uint64)
VP = ctypes.c_void_p


def lib():
    global _lib
    if _lib is None:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
        L = ctypes.CDLL(_PATH)
        L.mir_unpack.argtypes = [VP, ctypes.c_int64, I32, I32, I32, U64, U64, D]
        L.mir_far_same_parent.argtypes = [VP, ctypes.c_uint32, ctypes.c_uint32]
        L.mir_sort_keys.argtypes = [VP, ctypes.c_uint64, ctypes.c_int, I32, ctypes.c_int, U32, ctypes.c_uint64,
                                    ctypes.c_uint64, U32, U32, I32]
        L.mir_sort_keys.restype = ctypes.c_uint64
        L.mir_labels.argtypes = [VP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 I32, I32, I32, I32]
        L.mir_svd.argtypes = [ctypes.c_int, D, ctypes.c_double, D, D, D, D]
        L.mir_eval_fast.argtypes = [D, D, D, D, D, D, D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, VP, U32, ctypes.c_int64, D]
        L.mir_eval_gen.argtypes = [D, I64, D, I32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, VP, U32, ctypes.c_int64, D, ctypes.c_int]
        L.mir_eval_s_gen.argtypes = [D, I64, D, I32, ctypes.c_int, ctypes.c_int, ctypes.c_int, VP, U32,
                                     ctypes.c_int64, D]
        L.mir_eval_fs_fast.argtypes = [D, D, ctypes.c_double, ctypes.c_double, D, D, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, VP, U32, ctypes.c_int64, D]
        L.mir_eval_fs_gen.argtypes = [D, I64, D, I32, D, I64, D, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_int, VP, U32, ctypes.c_int64, D, ctypes.c_int]
        L.mir_philox.argtypes = [U32, ctypes.c_uint32, ctypes.c_uint32, U32]
        L.mir_uniform2.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, D]
        L.mir_fri.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.mir_fri.restype = ctypes.c_double
        L.mir_uniform_child.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double]
        L.mir_uniform_child.restype = ctypes.c_uint64
        L.mir_attempts.argtypes = [ctypes.c_double]
        L.mir_attempts.restype = ctypes.c_uint64
        L.mir_diagonal_change.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double]
        L.mir_diagonal_change.restype = ctypes.c_double
        L.mir_layout.argtypes = [ctypes.c_int, D, D, ctypes.c_int64, D]
        _lib = L
    return _lib


def p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def fast_tables(build):
    """Fast-layout arrays of one ordered pair from an oracle PairBuild (m_alpha = m_beta = 0)."""
    out = {}
    for s, (ss, hc) in enumerate(((build.aa, build.hcol0_a), (build.bb, build.hcol0_b))):
        recx = np.ascontiguousarray(np.stack([ss.x[0], hc], axis=-1))
        recy = np.ascontiguousarray(np.stack([ss.y[0], hc], axis=-1))
        j0 = ss.j[0].transpose(2, 3, 0, 1)             # reference stored order [i,j,r,c]
        jas = np.ascontiguousarray(j0 - j0.transpose(0, 3, 2, 1))
        out[s] = (recx, recy, jas, ss.phase * ss.tilde_s_prod, ss.f0h[0] + 0.5 * ss.v0[0])
    out["ii0"] = np.ascontiguousarray(build.ab.ii[(0, 0, 0, 0)])
    out["vab0"] = build.ab.vab0[0][0]
    return out


def eval_fast(build, n, oa, ob, enuc, dets, pairs):
    t = fast_tables(build)
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    hs = np.empty(2 * pairs.shape[0])
    (rxa, rya, ja, pa, ga), (rxb, ryb, jb, pb, gb) = t[0], t[1]
    lib().mir_eval_fast(p(rxa, ctypes.c_double), p(rya, ctypes.c_double), p(ja, ctypes.c_double),
                        p(rxb, ctypes.c_double), p(ryb, ctypes.c_double), p(jb, ctypes.c_double),
                        p(t["ii0"], ctypes.c_double), pa, ga, pb, gb, t["vab0"], n, oa, ob, enuc,
                        dets.ctypes.data_as(VP), p(pairs, ctypes.c_uint32), pairs.shape[0],
                        p(hs, ctypes.c_double))
    return hs[0::2], hs[1::2]


def eval_gen(orc, pidx, n, oa, ob, dets, pairs, exact=False, dispatch=False):
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    hs = np.empty(2 * pairs.shape[0])
    offs = np.ascontiguousarray(orc.offs[pidx])
    vals = np.ascontiguousarray(orc.vals[pidx])
    ints = np.ascontiguousarray(orc.ints[pidx])
    lib().mir_eval_gen(p(orc.slab, ctypes.c_double), p(offs, ctypes.c_int64), p(vals, ctypes.c_double),
                       p(ints, ctypes.c_int32), n, oa, ob, orc.enuc, orc.tol, 1 if exact else 0,
                       dets.ctypes.data_as(VP), p(pairs, ctypes.c_uint32), pairs.shape[0],
                       p(hs, ctypes.c_double), 1 if dispatch else 0)
    return hs[0::2], hs[1::2]


def eval_s_gen(orc, pidx, n, oa, ob, dets, pairs):
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    s = np.empty(pairs.shape[0])
    offs = np.ascontiguousarray(orc.offs[pidx])
    vals = np.ascontiguousarray(orc.vals[pidx])
    ints = np.ascontiguousarray(orc.ints[pidx])
    lib().mir_eval_s_gen(p(orc.slab, ctypes.c_double), p(offs, ctypes.c_int64), p(vals, ctypes.c_double),
                         p(ints, ctypes.c_int32), n, oa, ob, dets.ctypes.data_as(VP),
                         p(pairs, ctypes.c_uint32), pairs.shape[0], p(s, ctypes.c_double))
    return s


def svd(a, tol):
    o = a.shape[0]
    a = np.ascontiguousarray(a, dtype=np.float64)
    u = np.empty((o, o))
    v = np.empty((o, o))
    s = np.empty(o)
    ph = ctypes.c_double()
    lib().mir_svd(o, p(a, ctypes.c_double), tol, p(u, ctypes.c_double), p(v, ctypes.c_double),
                  p(s, ctypes.c_double), ctypes.byref(ph))
    return u, s, v, ph.value


def layout(which, td, te=None):
    n = td.shape[0]
    td = np.ascontiguousarray(td)
    te = np.ascontiguousarray(te if te is not None else td)
    out = np.empty(n ** 4)
    lib().mir_layout(which, p(td, ctypes.c_double), p(te, ctypes.c_double), n, p(out, ctypes.c_double))
    return out.reshape(n, n, n, n)


def eval_fs_fast(orc, build, pidx, n, oa, ob, dets, pairs):
    """(F, S) of one fast ordered pair through the device code, from the oracle's Fock tables."""
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    fs = np.empty(2 * pairs.shape[0])
    recs = []
    for sp, ss in enumerate((build.aa, build.bb)):
        ff00 = orc.fslab[orc.foffs[pidx, sp, 0]:orc.foffs[pidx, sp, 0] + n * n].reshape(n, n).T
        rx = np.ascontiguousarray(np.stack([ss.x[0], ff00], axis=-1))
        ry = np.ascontiguousarray(np.stack([ss.y[0], ff00], axis=-1))
        recs.append((rx, ry, float(orc.fvals[pidx, sp, 0]), ss.phase * ss.tilde_s_prod))
    (rxa, rya, fa, pa), (rxb, ryb, fb, pb) = recs
    lib().mir_eval_fs_fast(p(rxa, ctypes.c_double), p(rya, ctypes.c_double), fa, pa, p(rxb, ctypes.c_double),
                           p(ryb, ctypes.c_double), fb, pb, n, oa, ob, dets.ctypes.data_as(VP),
                           p(pairs, ctypes.c_uint32), pairs.shape[0], p(fs, ctypes.c_double))
    return fs[0::2], fs[1::2]


def eval_fs_gen(orc, pidx, n, oa, ob, dets, pairs, exact=False, dispatch=False):
    """(F, S) of one ordered pair with zero-overlap orbitals through the device code: the
    runtime-size evaluator, or with dispatch the kernel's (register twins up to rank 4)."""
    pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
    fs = np.empty(2 * pairs.shape[0])
    offs = np.ascontiguousarray(orc.offs[pidx])
    vals = np.ascontiguousarray(orc.vals[pidx])
    ints = np.ascontiguousarray(orc.ints[pidx])
    foffs = np.ascontiguousarray(orc.foffs[pidx].reshape(-1))
    fvals = np.ascontiguousarray(orc.fvals[pidx].reshape(-1))
    lib().mir_eval_fs_gen(p(orc.slab, ctypes.c_double), p(offs, ctypes.c_int64), p(vals, ctypes.c_double),
                          p(ints, ctypes.c_int32), p(orc.fslab, ctypes.c_double), p(foffs, ctypes.c_int64),
                          p(fvals, ctypes.c_double), n, oa, ob, orc.tol, 1 if exact else 0,
                          dets.ctypes.data_as(VP), p(pairs, ctypes.c_uint32), pairs.shape[0],
                          p(fs, ctypes.c_double), 1 if dispatch else 0)
    return fs[0::2], fs[1::2]
