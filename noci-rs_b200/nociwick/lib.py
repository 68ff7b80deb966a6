"""ctypes binding of libnociwick.so (the sm_100a engine) and a Python mirror of the noci-rs
interface for the Wick (H, S) path.

The mirror keeps the reference's names so a caller of noci-rs finds the same entry points:

* ``build_wicks_shared``  -> src/noci/wicks.rs:133-279 (intermediates for all reference pairs)
* ``WicksShared``         -> src/nonorthogonalwicks/storage.rs:35-150 (owner of the device slab)
* ``calculate_hs_pairs_wicks_batched`` -> src/noci/hs.rs:72-130 (batched (H, S) for pairs)

There is no CPU evaluation path: if the CUDA library cannot be loaded, or no GPU is present,
the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

from .synthetic import NW_DET_DTYPE

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnociwick.so")
_lib = None

NW_OK = 0
_STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "allocation failed", 4: "unsupported input",
           5: "call out of order", 6: "no CUDA device", 7: "cache file input/output failed"}
CONVENTIONS = {"reference": 0, "exact": 1}
NOALLOC_MAX_PAIRS = 1 << 20
TRANSFORMS = {"fp64": 0, "chol_fp64": 1, "chol_int8": 2, "chol_bf16x6": 3}


class NwError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        super().__init__(f"{where}: {_STATUS.get(status, status)}" + (f" ({detail})" if detail else ""))
        self.status = status


class NwSystem(ctypes.Structure):
    _fields_ = [("nao", ctypes.c_int32), ("nmo", ctypes.c_int32), ("enuc", ctypes.c_double),
                ("s", ctypes.POINTER(ctypes.c_double)), ("h", ctypes.POINTER(ctypes.c_double)),
                ("eri", ctypes.POINTER(ctypes.c_double))]


class NwSystemCd(ctypes.Structure):
    _fields_ = [("nao", ctypes.c_int32), ("nmo", ctypes.c_int32), ("naux", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("enuc", ctypes.c_double), ("s", ctypes.POINTER(ctypes.c_double)),
                ("h", ctypes.POINTER(ctypes.c_double)), ("chol", ctypes.POINTER(ctypes.c_double))]


# ExcitationCache of noci-rs (src/lib.rs:136-167): per spin the rank and holes[0..3] then
# particles[4..7]; 18 bytes, matching nw_exc_cache.
NW_EXC_CACHE_DTYPE = np.dtype([("rank_a", "u1"), ("idx_a", "u1", (8,)), ("rank_b", "u1"), ("idx_b", "u1", (8,))])


def exc_caches(dets: np.ndarray) -> np.ndarray:
    """The excitation caches (NW_EXC_CACHE_DTYPE) of nw_det records."""
    out = np.zeros(dets.shape[0], NW_EXC_CACHE_DTYPE)
    for f in ("rank_a", "idx_a", "rank_b", "idx_b"):
        out[f] = dets[f]
    return out


class NwRefs(ctypes.Structure):
    _fields_ = [("nref", ctypes.c_int32), ("nocc_a", ctypes.c_int32), ("nocc_b", ctypes.c_int32),
                ("c_alpha", ctypes.POINTER(ctypes.c_double)), ("c_beta", ctypes.POINTER(ctypes.c_double))]


class NwOpts(ctypes.Structure):
    _fields_ = [("tol", ctypes.c_double), ("convention", ctypes.c_int32), ("device", ctypes.c_int32)]


class NwQmcOpts(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("initial_population", ctypes.c_double),
                ("target_population", ctypes.c_double), ("sampling_cutoff", ctypes.c_double),
                ("spawn_cutoff", ctypes.c_double), ("shift_damping", ctypes.c_double),
                ("initial_shift", ctypes.c_double), ("ncycles", ctypes.c_int32), ("propagator", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("max_attempts", ctypes.c_uint64), ("update_cutoff", ctypes.c_double)]


class NwQmcReport(ctypes.Structure):
    _fields_ = [("shift", ctypes.c_double), ("eproj_num", ctypes.c_double), ("eproj_den", ctypes.c_double),
                ("nw", ctypes.c_double), ("nref", ctypes.c_double), ("sampled_norm", ctypes.c_double),
                ("nocc", ctypes.c_uint64), ("nattempts", ctypes.c_uint64)]


PROPAGATORS = {"unshifted": 0, "shifted": 1, "doubly-shifted": 2, "difference-doubly-shifted-u1": 3,
               "difference-doubly-shifted-u2": 4, "direct-overlap": 5}


class NwMlpOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_double),
                ("seed", ctypes.c_uint64)]


class NwMlpReport(ctypes.Structure):
    _fields_ = [("loss_first", ctypes.c_double), ("loss_last", ctypes.c_double), ("samples", ctypes.c_uint64),
                ("steps", ctypes.c_int32), ("pad", ctypes.c_int32)]


class NwTuneReport(ctypes.Structure):
    _fields_ = [("key_budget", ctypes.c_uint64), ("blocks_per_sm", ctypes.c_int32), ("trials", ctypes.c_int32),
                ("best_ms", ctypes.c_float), ("default_ms", ctypes.c_float)]


class NwPt2Projection(ctypes.Structure):
    _fields_ = [("e0", ctypes.c_double), ("s_a0", ctypes.c_void_p), ("s_0a", ctypes.c_void_p),
                ("f_a0", ctypes.c_void_p), ("f_0a", ctypes.c_void_p)]


class NwGmresOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int32), ("restart", ctypes.c_int32), ("res_tol", ctypes.c_double),
                ("preconditioner", ctypes.c_int32), ("pad", ctypes.c_int32)]


class NwGmresInfo(ctypes.Structure):
    _fields_ = [("residual_rms", ctypes.c_double), ("iterations", ctypes.c_int32), ("converged", ctypes.c_int32)]


class NwInfo(ctypes.Structure):
    _fields_ = [("nref", ctypes.c_int32), ("nmo", ctypes.c_int32), ("ngeneric", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("slab_bytes", ctypes.c_uint64), ("ndet", ctypes.c_uint64)]


EXPORTED = ("nw_ctx_create", "nw_ctx_create_cholesky", "nw_build_intermediates", "nw_save_intermediates",
            "nw_load_intermediates", "nw_eval_hs_pairs_blocked", "nw_pair_zero_counts",
            "nw_set_basis", "nw_eval_hs_pairs_device", "nw_eval_hs_pairs", "nw_eval_hs_pairs_noalloc",
            "nw_eval_hs_batched", "nw_eval_hs_batched_device", "nw_eval_s_batched", "nw_eval_s_batched_device",
            "nw_eval_fs_batched", "nw_eval_fs_batched_device", "nw_eval_s_pairs_device", "nw_eval_s_pairs",
            "nw_apply_overlap_device", "nw_update_fock", "nw_eval_fs_pairs_device", "nw_eval_fs_pairs",
            "nw_build_hs_matrix", "nw_build_fs_matrix", "nw_general_evp",
            "nw_qmc_create", "nw_qmc_run", "nw_qmc_set_shift", "nw_qmc_last_run_ms", "nw_qmc_populations", "nw_qmc_set_populations", "nw_qmc_cycle_delta",
            "nw_qmc_destroy", "nw_qmc_harvest", "nw_qmc_train_proposal", "nw_qmc_set_generator",
            "nw_qmc_proposal_dims", "nw_qmc_mlp_params", "nw_qmc_set_mlp_params", "nw_qmc_mlp_loss_grad",
            "nw_qmc_proposal_probs", "nw_pt2_create", "nw_pt2_create_matrix_free", "nw_pt2_apply_m", "nw_pt2_last_apply_ms", "nw_pt2_solve",
            "nw_pt2_destroy", "nw_screen_create", "nw_screen_train", "nw_screen_predict", "nw_screen_destroy",
            "nw_autotune", "nw_dgemm", "nw_set_transform", "nw_transform_product", "nw_sync",
            "nw_set_timing", "nw_last_timings", "nw_last_class_timings", "nw_ctx_info", "nw_ctx_destroy", "nw_status_string",
            "nw_last_error")


def load(path: Optional[str] = None):
    """Load libnociwick.so; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"CUDA engine library not found at {p}; build it with `make -C noci-rs_b200` "
                           "(or __graft_entry__.build()).")
    L = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    L.nw_ctx_create.argtypes = [ctypes.POINTER(NwSystem), ctypes.POINTER(NwRefs), ctypes.POINTER(NwOpts),
                                ctypes.POINTER(vp)]
    L.nw_ctx_create_cholesky.argtypes = [ctypes.POINTER(NwSystemCd), ctypes.POINTER(NwRefs), ctypes.POINTER(NwOpts),
                                         ctypes.POINTER(vp)]
    L.nw_build_intermediates.argtypes = [vp]
    L.nw_save_intermediates.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
    L.nw_load_intermediates.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
    L.nw_eval_hs_pairs_blocked.argtypes = [vp, vp, ctypes.c_uint64, vp, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_uint32), vp]
    L.nw_eval_hs_batched.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_hs_batched_device.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_uint64, vp, vp]
    for name in ("nw_eval_s_batched", "nw_eval_s_batched_device", "nw_eval_fs_batched", "nw_eval_fs_batched_device"):
        getattr(L, name).argtypes = [vp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_s_pairs.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_apply_overlap_device.argtypes = [vp, vp, vp, vp]
    L.nw_pair_zero_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.nw_set_basis.argtypes = [vp, vp, ctypes.c_uint64]
    L.nw_eval_hs_pairs_device.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_hs_pairs.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_hs_pairs_noalloc.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_s_pairs_device.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_update_fock.argtypes = [vp, vp, vp]
    L.nw_eval_fs_pairs_device.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_eval_fs_pairs.argtypes = [vp, vp, ctypes.c_uint64, vp, vp]
    L.nw_build_hs_matrix.argtypes = [vp, vp, ctypes.c_uint64, vp, ctypes.c_uint64, ctypes.c_int, vp, vp]
    L.nw_build_fs_matrix.argtypes = [vp, vp, ctypes.c_uint64, vp, ctypes.c_uint64, ctypes.c_int, vp, vp]
    L.nw_general_evp.argtypes = [vp, ctypes.c_int32, vp, vp, ctypes.c_int, ctypes.c_double, vp, vp,
                                 ctypes.POINTER(ctypes.c_int32)]
    L.nw_qmc_create.argtypes = [vp, ctypes.POINTER(NwQmcOpts), vp, vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.nw_qmc_run.argtypes = [vp, ctypes.c_int32, vp]
    L.nw_qmc_last_run_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.nw_qmc_set_shift.argtypes = [vp, ctypes.c_double]
    L.nw_qmc_populations.argtypes = [vp, vp]
    L.nw_qmc_set_populations.argtypes = [vp, vp]
    L.nw_qmc_cycle_delta.argtypes = [vp, ctypes.c_uint64, vp]
    L.nw_qmc_destroy.argtypes = [vp]
    L.nw_qmc_harvest.argtypes = [vp, ctypes.c_int32, ctypes.c_double]
    L.nw_qmc_train_proposal.argtypes = [vp, ctypes.POINTER(NwMlpOpts), ctypes.POINTER(NwMlpReport)]
    L.nw_qmc_set_generator.argtypes = [vp, ctypes.c_int32, ctypes.c_double]
    L.nw_qmc_proposal_dims.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_uint64)]
    L.nw_qmc_mlp_params.argtypes = [vp, vp]
    L.nw_qmc_set_mlp_params.argtypes = [vp, vp]
    L.nw_qmc_mlp_loss_grad.argtypes = [vp, vp, vp, vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_double), vp]
    L.nw_qmc_proposal_probs.argtypes = [vp, ctypes.c_uint32, vp]
    L.nw_pt2_create.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(vp)]
    L.nw_pt2_create_matrix_free.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(vp)]
    L.nw_pt2_apply_m.argtypes = [vp, vp, vp]
    L.nw_pt2_last_apply_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.nw_pt2_solve.argtypes = [vp, ctypes.POINTER(NwPt2Projection), vp, ctypes.POINTER(NwGmresOpts), vp,
                               ctypes.POINTER(NwGmresInfo)]
    L.nw_pt2_destroy.argtypes = [vp]
    L.nw_screen_create.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.nw_screen_train.argtypes = [vp, vp, vp, ctypes.c_uint64, ctypes.POINTER(NwMlpOpts), ctypes.POINTER(NwMlpReport)]
    L.nw_screen_predict.argtypes = [vp, vp, ctypes.c_uint64, vp]
    L.nw_screen_destroy.argtypes = [vp]
    L.nw_autotune.argtypes = [vp, vp, ctypes.c_uint64, vp, vp, ctypes.POINTER(NwTuneReport)]
    L.nw_sync.argtypes = [vp, vp]
    L.nw_dgemm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                           vp, ctypes.c_int, ctypes.c_longlong, vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_double,
                           vp, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, vp]
    L.nw_set_transform.argtypes = [vp, ctypes.c_int32]
    L.nw_transform_product.argtypes = [ctypes.c_int32, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp]
    L.nw_set_timing.argtypes = [vp, ctypes.c_int]
    L.nw_last_timings.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.nw_last_class_timings.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.nw_ctx_info.argtypes = [vp, ctypes.POINTER(NwInfo)]
    L.nw_ctx_destroy.argtypes = [vp]
    L.nw_status_string.argtypes = [ctypes.c_int]
    L.nw_status_string.restype = ctypes.c_char_p
    L.nw_last_error.argtypes = [vp]
    L.nw_last_error.restype = ctypes.c_char_p
    for name in EXPORTED:
        if name not in ("nw_status_string", "nw_last_error"):
            getattr(L, name).restype = ctypes.c_int
    if path is None:
        _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class WicksShared:
    """Device-resident Wick intermediates for every ordered reference pair, plus the resident
    determinant basis.  Mirrors noci-rs WicksShared/WicksView (storage.rs:35-150, view.rs:20-147)."""

    def __init__(self, s, h, eri, enuc: float, refs: Sequence[Tuple[np.ndarray, int, np.ndarray, int]],
                 tol: float = 1e-8, convention: str = "reference", device: int = 0, chol=None):
        """With ``chol`` (naux x nao x nao Cholesky vectors) instead of ``eri`` (pass None) the
        context is created from the factored integrals (nw_ctx_create_cholesky)."""
        self._lib = load()
        self._ctx = ctypes.c_void_p()
        nmo = refs[0][0].shape[1]
        nao = refs[0][0].shape[0]
        nocc_a = bin(refs[0][1]).count("1")
        nocc_b = bin(refs[0][3]).count("1")
        for (ca, oa, cb, ob) in refs:
            if oa != (1 << nocc_a) - 1 or ob != (1 << nocc_b) - 1:
                raise ValueError("reference occupations must be the first nocc orbitals (aufbau order)")
        self._s = np.ascontiguousarray(s, dtype=np.float64)
        self._h = np.ascontiguousarray(h, dtype=np.float64)
        self._ca = np.ascontiguousarray(np.stack([r[0] for r in refs]), dtype=np.float64)
        self._cb = np.ascontiguousarray(np.stack([r[2] for r in refs]), dtype=np.float64)
        rd = NwRefs(len(refs), nocc_a, nocc_b, _dp(self._ca), _dp(self._cb))
        od = NwOpts(float(tol), CONVENTIONS[convention], int(device))
        if chol is not None:
            self._chol = np.ascontiguousarray(chol, dtype=np.float64)
            sysc = NwSystemCd(nao, nmo, self._chol.shape[0], 0, float(enuc), _dp(self._s), _dp(self._h),
                              _dp(self._chol))
            st = self._lib.nw_ctx_create_cholesky(ctypes.byref(sysc), ctypes.byref(rd), ctypes.byref(od),
                                                  ctypes.byref(self._ctx))
            where = "nw_ctx_create_cholesky"
        else:
            self._eri = np.ascontiguousarray(eri, dtype=np.float64)
            sysd = NwSystem(nao, nmo, float(enuc), _dp(self._s), _dp(self._h), _dp(self._eri))
            st = self._lib.nw_ctx_create(ctypes.byref(sysd), ctypes.byref(rd), ctypes.byref(od),
                                         ctypes.byref(self._ctx))
            where = "nw_ctx_create"
        if st != NW_OK:
            raise NwError(st, where)
        self.nref, self.nmo, self.nocc_a, self.nocc_b = len(refs), nmo, nocc_a, nocc_b
        self.tol, self.convention = tol, convention
        self._basis = None

    # -- lifetime --------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            self._lib.nw_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, where: str):
        if st != NW_OK:
            detail = self._lib.nw_last_error(self._ctx)
            raise NwError(st, where, detail.decode() if detail else "")

    # -- build / basis ---------------------------------------------------------------------
    def build(self):
        self._check(self._lib.nw_build_intermediates(self._ctx), "nw_build_intermediates")
        return self

    def save(self, slab_path, meta_path):
        """Write the built intermediates to a slab file and a metadata file (nw_save_intermediates)."""
        self._check(self._lib.nw_save_intermediates(self._ctx, str(slab_path).encode(), str(meta_path).encode()),
                    "nw_save_intermediates")
        return self

    def load(self, slab_path, meta_path):
        """Restore intermediates saved for this system instead of building them (nw_load_intermediates)."""
        self._check(self._lib.nw_load_intermediates(self._ctx, str(slab_path).encode(), str(meta_path).encode()),
                    "nw_load_intermediates")
        return self

    def set_transform(self, mode: str):
        """Four-index transform of the next build: "fp64" (quarter transforms of the full
        tensor), or on a Cholesky context "chol_fp64", "chol_int8" (tcgen05 Ozaki slices,
        FP64-faithful) or "chol_bf16x6" (tcgen05 BF16 pieces, FP32 class)."""
        self._check(self._lib.nw_set_transform(self._ctx, TRANSFORMS[mode]), "nw_set_transform")
        return self

    def zero_counts(self) -> np.ndarray:
        m = np.zeros(2 * self.nref * self.nref, np.int32)
        self._check(self._lib.nw_pair_zero_counts(self._ctx, m.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))),
                    "nw_pair_zero_counts")
        return m.reshape(self.nref, self.nref, 2)

    def set_basis(self, dets: np.ndarray):
        dets = np.ascontiguousarray(dets)
        if dets.dtype != NW_DET_DTYPE:
            raise TypeError("basis must use the nw_det record dtype")
        self._check(self._lib.nw_set_basis(self._ctx, dets.ctypes.data, dets.shape[0]), "nw_set_basis")
        self._basis = dets
        return self

    def info(self) -> dict:
        inf = NwInfo()
        self._check(self._lib.nw_ctx_info(self._ctx, ctypes.byref(inf)), "nw_ctx_info")
        return {"nref": inf.nref, "nmo": inf.nmo, "ngeneric": inf.ngeneric, "slab_bytes": inf.slab_bytes,
                "ndet": inf.ndet}

    # -- evaluation ------------------------------------------------------------------------
    def eval_pairs(self, pairs: np.ndarray, out: Optional[np.ndarray] = None, stream: int = 0):
        """(H, S) for host pairs (n, 2) -> host array (n, 2); copies in and out inside the call."""
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
        n = pairs.shape[0]
        if out is None:
            out = np.empty((n, 2), np.float64)
        self._check(self._lib.nw_eval_hs_pairs(self._ctx, pairs.ctypes.data, n, out.ctypes.data,
                                               ctypes.c_void_p(stream)), "nw_eval_hs_pairs")
        return out

    def eval_batched(self, lp: int, gp: int, x_caches: np.ndarray, w_caches: np.ndarray, phase: np.ndarray,
                     stream: int = 0, kind: str = "hs") -> np.ndarray:
        """One ordered reference pair (lp, gp) from caller-held excitation caches
        (xw_hamiltonian_overlap_prepared_batched): x_caches / w_caches of NW_EXC_CACHE_DTYPE,
        phase the product of both excitation phases per request.  kind "hs" returns (H, S) as
        (n, 2), "s" the overlaps (n,), "fs" (F, S) as (n, 2) after update_fock."""
        x = np.ascontiguousarray(x_caches, dtype=NW_EXC_CACHE_DTYPE)
        w = np.ascontiguousarray(w_caches, dtype=NW_EXC_CACHE_DTYPE)
        ph = np.ascontiguousarray(phase, dtype=np.float64)
        n = x.shape[0]
        if w.shape[0] != n or ph.shape[0] != n:
            raise ValueError("x_caches, w_caches and phase must have one entry per request")
        fn = {"hs": "nw_eval_hs_batched", "s": "nw_eval_s_batched", "fs": "nw_eval_fs_batched"}[kind]
        out = np.empty((n,) if kind == "s" else (n, 2), np.float64)
        self._check(getattr(self._lib, fn)(self._ctx, int(lp), int(gp), x.ctypes.data, w.ctypes.data,
                                           ph.ctypes.data, n, out.ctypes.data, ctypes.c_void_p(stream)), fn)
        return out

    def eval_overlap(self, pairs: np.ndarray, stream: int = 0) -> np.ndarray:
        """S for host pairs (n, 2) (nw_eval_s_pairs)."""
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
        out = np.empty(pairs.shape[0], np.float64)
        self._check(self._lib.nw_eval_s_pairs(self._ctx, pairs.ctypes.data, pairs.shape[0], out.ctypes.data,
                                              ctypes.c_void_p(stream)), "nw_eval_s_pairs")
        return out

    def eval_pairs_blocked(self, pairs_ptr: int, npairs: int, out_ptr: int, slab_budget: int = 0,
                           stream: int = 0) -> int:
        """(H, S) of device pairs in blocks of reference pairs whose intermediates fit
        slab_budget bytes (nw_eval_hs_pairs_blocked); returns the number of blocks."""
        nb = ctypes.c_uint32(0)
        self._check(self._lib.nw_eval_hs_pairs_blocked(self._ctx, ctypes.c_void_p(pairs_ptr), npairs,
                                                       ctypes.c_void_p(out_ptr), int(slab_budget), ctypes.byref(nb),
                                                       ctypes.c_void_p(stream)), "nw_eval_hs_pairs_blocked")
        return int(nb.value)

    def eval_pairs_device(self, pairs_ptr: int, npairs: int, out_ptr: int, stream: int = 0):
        self._check(self._lib.nw_eval_hs_pairs_device(self._ctx, ctypes.c_void_p(pairs_ptr), npairs,
                                                      ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)),
                    "nw_eval_hs_pairs_device")

    def eval_pairs_noalloc(self, pairs_ptr: int, npairs: int, out_ptr: int, stream: int = 0):
        """(H, S) into device memory without any device allocation (fixed scratch array; at most
        NOALLOC_MAX_PAIRS pairs per call; calls sharing the GPU must not overlap)."""
        self._check(self._lib.nw_eval_hs_pairs_noalloc(self._ctx, ctypes.c_void_p(pairs_ptr), npairs,
                                                       ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)),
                    "nw_eval_hs_pairs_noalloc")

    def apply_overlap_device(self, x_ptr: int, y_ptr: int, stream: int = 0):
        """y += S x over the resident basis (device buffers of ndet doubles; nw_apply_overlap_device).
        The first call on a basis builds the spin-factor tables."""
        self._check(self._lib.nw_apply_overlap_device(self._ctx, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                                      ctypes.c_void_p(stream)), "nw_apply_overlap_device")

    def eval_overlap_device(self, pairs_ptr: int, npairs: int, out_ptr: int, stream: int = 0):
        self._check(self._lib.nw_eval_s_pairs_device(self._ctx, ctypes.c_void_p(pairs_ptr), npairs,
                                                     ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)),
                    "nw_eval_s_pairs_device")

    # -- Fock (F, S) path ---------------------------------------------------------------------
    def update_fock(self, fock_a: np.ndarray, fock_b: np.ndarray):
        """update_wicks_fock (src/noci/wicks.rs:290-330): Fock tables from AO Fock matrices."""
        fa = np.ascontiguousarray(fock_a, dtype=np.float64)
        fb = np.ascontiguousarray(fock_b, dtype=np.float64)
        self._check(self._lib.nw_update_fock(self._ctx, fa.ctypes.data, fb.ctypes.data), "nw_update_fock")
        return self

    def eval_fs_pairs(self, pairs: np.ndarray, out: Optional[np.ndarray] = None, stream: int = 0):
        """(F, S) for host pairs (n, 2) -> host array (n, 2); M = F - E0 S is the SNOCI element."""
        pairs = np.ascontiguousarray(pairs, dtype=np.uint32)
        n = pairs.shape[0]
        if out is None:
            out = np.empty((n, 2), np.float64)
        self._check(self._lib.nw_eval_fs_pairs(self._ctx, pairs.ctypes.data, n, out.ctypes.data,
                                               ctypes.c_void_p(stream)), "nw_eval_fs_pairs")
        return out

    def eval_fs_pairs_device(self, pairs_ptr: int, npairs: int, out_ptr: int, stream: int = 0):
        self._check(self._lib.nw_eval_fs_pairs_device(self._ctx, ctypes.c_void_p(pairs_ptr), npairs,
                                                      ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream)),
                    "nw_eval_fs_pairs_device")

    # -- dense matrices and the generalised eigenproblem ------------------------------------
    def _matrix(self, fn, where, left, right, symmetric):
        nd = self.info()["ndet"]
        left = np.arange(nd, dtype=np.uint32) if left is None else np.ascontiguousarray(left, dtype=np.uint32)
        right = left if right is None else np.ascontiguousarray(right, dtype=np.uint32)
        a = np.empty((left.shape[0], right.shape[0]))
        s = np.empty_like(a)
        self._check(fn(self._ctx, left.ctypes.data, left.shape[0], right.ctypes.data, right.shape[0],
                       1 if symmetric else 0, a.ctypes.data, s.ctypes.data), where)
        return a, s

    def build_hs_matrix(self, left=None, right=None, symmetric: bool = True):
        """build_noci_hs (src/noci/matrix.rs): dense H and S over a block of the resident basis
        (default: the whole basis, symmetric)."""
        return self._matrix(self._lib.nw_build_hs_matrix, "nw_build_hs_matrix", left, right, symmetric)

    def build_fs_matrix(self, left=None, right=None, symmetric: bool = True):
        """build_noci_fock (src/noci/matrix.rs): dense F and S after update_fock."""
        return self._matrix(self._lib.nw_build_fs_matrix, "nw_build_fs_matrix", left, right, symmetric)

    def general_evp(self, h: np.ndarray, s: np.ndarray, project: bool = True, tol: float = 1e-8):
        """general_evp (src/maths/linalg.rs:230-256) on the GPU: (eigenvalues, eigenvectors C)."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        s = np.ascontiguousarray(s, dtype=np.float64)
        n = h.shape[0]
        evals = np.empty(n)
        c = np.empty(n * n)
        k = ctypes.c_int32()
        self._check(self._lib.nw_general_evp(self._ctx, n, h.ctypes.data, s.ctypes.data, 1 if project else 0, tol,
                                             evals.ctypes.data, c.ctypes.data, ctypes.byref(k)), "nw_general_evp")
        k = k.value
        return evals[:k].copy(), c[:n * k].reshape(n, k).copy()

    def autotune(self, pairs_ptr: int, npairs: int, out_ptr: int, stream: int = 0) -> dict:
        """nw_autotune on device pairs: picks the fine-key budget and blocks per SM of later calls."""
        rep = NwTuneReport()
        self._check(self._lib.nw_autotune(self._ctx, ctypes.c_void_p(pairs_ptr), npairs, ctypes.c_void_p(out_ptr),
                                          ctypes.c_void_p(stream), ctypes.byref(rep)), "nw_autotune")
        return {"key_budget": rep.key_budget, "blocks_per_sm": rep.blocks_per_sm, "trials": rep.trials,
                "best_ms": rep.best_ms, "default_ms": rep.default_ms}

    def pt2(self, candidates, e0: float, matrix_free: bool = False) -> "Pt2":
        """The candidate operator M = F - E0 S over resident determinants: packed on the device
        (nw_pt2_create) or applied matrix-free (nw_pt2_create_matrix_free)."""
        return Pt2(self, candidates, e0, matrix_free=matrix_free)

    def set_timing(self, enable: bool = True, serial_classes: bool = False):
        """Phase timing of the following evaluations; serial_classes runs the class evaluators
        one after another (a profiling mode, last_class_timings)."""
        mode = (2 if serial_classes else 1) if enable else 0
        self._check(self._lib.nw_set_timing(self._ctx, mode), "nw_set_timing")

    def last_class_timings(self) -> dict:
        """Device ms of each class evaluator of the last serially timed evaluation."""
        ms = (ctypes.c_float * 5)()
        self._check(self._lib.nw_last_class_timings(self._ctx, ms), "nw_last_class_timings")
        return dict(zip(("light", "medium", "heavy", "rt", "gen"), [float(v) for v in ms]))

    def last_timings(self) -> dict:
        """Device ms of the phases of the last evaluation (CUDA events on its stream)."""
        ms = (ctypes.c_float * 5)()
        self._check(self._lib.nw_last_timings(self._ctx, ms), "nw_last_timings")
        return dict(zip(("classify", "scan", "scatter", "eval_m0", "eval_gen"), [float(v) for v in ms]))

    def sync(self, stream: int = 0):
        self._check(self._lib.nw_sync(self._ctx, ctypes.c_void_p(stream)), "nw_sync")


class Qmc:
    """NOCI-QMC on the GPU: signed real walkers (qmc_step of src/stochastic/walkers.rs), or with
    propagator="direct-overlap" the real metric population of qmc_step in src/stochastic/metric.rs
    (N_0 = S c_0, each report's change applied through the overlap, FRI-compressed with
    ``update_cutoff``), with the uniform generator.  ``c0`` has one coefficient per determinant of
    the resident basis; ``ref_idx`` are the reference determinants used for the projected energy."""

    REPORT_FIELDS = ("shift", "eproj_num", "eproj_den", "nw", "nref", "sampled_norm", "nocc", "nattempts")

    def __init__(self, wicks: "WicksShared", c0, ref_idx, dt: float, initial_population: float = 100.0,
                 target_population: float = 1e5, sampling_cutoff: float = 0.0, spawn_cutoff: float = 0.0,
                 shift_damping: float = 5e-4, initial_shift: float = 0.0, ncycles: int = 10,
                 propagator: str = "unshifted", seed: int = 1, max_attempts: int = 0, update_cutoff: float = 0.0):
        self._w = wicks
        self._lib = wicks._lib
        c0 = np.ascontiguousarray(c0, dtype=np.float64)
        ref = np.ascontiguousarray(ref_idx, dtype=np.uint32)
        o = NwQmcOpts(dt, initial_population, target_population, sampling_cutoff, spawn_cutoff, shift_damping,
                      initial_shift, ncycles, PROPAGATORS[propagator] if isinstance(propagator, str) else propagator,
                      seed, max_attempts, update_cutoff)
        self._q = ctypes.c_void_p()
        self.ndet = c0.shape[0]
        wicks._check(self._lib.nw_qmc_create(wicks._ctx, ctypes.byref(o), c0.ctypes.data, ref.ctypes.data,
                                             ref.shape[0], ctypes.byref(self._q)), "nw_qmc_create")

    def run(self, nreports: int) -> np.ndarray:
        """Run report blocks; returns a structured array of per-block statistics."""
        reps = (NwQmcReport * max(nreports, 1))()
        self._w._check(self._lib.nw_qmc_run(self._q, nreports, reps), "nw_qmc_run")
        dt = np.dtype([(f, np.float64) for f in self.REPORT_FIELDS[:6]] + [("nocc", np.uint64), ("nattempts", np.uint64)])
        out = np.frombuffer(bytes(reps), dtype=dt)[:nreports].copy()
        return out

    def set_shift(self, shift: float):
        self._w._check(self._lib.nw_qmc_set_shift(self._q, shift), "nw_qmc_set_shift")

    def last_run_ms(self) -> float:
        """Device ms of the report blocks of the last run (CUDA events on the run's stream)."""
        ms = ctypes.c_float()
        self._w._check(self._lib.nw_qmc_last_run_ms(self._q, ctypes.byref(ms)), "nw_qmc_last_run_ms")
        return float(ms.value)

    def populations(self) -> np.ndarray:
        out = np.empty(self.ndet)
        self._w._check(self._lib.nw_qmc_populations(self._q, out.ctypes.data), "nw_qmc_populations")
        return out

    def set_populations(self, pop):
        pop = np.ascontiguousarray(pop, dtype=np.float64)
        self._w._check(self._lib.nw_qmc_set_populations(self._q, pop.ctypes.data), "nw_qmc_set_populations")

    def cycle_delta(self, cycle: int) -> np.ndarray:
        out = np.empty(self.ndet)
        self._w._check(self._lib.nw_qmc_cycle_delta(self._q, cycle, out.ctypes.data), "nw_qmc_cycle_delta")
        return out

    # -- learned proposal -------------------------------------------------------------------
    def harvest(self, enable: bool = True, keep: float = 1.0):
        """Record the attempts of the following runs (each with probability `keep`) for training
        the proposal."""
        self._w._check(self._lib.nw_qmc_harvest(self._q, 1 if enable else 0, keep), "nw_qmc_harvest")

    def train_proposal(self, epochs: int = 2, batch: int = 4096, lr: float = 1e-3, seed: int = 7) -> dict:
        rep = NwMlpReport()
        self._w._check(self._lib.nw_qmc_train_proposal(self._q, ctypes.byref(NwMlpOpts(epochs, batch, lr, seed)),
                                                       ctypes.byref(rep)), "nw_qmc_train_proposal")
        return {"loss_first": rep.loss_first, "loss_last": rep.loss_last, "samples": rep.samples, "steps": rep.steps}

    def set_generator(self, learned: bool, mix: float = 0.1):
        self._w._check(self._lib.nw_qmc_set_generator(self._q, 1 if learned else 0, mix), "nw_qmc_set_generator")

    def proposal_dims(self):
        din, nbin, npar = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_uint64()
        self._w._check(self._lib.nw_qmc_proposal_dims(self._q, ctypes.byref(din), ctypes.byref(nbin),
                                                      ctypes.byref(npar)), "nw_qmc_proposal_dims")
        return din.value, nbin.value, npar.value

    def mlp_params(self) -> np.ndarray:
        out = np.empty(self.proposal_dims()[2], np.float32)
        self._w._check(self._lib.nw_qmc_mlp_params(self._q, out.ctypes.data), "nw_qmc_mlp_params")
        return out

    def set_mlp_params(self, params):
        params = np.ascontiguousarray(params, dtype=np.float32)
        self._w._check(self._lib.nw_qmc_set_mlp_params(self._q, params.ctypes.data), "nw_qmc_set_mlp_params")

    def mlp_loss_grad(self, parents, bins, w):
        parents = np.ascontiguousarray(parents, dtype=np.uint32)
        bins = np.ascontiguousarray(bins, dtype=np.uint32)
        w = np.ascontiguousarray(w, dtype=np.float32)
        loss = ctypes.c_double()
        grads = np.empty(self.proposal_dims()[2], np.float32)
        self._w._check(self._lib.nw_qmc_mlp_loss_grad(self._q, parents.ctypes.data, bins.ctypes.data, w.ctypes.data,
                                                      parents.shape[0], ctypes.byref(loss), grads.ctypes.data),
                       "nw_qmc_mlp_loss_grad")
        return loss.value, grads

    def proposal_probs(self, det: int) -> np.ndarray:
        out = np.empty(self.proposal_dims()[1])
        self._w._check(self._lib.nw_qmc_proposal_probs(self._q, det, out.ctypes.data), "nw_qmc_proposal_probs")
        return out

    def close(self):
        if getattr(self, "_q", None) and self._q.value:
            self._lib.nw_qmc_destroy(self._q)
            self._q = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Pt2:
    """NOCI-PT2 / SNOCI linear solve on the GPU: M = F - E0 S over candidate determinants of the
    resident basis (packed on the device), its mat-vec and GMRES on the projected operator
    (build_candidate_m, apply_candidate_m, apply_omega_m and gmres of src/snoci)."""

    def __init__(self, wicks: "WicksShared", candidates, e0: float, matrix_free: bool = False):
        """With ``matrix_free`` M is not stored: every product evaluates its pairs again
        (nw_pt2_create_matrix_free), O(n) device memory instead of n^2 / 2 doubles."""
        self._w = wicks
        self._lib = wicks._lib
        cand = np.ascontiguousarray(candidates, dtype=np.uint32)
        self.n = cand.shape[0]
        self._p = ctypes.c_void_p()
        fn = self._lib.nw_pt2_create_matrix_free if matrix_free else self._lib.nw_pt2_create
        wicks._check(fn(wicks._ctx, cand.ctypes.data, self.n, e0, ctypes.byref(self._p)),
                     "nw_pt2_create_matrix_free" if matrix_free else "nw_pt2_create")

    def apply_m(self, x) -> np.ndarray:
        """y = M x (apply_candidate_m)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        self._w._check(self._lib.nw_pt2_apply_m(self._p, x.ctypes.data, y.ctypes.data), "nw_pt2_apply_m")
        return y

    def last_apply_ms(self) -> float:
        ms = ctypes.c_float()
        self._w._check(self._lib.nw_pt2_last_apply_ms(self._p, ctypes.byref(ms)), "nw_pt2_last_apply_ms")
        return float(ms.value)

    def solve(self, e0, s_a0, s_0a, f_a0, f_0a, rhs, max_iter: int = 100, restart: int = 200,
              res_tol: float = 1e-8, preconditioner: str = "woodbury"):
        """GMRES on M^Omega x = rhs; returns (x, info)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (s_a0, s_0a, f_a0, f_0a, rhs)]
        proj = NwPt2Projection(e0, *(a.ctypes.data for a in arrs[:4]))
        opts = NwGmresOpts(max_iter, restart, res_tol, 1 if preconditioner == "woodbury" else 0, 0)
        x = np.empty(self.n)
        info = NwGmresInfo()
        self._w._check(self._lib.nw_pt2_solve(self._p, ctypes.byref(proj), arrs[4].ctypes.data, ctypes.byref(opts),
                                              x.ctypes.data, ctypes.byref(info)), "nw_pt2_solve")
        return x, {"residual_rms": info.residual_rms, "iterations": info.iterations, "converged": bool(info.converged)}

    def close(self):
        if getattr(self, "_p", None) and self._p.value:
            self._lib.nw_pt2_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Screen:
    """Learned SNOCI candidate screener on the GPU (nw_screen_*): an MLP over determinant
    descriptors regressing a per-determinant target (log10 of the PT2 selection score).
    Indices refer to the resident basis at the time of each call."""

    def __init__(self, wicks: "WicksShared", seed: int = 17):
        self._w = wicks
        self._lib = wicks._lib
        self._s = ctypes.c_void_p()
        wicks._check(self._lib.nw_screen_create(wicks._ctx, seed, ctypes.byref(self._s)), "nw_screen_create")

    def train(self, idx, target, epochs: int = 20, batch: int = 1024, lr: float = 1e-3, seed: int = 3) -> dict:
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        target = np.ascontiguousarray(target, dtype=np.float64)
        rep = NwMlpReport()
        self._w._check(self._lib.nw_screen_train(self._s, idx.ctypes.data, target.ctypes.data, idx.shape[0],
                                                 ctypes.byref(NwMlpOpts(epochs, batch, lr, seed)), ctypes.byref(rep)),
                       "nw_screen_train")
        return {"loss_first": rep.loss_first, "loss_last": rep.loss_last, "samples": rep.samples, "steps": rep.steps}

    def predict(self, idx) -> np.ndarray:
        idx = np.ascontiguousarray(idx, dtype=np.uint32)
        out = np.empty(idx.shape[0])
        self._w._check(self._lib.nw_screen_predict(self._s, idx.ctypes.data, idx.shape[0], out.ctypes.data),
                       "nw_screen_predict")
        return out

    def close(self):
        if getattr(self, "_s", None) and self._s.value:
            self._lib.nw_screen_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def build_wicks_shared(ao, refs, tol: float = 1e-8, convention: str = "reference", device: int = 0) -> WicksShared:
    """noci-rs build_wicks_shared (src/noci/wicks.rs:133-279): intermediates for all ordered
    reference pairs, built on the GPU.  ``ao`` has attributes s, h, eri, enuc."""
    return WicksShared(ao.s, ao.h, ao.eri, ao.enuc, refs, tol, convention, device).build()


def calculate_hs_pairs_wicks_batched(wicks: WicksShared, pairs: np.ndarray,
                                     reduced_basis: Optional[np.ndarray] = None) -> np.ndarray:
    """noci-rs calculate_hs_pairs_wicks_batched (src/noci/hs.rs:72-130): (H, S) per pair.

    ``pairs`` is (n, 2) determinant indices; ``reduced_basis`` (nw_det records) replaces the
    resident basis when given.  Returns an (n, 2) array of (H, S).
    """
    if reduced_basis is not None:
        wicks.set_basis(reduced_basis)
    return wicks.eval_pairs(pairs)
