"""B200 engine for the nonorthogonal Wick (H, S) matrix-element path of noci-rs.

``lib`` binds the sm_100a CUDA library (include/nociwick.h); ``synthetic`` builds seeded
stand-in systems and determinant workloads.
"""
from .lib import (WicksShared, build_wicks_shared, calculate_hs_pairs_wicks_batched, load,  # noqa: F401
                  NwError, LIB_PATH, Qmc, Pt2, Screen)
from .synthetic import NW_DET_DTYPE  # noqa: F401
