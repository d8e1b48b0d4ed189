"""numpy record types of the C ABI's structs (include/sabertooth_b200.h).

Pure numpy: importing this module loads no library, so input generators can
build arrays in these layouts without mapping the CUDA library.
"""
import numpy as np

PAIR_DTYPE = np.dtype([("profile", "<u4"), ("target", "<u4"), ("band_center", "<i4"), ("band_radius", "<i4")])
LANE_DTYPE = np.dtype([("target", "<u4"), ("lo", "<u4"), ("hi", "<u4"), ("diag", "<i4")])
HIT_DTYPE = np.dtype([("query", "<u4"), ("target", "<u4"), ("diag", "<i4")])
SEED_HIT_DTYPE = np.dtype([("query", "<u4"), ("target", "<u4"), ("diag", "<i4"), ("qpos", "<u4")])
CANDIDATE_DTYPE = np.dtype([("query", "<u4"), ("target", "<u4"), ("hits", "<u4"), ("diag_score", "<i4"),
                            ("best_diag", "<i8"), ("t_lo", "<u4"), ("t_hi", "<u4")])
