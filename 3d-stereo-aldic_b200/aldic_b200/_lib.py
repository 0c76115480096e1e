"""ctypes binding of the in-tree CUDA library ``libaldic_b200.so`` (C ABI in
include/aldic_b200.h).  There is no CPU fallback: if the library is missing or cannot be
loaded, every entry point raises."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaldic_b200.so")

ALDIC_OK = 0
ALDIC_ERR_ARG = 1
ALDIC_ERR_CUDA = 2
ALDIC_ERR_TIMEOUT = 3
ALDIC_ERR_STATE = 4

U8, U16, F32, F64 = 0, 1, 2, 3
SLOT_REF, SLOT_DEF = 0, 1
UNIFORM, QUADTREE = 0, 1
OPT_ITERATION_CAP, OPT_STAGING, OPT_SLOW_WARPS, OPT_SEARCH_IMPL, OPT_SEARCH_CHUNK, OPT_AUTOTUNE = 0, 1, 2, 3, 4, 5
OPT_SLOW_FP64, OPT_FP64_THREADS = 6, 7
STAT_FP64_RESOLVES, STAT_STAGING_TIMEOUT = 100, 101
# iterations the one-warp solver pass gives a subset before the multi-warp pass restarts it, when
# aldic_set_iteration_cap has not been called (kDefaultWarpCap in csrc/kernels.h)
DEFAULT_ITERATION_CAP = 8
# relative band around tol in which an FP32 convergence test is re-decided in FP64, when
# aldic_set_fp64_band has not been called (kDefaultFp64Band in csrc/kernels.h)
DEFAULT_FP64_BAND = 1e-3
DEFAULT_FP64_NOISE = 4.0

# Every symbol the header declares, with (restype, argtypes).
_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
SIGNATURES = {
    "aldic_create": (_i, [C.POINTER(_vp), _i]),
    "aldic_destroy": (None, [_vp]),
    "aldic_last_error": (C.c_char_p, [_vp]),
    "aldic_set_stream": (_i, [_vp, _vp]),
    "aldic_synchronize": (_i, [_vp]),
    "aldic_launch_count": (_i64, [_vp]),
    "aldic_abi_version": (_i, []),
    "aldic_load_image_raw": (_i, [_vp, _i, _vp, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "aldic_load_image": (_i, [_vp, _i, _vp, _i, _i]),
    "aldic_set_mask": (_i, [_vp, _vp, _i, _i]),
    "aldic_compute_gradients": (_i, [_vp]),
    "aldic_set_gradients": (_i, [_vp, _vp, _vp, _i, _i]),
    "aldic_get_state": (_i, [_vp, _i, _vp]),
    "aldic_interp2": (_i, [_vp, _i, _i64, _vp, _vp, _vp]),
    "aldic_search_grid": (_i, [_vp, _vp, _i, _i, C.POINTER(_i), C.POINTER(_i)]),
    "aldic_integer_search": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp]),
    "aldic_local_icgn": (_i, [_vp, _i, _i64, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp, _vp]),
    "aldic_subpb1": (_i, [_vp, _i, _i64, _vp, _vp, _vp, _vp, _vp, _i, _vp, _d, _d, _vp, _vp]),
    "aldic_epipolar_icgn": (_i, [_vp, _i64, _vp, _i, _d, _vp]),
    "aldic_triangulate": (_i, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "aldic_undistort_points": (_i, [_vp, _i64, _vp, _vp, _vp, _i, _vp, _vp]),
    "aldic_inpaint_nans": (_i, [_vp, _i, _i, _vp, _vp]),
    "aldic_init_u0": (_i, [_vp, _i, _i, _vp, _vp, _i, _vp]),
    "aldic_remove_outliers": (_i, [_vp, _i, _i, _vp, _vp, _d, _i, _vp]),
    "aldic_subpb2_set_mesh": (_i, [_vp, _i64, _i64, _vp, _i64, _vp]),
    "aldic_sibson_weights": (_i, [_i64, _vp, _i64, _vp, _vp, _vp, _vp, _d, _i64, _vp, _vp, _i, _vp, _vp, _vp]),
    "aldic_subpb2": (_i, [_vp, _i64, _vp, _i64, _vp, _i, _d, _d, _d, _vp, _vp, _i64, _vp, _d, _i, _vp,
                          _vp]),
    "aldic_measure_fp32_peak": (_i, [_vp, C.POINTER(_d)]),
    "aldic_set_profiling": (_i, [_vp, _i]),
    "aldic_set_iteration_cap": (_i, [_vp, _i]),
    "aldic_set_fp64_band": (_i, [_vp, _d, _d]),
    "aldic_set_option": (_i, [_vp, _i, _i]),
    "aldic_get_option": (_i, [_vp, _i, C.POINTER(_i)]),
    "aldic_tuning_report": (_i, [_vp, C.c_char_p, _i64]),
    "aldic_profile_read": (_i, [_vp, C.POINTER(_d), C.POINTER(_i)]),
    "aldic_net_create": (_i, [C.POINTER(_vp), _i, _i]),
    "aldic_net_destroy": (None, [_vp]),
    "aldic_net_last_error": (C.c_char_p, [_vp]),
    "aldic_net_set_stream": (_i, [_vp, _vp]),
    "aldic_net_launch_count": (_i64, [_vp]),
    "aldic_net_param_count": (_i64, []),
    "aldic_net_set_params": (_i, [_vp, _vp]),
    "aldic_net_get_params": (_i, [_vp, _vp]),
    "aldic_net_forward": (_i, [_vp, _i, _vp, _vp]),
    "aldic_net_gradients": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "aldic_net_train_step": (_i, [_vp, _i, _vp, _vp, C.c_float, _vp]),
    "aldic_net_status": (_i, [_vp]),
    "aldic_net_predict": (_i, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "aldic_net_extract": (_i, [_vp, _i64, _vp, _vp]),
    "aldic_local_icgn_guess": (_i, [_vp, _i, _i64, _vp, _vp, _vp, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp]),
    "aldic_subset_zncc": (_i, [_vp, _i64, _vp, _vp, _vp, _i, _vp]),
    "aldic_fallback_select": (_i, [_vp, _i64, _vp, _vp, _d, _vp, _vp]),
    "aldic_integer_search_list": (_i, [_vp, _vp, _vp, _vp, _i, _i, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "aldic_gemm_bf16": (_i, [_vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp, _i64, _i, _vp]),
    "aldic_local_icgn_noalloc": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _i, _i, _i64, _vp, _vp, _i, _d, _vp, _vp, _vp,
                                      _vp, _vp, _vp]),
}

_LIB = None


class AldicError(RuntimeError):
    pass


def load(path: str | None = None):
    """Load the library once; raise AldicError (never fall back) when it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise AldicError(f"CUDA library not built: {p} (run __graft_entry__.build() or make -C 3d-stereo-aldic_b200)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib
