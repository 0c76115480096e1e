"""B200 (sm_100a) implementation of the 3D-Stereo-ALDIC per-subset hot path.

The compute runs in the in-tree CUDA library libaldic_b200.so (C ABI:
include/aldic_b200.h); this package is its host-side mirror of the reference's MATLAB
interface (funIntegerSearch, LocalICGN, LocalICGNQuadtree, Subpb1, Subpb1Quadtree,
epipolar_ICGN1, stereoReconstruction_quadtree, ...).
"""
from ._lib import (DEFAULT_FP64_BAND, DEFAULT_FP64_NOISE, DEFAULT_ITERATION_CAP, OPT_AUTOTUNE, OPT_FP64_THREADS,  # noqa: F401
                   OPT_ITERATION_CAP, OPT_SEARCH_CHUNK, OPT_SLOW_FP64, OPT_SEARCH_IMPL, OPT_SLOW_WARPS, OPT_STAGING, QUADTREE, STAT_FP64_RESOLVES,
                   STAT_STAGING_TIMEOUT, UNIFORM, AldicError, load as load_library)
from .api import *  # noqa: F401,F403
from . import api, synth  # noqa: F401
