"""CPU tests of the C ABI boundary: the library loads, exports every symbol that
include/aldic_b200.h declares, and fails loudly (no CPU fallback) without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aldic_b200.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(aldic_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import aldic_b200

    lib = aldic_b200.load_library()
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    from aldic_b200 import _lib

    assert set(names) == set(_lib.SIGNATURES), "ctypes signatures out of sync with the header"


def test_abi_version_and_grid_without_device():
    import aldic_b200

    lib = aldic_b200.load_library()
    assert lib.aldic_abi_version() == 1
    gx = np.array([1, 512], dtype=np.int32)
    gy = np.array([1, 512], dtype=np.int32)
    nx, ny = C.c_int(), C.c_int()
    rc = lib.aldic_search_grid(C.c_void_p(gx.ctypes.data), C.c_void_p(gy.ctypes.data), 30, 16, C.byref(nx),
                               C.byref(ny))
    assert rc == 0 and (nx.value, ny.value) == (30, 30)  # XList = 1:16:466 (funIntegerSearch.m:106)


def test_grid_matches_oracle():
    import aldic_b200
    import oracle as O

    lib = aldic_b200.load_library()
    for gx, gy, w, st in (([1, 2048], [1, 2048], 40, 10), ([5, 300], [9, 280], 20, 7), ([1, 60], [1, 60], 40, 30)):
        a = np.array(gx, dtype=np.int32)
        b = np.array(gy, dtype=np.int32)
        nx, ny = C.c_int(), C.c_int()
        lib.aldic_search_grid(C.c_void_p(a.ctypes.data), C.c_void_p(b.ctypes.data), w, st, C.byref(nx), C.byref(ny))
        assert (nx.value, ny.value) == O.search_grid(gx, gy, w, st)


def test_no_cpu_fallback_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import aldic_b200

    with pytest.raises(aldic_b200.AldicError):
        aldic_b200.Context(0)
    with pytest.raises(aldic_b200.AldicError):
        aldic_b200.ba_interp2_spline(np.zeros((10, 10)), [1.0], [1.0])


def test_null_context_is_rejected():
    import aldic_b200

    lib = aldic_b200.load_library()
    assert lib.aldic_compute_gradients(None) == 1
    assert lib.aldic_local_icgn(None, 1, 0, None, None, 30, 1e-3, None, None, None, None, None) == 1
    assert lib.aldic_last_error(None) == b"null context"


def test_package_exports_the_names_callers_use():
    # the names __graft_entry__.smoke() and MATLAB-style callers take from the package
    import aldic_b200 as A

    assert (A.UNIFORM, A.QUADTREE) == (0, 1)
    for name in ("Context", "AldicError", "load_library", "LocalICGNQuadtree", "funIntegerSearch", "synth"):
        assert hasattr(A, name), name
    # the Python copy of the library's default iteration cap matches the C constant
    src = open(os.path.join(ROOT, "3d-stereo-aldic_b200", "csrc", "kernels.h")).read()
    cap = int(re.search(r"constexpr int kDefaultWarpCap = (\d+);", src).group(1))
    assert A.DEFAULT_ITERATION_CAP == cap


def test_output_arrays_are_written_in_place_or_refused():
    """Host outputs passed through `out=` must be the exact arrays the library writes:
    a conversion would leave the results in a temporary, so it is refused."""
    from aldic_b200.api import AldicError, _Keep

    k = _Keep()
    good = np.empty(10, dtype=np.float64)
    assert k.dst(good, np.float64, 10).value == good.ctypes.data
    fcol = np.empty((5, 2), dtype=np.float64, order="F")
    assert k.dst(fcol, np.float64, 10).value == fcol.ctypes.data
    assert k.dst(None, np.float64, 10) is None
    bad = [np.empty(10, dtype=np.float32),            # would need a conversion
           np.empty((10, 2), dtype=np.float64)[:, 0],  # strided view
           np.empty(9, dtype=np.float64),             # too small
           [0.0] * 10]                                # not an array
    ro = np.empty(10, dtype=np.float64)
    ro.flags.writeable = False
    bad.append(ro)
    for b in bad:
        with pytest.raises(AldicError):
            k.dst(b, np.float64, 10)
