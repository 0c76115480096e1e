"""CPU checks of the benchmark's workload arithmetic: the solve mesh is the library's search
grid (XList rule), the roofline's FLOP count is the tile kernel's shape, every workload is
defined, and the measured correlation-kernel traffic covers the stereo workloads."""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_mesh_is_the_library_search_grid():
    import aldic_b200

    lib = aldic_b200.load_library()
    for M, N, w, st in ((2048, 2048, 40, 10), (512, 512, 30, 16), (4096, 3000, 40, 10), (330, 300, 24, 7)):
        coords, nx, ny = bench.grid_coords(M, N, w, st)
        gx = np.array([1, M], dtype=np.int32)
        gy = np.array([1, N], dtype=np.int32)
        cnx, cny = C.c_int(), C.c_int()
        assert lib.aldic_search_grid(gx.ctypes.data_as(C.c_void_p), gy.ctypes.data_as(C.c_void_p), w, st,
                                     C.byref(cnx), C.byref(cny)) == 0
        assert (nx, ny) == (cnx.value, cny.value)
        assert coords.shape == (nx * ny, 2)
        # XList fastest, subset centres at x0 + w/2
        assert coords[1, 0] - coords[0, 0] == st and coords[1, 1] == coords[0, 1]
        assert coords[0, 0] == 1 + w / 2.0


def test_roofline_flops_follow_the_tile_shape():
    # stereo2048: tiles of 9 x 8 subsets (121 x 111 pixels), 200 x 200 subsets -> 23 x 25 tiles,
    # (70 + 70 + 3)^2 shifts, 2 flops per product
    assert bench.tile_flops(2048, 2048, 40, 10, 70, 70) == 2.0 * 121 * 111 * 143 ** 2 * (23 * 25)


def test_workloads_are_defined():
    for name in ("stereo2048", "stereo1024", "temporal512", "quadtree2048", "sequence4096"):
        P = bench.workload_params(name)
        assert P["w"] % 2 == 0 and P["step"] > 0
    assert set(bench.TILE_TRAFFIC) == {"stereo2048", "stereo1024"}


def test_admm_beta_follows_the_reference_rule():
    import bench

    betas = [c * 16.0 ** 2 * 1e-3 for c in (1e-3, 1e-2, 1e-1)]
    assert bench.admm_beta(betas, [1.0, 2.0, 3.0]) == betas[0]
    assert bench.admm_beta(betas, [3.0, 2.0, 1.0]) == betas[2]
    # minimum in the middle: the vertex of the parabola through the normalised errors
    errs = [2.0, 1.0, 1.5]
    b = bench.admm_beta(betas, errs)
    x = np.log10(betas)
    z = (np.array(errs) - np.mean(errs)) / np.std(errs, ddof=1)
    p = np.polyfit(x, z, 2)
    assert abs(np.log10(b) - (-p[1] / (2 * p[0]))) < 1e-12 and x[0] < np.log10(b) < x[2]
    assert bench.admm_beta(betas, [1.0, 1.0, 1.0]) == betas[0]  # no spread: MATLAB's min of NaN
