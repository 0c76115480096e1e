"""CPU check of the tile search's shared-product algebra.

The two passes of the tile kernel (row-band sums per tile row, then block sums over rows)
are compiled for the host from the library source and compared with FP64 direct window
sums on random tiles, for every (step, window) shape that has a tile kernel.  No GPU is
involved: this pins the index arithmetic of the shared products before any device run.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host", "tile_passes_check.cu")


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_tile_passes_match_direct_window_sums(tmp_path):
    exe = str(tmp_path / "tile_passes_check")
    cmd = ["nvcc", "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-o", exe, SRC]
    build = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert build.returncode == 0, build.stderr[-2000:]
    run = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.count("0 of") == 7, run.stdout
