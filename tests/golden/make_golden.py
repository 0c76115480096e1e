"""Generate the interpolation golden vectors from the reference's own
ba_interp2_spline.cpp, compiled unmodified under oracle/_ref (make -C oracle ref).

    python tests/golden/make_golden.py

Writes tests/golden/interp_golden.npz: images F (column-major as stored), query points
X (dim-2) and Y (dim-1) in 1-based coordinates covering the interior, integer
positions, the clamped border band and points outside the image, and the reference's
output Z.  Seeds are fixed.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402


def main():
    if oracle.ref_lib() is None:
        raise SystemExit("build the reference library first: make -C oracle ref")
    rng = np.random.default_rng(20240925)
    cases = {}
    # speckle-like random image, 37 x 29
    F1 = rng.normal(0.0, 1.0, (37, 29)) * 40 + 100
    n = 3000
    X1 = np.concatenate([rng.uniform(1, 29, n), np.arange(1, 30, dtype=float), rng.uniform(-3, 33, 400)])
    Y1 = np.concatenate([rng.uniform(1, 37, n), np.linspace(1, 37, 29), rng.uniform(-3, 41, 400)])
    cases["speckle"] = (F1, X1, Y1)
    # linear ramp along dim 1 (the local stencil does not reproduce ramps exactly)
    F2 = np.add.outer(np.arange(1.0, 41.0), np.zeros(33)) * 1.5 + 7.0
    X2 = rng.uniform(4, 30, 500)
    Y2 = rng.uniform(4, 37, 500)
    cases["ramp"] = (F2, X2, Y2)
    # normalised uint8 speckle frame patch (the solver's input domain)
    raw = rng.integers(0, 256, (64, 48)).astype(np.float64)
    F3 = (raw - raw.mean()) / raw.std(ddof=1)
    X3 = rng.uniform(3, 46, 2000)
    Y3 = rng.uniform(3, 62, 2000)
    cases["normalised"] = (F3, X3, Y3)
    out = {}
    for name, (F, X, Y) in cases.items():
        out[f"{name}_F"] = F
        out[f"{name}_X"] = X
        out[f"{name}_Y"] = Y
        out[f"{name}_Z"] = oracle.ref_interp(F, X, Y)
    np.savez_compressed(os.path.join(HERE, "interp_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "interp_golden.npz"))


if __name__ == "__main__":
    main()
