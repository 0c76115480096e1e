"""CPU checks of ALDIC's global step (Subpb2Quadtree).

The oracle's restatement is checked against closed forms: a linear displacement field with
its own constant gradient as F comes back exactly at every Gauss order (the hanging-node
shape functions are linearly complete), beta = 0 gives Uhat = U, and dirichlet nodes keep
U.  The library's element rows, mesh tables and conjugate-gradient steps (subpb2.cu,
compiled for the host) are then compared with the oracle on quadtree meshes with hanging
nodes.  No GPU is involved.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "host", "subpb2_check.cu")


def quadtree_mesh(nc, refine, h=8.0, origin=10.0):
    """A one-level quadtree mesh over nc x nc coarse cells of size 2h: the cells in `refine`
    (set of (i, j)) are split in four; an unrefined cell takes a refined neighbour's edge
    midpoint as its hanging node (slot 5 right, 6 top, 7 left, 8 bottom edge)."""
    P = {}

    def node(x, y):
        return P.setdefault((x, y), len(P) + 1)

    E = []
    for j in range(nc):
        for i in range(nc):
            x0, y0 = 2 * i, 2 * j
            if (i, j) in refine:
                for dx, dy in ((0, 0), (1, 0), (1, 1), (0, 1)):
                    a, b = x0 + dx, y0 + dy
                    E.append([node(a, b), node(a + 1, b), node(a + 1, b + 1), node(a, b + 1), 0, 0, 0, 0])
            else:
                E.append([node(x0, y0), node(x0 + 2, y0), node(x0 + 2, y0 + 2), node(x0, y0 + 2), 0, 0, 0, 0])
    # hanging nodes: midpoints of unrefined cells' edges that a refined neighbour created
    k = 0
    for j in range(nc):
        for i in range(nc):
            x0, y0 = 2 * i, 2 * j
            if (i, j) in refine:
                k += 4
                continue
            for slot, mid in ((4, (x0 + 2, y0 + 1)), (5, (x0 + 1, y0 + 2)), (6, (x0, y0 + 1)), (7, (x0 + 1, y0))):
                if mid in P:
                    E[k][slot] = P[mid]
            k += 1
    C = np.zeros((len(P), 2))
    for (x, y), idx in P.items():
        C[idx - 1] = (origin + h * x, origin + h * y)
    return C, np.array(E, dtype=np.int64)


def _linear_case(C):
    n = C.shape[0]
    G = np.array([[0.01, -0.02], [0.03, 0.005]])
    U = np.zeros(2 * n)
    U[0::2] = 3 + C @ G[0]
    U[1::2] = -1 + C @ G[1]
    F = np.zeros(4 * n)
    F[0::4], F[1::4], F[2::4], F[3::4] = G[0, 0], G[1, 0], G[0, 1], G[1, 1]
    return U, F


def test_mesh_has_hanging_nodes():
    C, E = quadtree_mesh(4, {(1, 1), (2, 1)})
    assert (E[:, 4:] > 0).sum() >= 4


@pytest.mark.parametrize("order", [2, 3, 4, 5])
def test_oracle_patch_test(order):
    C, E = quadtree_mesh(4, {(1, 1), (2, 2)})
    U, F = _linear_case(C)
    assert np.abs(O.subpb2_quadtree(C, E, order, 0.064, 1e-3, U, F) - U).max() < 1e-12


def test_oracle_mass_only_and_dirichlet():
    C, E = quadtree_mesh(3, {(1, 1)})
    n = C.shape[0]
    rng = np.random.default_rng(0)
    U = rng.standard_normal(2 * n)
    assert np.abs(O.subpb2_quadtree(C, E, 2, 0.0, 1e-3, U, np.zeros(4 * n)) - U).max() < 1e-12
    Uh = O.subpb2_quadtree(C, E, 2, 0.064, 1e-3, U, rng.standard_normal(4 * n), dirichlet=[1, 5])
    assert np.array_equal(Uh[[0, 1, 8, 9]], U[[0, 1, 8, 9]])


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("sp2") / "subpb2_check")
    cmd = ["nvcc", "-std=c++17", "-O1", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
           "-o", exe, SRC]
    b = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert b.returncode == 0, b.stderr[-2000:]
    return exe


def _run(exe, tmp_path, C, E, order, beta, mu, alpha, U, F, dirichlet=(), tol=1e-13):
    n, n_el = C.shape[0], E.shape[0]
    d = np.asarray(dirichlet, dtype=np.int32).ravel()
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(np.array([n, n_el, d.size], np.int64).tobytes())
        f.write(np.array([order], np.int32).tobytes())
        f.write(np.array([beta, mu, alpha, tol], np.float64).tobytes())
        f.write(C.ravel(order="F").tobytes())
        f.write(E.astype(np.int32).ravel(order="F").tobytes())
        f.write(np.asarray(U, np.float64).tobytes())
        f.write(np.asarray(F, np.float64).tobytes())
        f.write(d.tobytes())
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = open(fout, "rb").read()
    Ke = np.frombuffer(raw, np.float64, 64 * n_el, 0).reshape(n_el, 8, 8)
    off = 64 * n_el * 8
    be = np.frombuffer(raw, np.float64, 16 * n_el, off).reshape(n_el, 16)
    off += 16 * n_el * 8
    x = np.frombuffer(raw, np.float64, 2 * n, off)
    off += 2 * n * 8
    it, ok = np.frombuffer(raw, np.int32, 2, off)
    kind = np.frombuffer(raw, np.int32, n, off + 8)
    return Ke, be, x, int(it), int(ok), kind


@pytest.mark.parametrize("order", [2, 3, 4, 5])
def test_element_rows_match_the_oracle(harness, tmp_path, order):
    C, E = quadtree_mesh(4, {(1, 1), (2, 1), (0, 3)})
    n = C.shape[0]
    rng = np.random.default_rng(order)
    U, F = rng.standard_normal(2 * n), rng.standard_normal(4 * n)
    beta, mu, alpha = 0.0512, 1e-3, 0.003
    Ke, be, _, _, _, _ = _run(harness, tmp_path, C, E, order, beta, mu, alpha, U, F)
    for e in range(E.shape[0]):
        ids = E[e]
        present = [ids[k] != 0 for k in range(4, 8)]
        xy = np.array([C[i - 1] if i else (0.0, 0.0) for i in ids])
        A, gp = O.subpb2_element(xy, present, order, beta, mu, alpha)
        # K_e (x) I_2 in the reference's [x1 y1 x2 y2 ...] dof order
        assert np.allclose(A[0::2, 0::2], Ke[e], rtol=1e-13, atol=1e-15)
        assert np.allclose(A[1::2, 1::2], Ke[e], rtol=1e-13, atol=1e-15)
        assert np.abs(A[0::2, 1::2]).max() == 0 and np.abs(A[1::2, 0::2]).max() == 0
        ue = np.array([U[2 * (i - 1) + c] if i else 0.0 for i in ids for c in (0, 1)])
        Fr = np.zeros((16, 4))
        for k, i in enumerate(ids):
            if i:
                a = i - 1
                Fr[2 * k] = Fr[2 * k + 1] = [F[4 * a], F[4 * a + 2], F[4 * a + 1], F[4 * a + 3]]
        want = O.subpb2_element_rhs(gp, beta, mu, alpha, ue, Fr)
        assert np.allclose(be[e], want, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("order,dirichlet", [(2, ()), (2, (3, 7, 12)), (3, (1,))])
def test_solution_matches_the_direct_solve(harness, tmp_path, order, dirichlet):
    C, E = quadtree_mesh(5, {(1, 1), (2, 1), (3, 3)})
    n = C.shape[0]
    rng = np.random.default_rng(7)
    U = 2.0 + rng.standard_normal(2 * n)
    F = 0.01 * rng.standard_normal(4 * n)
    beta, mu = 1e-2 * 16 ** 2 * 1e-3, 1e-3
    _, _, x, it, ok, kind = _run(harness, tmp_path, C, E, order, beta, mu, 0.0, U, F, dirichlet)
    ref = O.subpb2_quadtree(C, E, order, beta, mu, U, F, dirichlet=dirichlet)
    assert ok == 1 and 0 < it < 2 * n
    assert np.abs(x - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())
    want = np.zeros(n, np.int32)
    want[np.unique(E)[1:] - 1] = 1
    want[np.asarray(dirichlet, dtype=np.int64) - 1] = 2
    assert np.array_equal(kind, want)


def test_patch_test_through_the_library_steps(harness, tmp_path):
    C, E = quadtree_mesh(4, {(0, 0), (3, 2)})
    U, F = _linear_case(C)
    _, _, x, _, ok, _ = _run(harness, tmp_path, C, E, 2, 0.256, 1e-3, 0.0, U, F)
    assert ok == 1 and np.abs(x - U).max() < 1e-9


def _plate_mesh(min_size=4):
    import aldic_b200 as A
    from aldic_b200 import synth

    sc = synth.plate_with_hole(size=384, hole_r=60.0, peak=2.0, sin_amp=0.3, sin_wl=120.0)
    w, st = 32, 16
    xl = np.arange(1 + w // 2, 384 - w // 2 + 1, st, dtype=float)
    X, Y = np.meshgrid(xl, xl)
    mesh = A.MeshSetUp(X, Y, {"winstepsize": st, "ImgSize": [384, 384]})
    mesh["elementMinSize"] = min_size
    C0 = mesh["coordinatesFEM"]
    U0 = np.stack([0.5 + 0.01 * C0[:, 0] - 0.002 * C0[:, 1], -1.0 + 0.003 * C0[:, 1]], 1).ravel()
    m2, _, U = A.GenerateQuadtreeMesh(U0, None, sc.mask, mesh, {"winstepsize": st, "winsize": w})
    return sc.mask, mesh, m2, U


def test_quadtree_mesh_structure():
    mask, mesh0, m, U = _plate_mesh()
    C, E = m["coordinatesFEM"], m["elementsFEM"]
    n0 = mesh0["coordinatesFEM"].shape[0]
    assert np.array_equal(C[:n0], mesh0["coordinatesFEM"])  # old nodes keep their numbers
    x1, y1 = C[E[:, 0] - 1].T
    x2, y2 = C[E[:, 1] - 1].T
    x3, y3 = C[E[:, 2] - 1].T
    x4, y4 = C[E[:, 3] - 1].T
    s = x2 - x1
    # squares, corners (xmin, ymin), (xmax, ymin), (xmax, ymax), (xmin, ymax)
    assert (s > 0).all() and np.array_equal(y2, y1) and np.array_equal(x3, x2) and np.array_equal(y3 - y2, s)
    assert np.array_equal(x4, x1) and np.array_equal(y4, y3)
    assert set(np.unique(s)) == {4.0, 8.0, 16.0}
    # hanging nodes sit at the midpoints of their edges; no other node lies inside any edge
    mids = {4: ((x2 + x3) / 2, (y2 + y3) / 2), 5: ((x3 + x4) / 2, (y3 + y4) / 2), 6: ((x4 + x1) / 2, (y4 + y1) / 2),
            7: ((x1 + x2) / 2, (y1 + y2) / 2)}
    for slot, (mx, my) in mids.items():
        h = E[:, slot] > 0
        assert np.array_equal(C[E[h, slot] - 1, 0], mx[h]) and np.array_equal(C[E[h, slot] - 1, 1], my[h])
    pts = {tuple(p) for p in C}
    for e in range(E.shape[0]):
        q = s[e] / 4  # a 2-irregular edge would have nodes at the quarter points
        for (ax, ay), (bx, by) in (((x1[e], y1[e]), (x2[e], y2[e])), ((x2[e], y2[e]), (x3[e], y3[e])),
                                   ((x3[e], y3[e]), (x4[e], y4[e])), ((x4[e], y4[e]), (x1[e], y1[e]))):
            for t in (0.25, 0.75):
                assert (ax + t * (bx - ax), ay + t * (by - ay)) not in pts, (e, q)
    # refinement finished: no kept element larger than the minimum still meets both mask values
    for e in range(E.shape[0]):
        blk = mask[int(x1[e]) - 1:int(x2[e]), int(y1[e]) - 1:int(y4[e])]
        assert not (s[e] > 4 and blk.max() > blk.min())
        assert blk.sum() >= 0.5 * s[e] * s[e]  # funMarkInside kept it
    # the dirichlet set holds the nodes of every refined element
    fine = E[s < 16][:, :4].ravel()
    assert np.isin(fine, m["dirichlet"]).all()
    # U0 (linear in x, y) carried exactly to the new nodes
    want = np.stack([0.5 + 0.01 * C[:, 0] - 0.002 * C[:, 1], -1.0 + 0.003 * C[:, 1]], 1).ravel()
    assert np.abs(U - want).max() < 1e-12


def test_generated_mesh_passes_the_global_step_patch_test():
    _, _, m, _ = _plate_mesh()
    C, E = m["coordinatesFEM"], m["elementsFEM"]
    U, F = _linear_case(C)
    Uh = O.subpb2_quadtree(C, E, 2, 0.0256, 1e-3, U, F, dirichlet=m["dirichlet"])
    used = np.unique(E[E > 0]) - 1
    d = np.abs(Uh - U).reshape(-1, 2)[used]
    assert d.max() < 1e-10


def test_quadtree_mesh_nonbinary_mask_and_integer_corners():
    import aldic_b200 as A
    from aldic_b200 import synth

    sc = synth.plate_with_hole(size=256, hole_r=40.0, peak=1.0, sin_amp=0.1, sin_wl=100.0)
    w, st = 32, 16
    xl = np.arange(1 + w // 2, 256 - w // 2 + 1, st, dtype=float)
    X, Y = np.meshgrid(xl, xl)
    mesh = A.MeshSetUp(X, Y, {"winstepsize": st, "ImgSize": [256, 256]})
    mesh["elementMinSize"] = 4
    para = {"winstepsize": st, "winsize": w}
    U0 = np.zeros(2 * mesh["coordinatesFEM"].shape[0])
    mask = sc.mask * 0.7 + 0.2  # two levels, not 0 / 1: the min / max and sum rules on values
    m, _, _ = A.GenerateQuadtreeMesh(U0, None, mask, mesh, para)
    C, E = m["coordinatesFEM"], m["elementsFEM"]
    for e in range(E.shape[0]):
        x0, y0 = C[E[e, 0] - 1].astype(int)
        x1, y1 = C[E[e, 2] - 1].astype(int)
        blk = mask[x0 - 1:x1, y0 - 1:y1]
        assert not (x1 - x0 > 4 and blk.max() > blk.min())          # nothing left to refine
        assert blk.sum() >= 0.5 * (x1 - x0) * (y1 - y0)              # funMarkInside kept it
    assert (E[:, 4:] > 0).any()
    # a minimum size that halves 16-px elements into 2-px ones reaches 1-px corners only
    # through non-integer boxes for odd sizes: step 10 -> 5 -> 2.5 must raise
    xl10 = np.arange(1 + w // 2, 256 - w // 2 + 1, 10, dtype=float)
    X10, Y10 = np.meshgrid(xl10, xl10)
    mesh10 = A.MeshSetUp(X10, Y10, {"winstepsize": 10, "ImgSize": [256, 256]})
    mesh10["elementMinSize"] = 2
    with pytest.raises(A.AldicError):
        A.GenerateQuadtreeMesh(np.zeros(2 * mesh10["coordinatesFEM"].shape[0]), None, sc.mask, mesh10,
                               {"winstepsize": 10, "winsize": w})
