"""GPU tests of the learned initial guess's host-facing pieces: IC-GN started from [F0 U0]
against the FP64 oracle, the subset ZNCC check, the integer search on a list of grid subsets,
the network's input patches and prediction, and a short training run that shows what the
trained network gains over the integer-search initial guess on a held-out frame."""
import numpy as np
import pytest

import cnn_oracle as CO
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import aldic_b200 as A
    from aldic_b200 import synth_gpu

    O.build()
    pair = synth_gpu.field_pair(7, M=256, N=256, umax=6.0, gmax=0.04)
    ctx = A.Context(0)
    M, N = pair.M, pair.N
    ctx.load_image_raw(0, pair.ref, [1, M], [1, N], want_stats=False, shape=(M, N))
    ctx.load_image_raw(1, pair.deff, [1, M], [1, N], want_stats=False, shape=(M, N))
    ctx.compute_gradients()
    ref = pair.ref.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    deff = pair.deff.cpu().numpy().reshape((M, N), order="F").astype(np.float64)
    f, _ = O.normalize(ref, [1, M], [1, N])
    g, _ = O.normalize(deff, [1, M], [1, N])
    gx, gy = O.gradient(f)
    yield {"A": A, "torch": torch, "pair": pair, "ctx": ctx, "f": f, "g": g,
           "frame": O.Frame(f, g, None, gx, gy)}
    ctx.close()


def _nodes(M, N, w=32, step=12):
    from aldic_b200.learned import grid_nodes

    return grid_nodes(M, N, w, step).T.copy()  # n x 2


def test_icgn_from_a_gradient_guess_matches_the_oracle(env):
    A, ctx, pair = env["A"], env["ctx"], env["pair"]
    crd = _nodes(pair.M, pair.N)
    n = crd.shape[0]
    u, v = pair.field.disp(crd[:, 0], crd[:, 1])
    rng = np.random.default_rng(1)
    U0 = (np.stack([u, v], 1) + rng.uniform(-0.6, 0.6, (n, 2))).ravel()
    F0 = (pair.field.grad(crd[:, 0], crd[:, 1]) + rng.uniform(-0.01, 0.01, (n, 4))).ravel()
    for variant in (A.UNIFORM, A.QUADTREE):
        d = ctx.local_icgn(variant, crd, U0, 32, 1e-3, F0=F0)
        o = O.local_icgn(env["frame"], crd, U0, 32, 1e-3, variant=variant, F0=F0)
        fg = (d["conv"] > 0) & (d["conv"] < 100)
        fo = (o["conv"] > 0) & (o["conv"] < 100)
        assert fg.mean() > 0.95
        assert np.mean(fg == fo) >= 0.999
        both = fg & fo
        assert np.abs(d["U"] - o["U"]).reshape(-1, 2)[both].max() <= 1e-3
        assert np.abs(d["F"] - o["F"]).reshape(-1, 4)[both].max() <= 1e-4
        assert np.mean(d["conv"] == o["conv"]) >= 0.99


def test_zero_gradient_guess_is_the_reference_start(env):
    A, ctx, pair = env["A"], env["ctx"], env["pair"]
    crd = _nodes(pair.M, pair.N)
    n = crd.shape[0]
    u, v = pair.field.disp(crd[:, 0], crd[:, 1])
    U0 = np.round(np.stack([u, v], 1)).ravel()
    a = ctx.local_icgn(A.QUADTREE, crd, U0, 32, 1e-3)
    b = ctx.local_icgn(A.QUADTREE, crd, U0, 32, 1e-3, F0=np.zeros(4 * n))
    for k in ("U", "F", "conv"):
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_subset_zncc_matches_numpy(env):
    ctx, pair = env["ctx"], env["pair"]
    crd = _nodes(pair.M, pair.N)
    n = crd.shape[0]
    u, v = pair.field.disp(crd[:, 0], crd[:, 1])
    U = np.stack([u, v], 1)
    F = pair.field.grad(crd[:, 0], crd[:, 1])
    z = ctx.subset_zncc(crd, U.ravel(), F.ravel(), 32)
    f, g, w = env["f"], env["g"], 32
    h = w // 2
    d = np.arange(-h, h + 1, dtype=np.float64)
    DX, DY = np.meshgrid(d, d, indexing="ij")  # dim 1, dim 2
    want = np.empty(n)
    for t in range(n):
        x0, y0 = crd[t]
        fx = f[int(x0) - h - 1:int(x0) + h, int(y0) - h - 1:int(y0) + h]
        X = x0 + DX + F[t, 0] * DX + F[t, 2] * DY + U[t, 0]
        Y = y0 + DY + F[t, 3] * DY + F[t, 1] * DX + U[t, 1]
        gx = O.interp(g, Y, X).reshape(DX.shape)
        a, b = fx - fx.mean(), gx - gx.mean()
        want[t] = (a * b).sum() / np.sqrt((a * a).sum() * (b * b).sum())
    assert np.all(np.isfinite(z))
    assert np.abs(z - want).max() < 1e-5
    assert z.min() > 0.9  # the analytic warp matches
    # a warp off by 3 px decorrelates the speckle
    z2 = ctx.subset_zncc(crd, (U + 3.0).ravel(), F.ravel(), 32)
    assert np.median(z2) < 0.5


def test_list_search_matches_the_whole_grid(env):
    torch, ctx = env["torch"], env["ctx"]
    M = N = 256
    gx, gy, w, st = [17, M - 16], [17, N - 16], 32, 16
    full = ctx.integer_search([8, 8], gx, gy, w, st)
    nx, ny = ctx.search_grid(gx, gy, w, st)
    rng = np.random.default_rng(3)
    idx = rng.choice(nx * ny, size=min(37, nx * ny), replace=False).astype(np.int32)
    lst = ctx.integer_search_list([8, 8], gx, gy, w, st, idx)
    for k in ("x", "y", "u", "v", "phi"):
        want = full[k].ravel()[idx]  # the (nY, nX) grid in list order i + j nX
        assert np.array_equal(lst[k], want, equal_nan=True), k
    # device list and outputs
    dev = torch.device("cuda:0")
    out = {k: torch.empty(idx.size, dtype=torch.float64, device=dev) for k in ("x", "y", "u", "v", "phi")}
    ctx.integer_search_list([8, 8], gx, gy, w, st, torch.from_numpy(idx).to(dev), out=out)
    ctx.synchronize()
    for k in out:
        assert np.array_equal(out[k].cpu().numpy(), lst[k], equal_nan=True), k
    # the grid centres are the search's x, y
    from aldic_b200.learned import search_nodes

    nodes, nx2, ny2 = search_nodes(gx, gy, w, st)
    assert (nx2, ny2) == (nx, ny)
    assert np.array_equal(nodes[0], full["x"].ravel())
    assert np.array_equal(nodes[1], full["y"].ravel())


def _patches_numpy(f, g, crd):
    M, N = f.shape
    out = np.zeros((crd.shape[0], 64, 64, 2))
    for t, (x, y) in enumerate(crd):
        x0, y0 = int(round(x)), int(round(y))
        ri = np.clip(np.arange(x0 - 32, x0 + 32), 1, M) - 1
        ci = np.clip(np.arange(y0 - 32, y0 + 32), 1, N) - 1
        d = g[np.ix_(ri, ci)]
        r = f[np.ix_(ri[16:48], ci[16:48])]
        out[t, :, :, 1] = (d - d.mean()) / np.sqrt(max(d.var(), 1e-12))
        out[t, 16:48, 16:48, 0] = (r - r.mean()) / np.sqrt(max(r.var(), 1e-12))
    return out


def test_network_patches_and_prediction(env):
    torch, ctx, pair = env["torch"], env["ctx"], env["pair"]
    from aldic_b200.learned import ProposalNet

    dev = torch.device("cuda:0")
    crd = _nodes(pair.M, pair.N, step=10)[:150]
    crd[-1] = [3.0, 250.0]  # a window clamped at the image border
    n = crd.shape[0]
    ct = torch.from_numpy(np.ascontiguousarray(crd.T)).to(dev)
    X = torch.empty((n, 64, 64, 2), dtype=torch.bfloat16, device=dev)
    ctx.net_extract(ct, X)
    ctx.synchronize()
    got = X.float().cpu().numpy()
    want = CO.bf16(_patches_numpy(env["f"], env["g"], crd).astype(np.float32))
    same = got == want
    assert same.mean() > 0.999
    assert np.abs(got - want).max() <= 2.0 ** -7 * max(1.0, np.abs(want).max())
    net = ProposalNet(0, max_batch=64, seed=5)
    try:
        b = {"U0": torch.empty(2 * n, dtype=torch.float64, device=dev),
             "F0": torch.empty(4 * n, dtype=torch.float64, device=dev)}
        net.predict(ctx, ct, b)
        ctx.synchronize()
        Y = torch.empty((n + 2, 6), dtype=torch.float32, device=dev)
        Xp = torch.cat([X, X[:2]])  # a multiple of 8 rows
        for s in range(0, n + 2, 64):
            e = min(s + 64, n + 2)
            net.forward(Xp[s:e].contiguous(), Y[s:e])
        torch.cuda.synchronize()
        y = Y[:n].cpu().numpy().astype(np.float64)
        assert np.array_equal(b["U0"].cpu().numpy().reshape(n, 2), 8.0 * y[:, :2].astype(np.float32))
        F0 = b["F0"].cpu().numpy().reshape(n, 4)
        assert np.abs(F0 - y[:, 2:] / 20.0).max() <= 1e-7 * max(1.0, np.abs(y).max())
    finally:
        net.close()


def test_trained_network_beats_the_search_guess():
    """Train on six 512 x 512 speckle pairs (labels: converged IC-GN from the analytic guess),
    then on a held-out pair: IC-GN from the network's guess converges on at least as many
    subsets as from the integer search's guess, in fewer iterations, with few fallbacks."""
    import torch

    import aldic_b200 as A
    from aldic_b200 import learned as L
    from aldic_b200 import synth_gpu

    ctx = A.Context(0)
    net = L.ProposalNet(0, max_batch=512, seed=0)
    try:
        Xs, Ts = [], []
        for s in range(6):
            X, T = L.label_pair(ctx, synth_gpu.field_pair(100 + s, M=512, N=512), w=32, step=6)
            Xs.append(X)
            Ts.append(T)
        X, T = torch.cat(Xs), torch.cat(Ts)
        log = L.train(net, X, T, steps=1500, batch=256, lr=2e-3, lr_end=2e-5)
        assert log[-1][1] < 0.2 * log[0][1]
        pair = synth_gpu.field_pair(999, M=512, N=512)
        M, N = pair.M, pair.N
        gx, gy, w, st, s = [17, M - 16], [17, N - 16], 32, 16, 16
        ctx.load_image_raw(0, pair.ref, gx, gy, want_stats=False, shape=(M, N))
        ctx.load_image_raw(1, pair.deff, gx, gy, want_stats=False, shape=(M, N))
        ctx.compute_gradients()
        li = L.LearnedInit(net, ctx, s, gx, gy, w, st, 1e-3)
        nf = li.run()
        li.stream.synchronize()
        conv_l = li.buf["conv"].cpu().numpy()
        # the reference's start: the integer search, outliers removed, inpainted, F = 0
        r = ctx.integer_search([s, s], gx, gy, w, st)
        u, v, _ = O.remove_outliers(r["u"], r["v"], 100.0)
        U0 = O.init_u0(u, v)
        crd = li.coords.cpu().numpy().T.copy()
        f = ctx.local_icgn(A.QUADTREE, crd, U0, w, 1e-3, want_H=False)
        ok_l = (conv_l > 0) & (conv_l < 100)
        ok_f = (f["conv"] > 0) & (f["conv"] < 100)
        assert ok_l.sum() >= ok_f.sum()
        both = ok_l & ok_f
        it_l, it_f = conv_l[both].mean(), f["conv"][both].mean()
        assert it_l < it_f, (it_l, it_f)
        assert nf <= 0.1 * li.n
        d = np.abs(li.buf["U"].cpu().numpy() - f["U"]).reshape(-1, 2)[both]
        assert np.median(d) < 1e-3
    finally:
        net.close()
        ctx.close()
