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


def test_icgn_zncc_output_is_the_final_warps_zncc(env):
    """The ZNCC IC-GN returns from its last iteration's sums equals the ZNCC of the returned
    [F U] (aldic_subset_zncc) on converged subsets, changes no other output, and is NaN for a
    subset no pass solves (its window leaves the image)."""
    A, ctx, pair = env["A"], env["ctx"], env["pair"]
    crd = np.vstack([_nodes(pair.M, pair.N), [[6.0, 6.0]]])
    n = crd.shape[0]
    u, v = pair.field.disp(crd[:, 0], crd[:, 1])
    rng = np.random.default_rng(5)
    U0 = (np.stack([u, v], 1) + rng.uniform(-0.6, 0.6, (n, 2))).ravel()
    F0 = (pair.field.grad(crd[:, 0], crd[:, 1]) + rng.uniform(-0.01, 0.01, (n, 4))).ravel()
    for variant in (A.UNIFORM, A.QUADTREE):
        a = ctx.local_icgn(variant, crd, U0, 32, 1e-3, F0=F0, want_H=False)
        d = ctx.local_icgn(variant, crd, U0, 32, 1e-3, F0=F0, want_H=False, want_zncc=True)
        for k in ("U", "F", "conv"):
            assert np.array_equal(a[k], d[k], equal_nan=True), k
        ok = (d["conv"] > 0) & (d["conv"] < 100)
        assert ok[:-1].mean() > 0.95 and not ok[-1]
        z = ctx.subset_zncc(crd, d["U"], d["F"], 32)
        assert np.abs(d["zncc"] - z)[ok].max() < 1e-5
        assert d["zncc"][ok].min() > 0.9
        assert np.isnan(d["zncc"][-1])
    with pytest.raises(ValueError):
        ctx.local_icgn(A.UNIFORM, crd, U0, 32, 1e-3, want_zncc=True)


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
    for k in ("x", "y", "u", "v"):
        want = full[k].ravel()[idx]  # the (nY, nX) grid in list order i + j nX
        assert np.array_equal(lst[k], want, equal_nan=True), k
    # the peak ZNCC: the list runs the direct correlation, the whole grid the shared-product
    # kernel, whose sums round differently
    assert np.abs(lst["phi"] - full["phi"].ravel()[idx]).max() < 1e-6
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


def test_fallback_selection(env):
    torch, ctx = env["torch"], env["ctx"]
    rng = np.random.default_rng(5)
    n = 5000
    conv = rng.integers(-1, 103, n).astype(np.int32)
    zncc = rng.uniform(0.5, 1.0, n)
    zncc[rng.choice(n, 40, replace=False)] = np.nan
    want = np.flatnonzero((conv < 1) | (conv > 100) | ~(zncc >= 0.9))
    out = np.empty(n, dtype=np.int32)
    k = ctx.fallback_select(conv, zncc, 0.9, out)
    assert k == want.size and np.array_equal(np.sort(out[:k]), want)
    dev = torch.device("cuda:0")
    outd = torch.empty(n, dtype=torch.int32, device=dev)
    k2 = ctx.fallback_select(torch.from_numpy(conv).to(dev), torch.from_numpy(zncc).to(dev), 0.9, outd)
    assert k2 == k and np.array_equal(np.sort(outd[:k2].cpu().numpy()), want)
    # the count on the device: queued without a wait
    cnt = torch.full((1,), -7, dtype=torch.int64, device=dev)
    outd.fill_(-1)
    assert ctx.fallback_select(torch.from_numpy(conv).to(dev), torch.from_numpy(zncc).to(dev), 0.9, outd,
                               count=cnt) is None
    ctx.synchronize()
    assert int(cnt.item()) == k and np.array_equal(np.sort(outd[:k].cpu().numpy()), want)


def _patches_numpy(f, g, crd):
    M, N = f.shape
    out = np.zeros((crd.shape[0], 72, 72, 2))
    for t, (x, y) in enumerate(crd):
        x0, y0 = int(round(x)), int(round(y))
        r1, c1 = np.arange(x0 - 36, x0 + 36), np.arange(y0 - 36, y0 + 36)
        inr, inc = (r1 >= 1) & (r1 <= M), (c1 >= 1) & (c1 <= N)
        ri, ci = np.clip(r1, 1, M) - 1, np.clip(c1, 1, N) - 1
        keep = np.outer(inr, inc)
        out[t, :, :, 1] = np.where(keep, g[np.ix_(ri, ci)], 0.0)
        out[t, 16:56, 16:56, 0] = np.where(keep, f[np.ix_(ri, ci)], 0.0)[16:56, 16:56]
    return out


def test_network_patches_and_prediction(env):
    torch, ctx, pair = env["torch"], env["ctx"], env["pair"]
    from aldic_b200.learned import ProposalNet

    dev = torch.device("cuda:0")
    # centres = 1 (mod 4) far enough from the border that every crop is the whole-image one,
    # one off the 4-grid (moved to its aligned neighbour), one at the border (no guess)
    g = np.arange(41, 216, 8, dtype=np.float64)
    X_, Y_ = np.meshgrid(g, g, indexing="ij")
    crd = np.stack([X_.ravel(), Y_.ravel()], 1)[:150].copy()
    crd[-2] = [102.0, 130.0]
    crd[-1] = [9.0, 120.0]
    n = crd.shape[0]
    ct = torch.from_numpy(np.ascontiguousarray(crd.T)).to(dev)
    X = torch.empty((n, 72, 72, 2), dtype=torch.bfloat16, device=dev)
    ctx.net_extract(ct, X)
    ctx.synchronize()
    got = X.float().cpu().numpy()
    # the device's normalised images are FP32 copies of the oracle's FP64 ones: BF16 values
    # agree up to the rare tie
    want = CO.bf16(_patches_numpy(env["f"], env["g"], crd).astype(np.float32))
    assert (got == want).mean() > 0.999
    assert np.abs(got - want).max() <= 2.0 ** -7 * max(1.0, np.abs(want).max())
    net = ProposalNet(0, max_batch=64, seed=5)
    try:
        b = {"U0": torch.empty(2 * n, dtype=torch.float64, device=dev),
             "F0": torch.empty(4 * n, dtype=torch.float64, device=dev)}
        net.predict(ctx, ct, b)
        ctx.synchronize()
        # the per-window network on the same windows (the off-grid one at its aligned centre)
        crd_al = crd.copy()
        crd_al[-2] = [101.0, 129.0]
        ca = torch.from_numpy(np.ascontiguousarray(crd_al.T)).to(dev)
        ctx.net_extract(ca, X)
        ctx.synchronize()
        Y = torch.empty((n + 2, 6), dtype=torch.float32, device=dev)
        Xp = torch.cat([X, X[:2]])  # a multiple of 8 rows
        for s in range(0, n + 2, 64):
            e = min(s + 64, n + 2)
            net.forward(Xp[s:e].contiguous(), Y[s:e])
        torch.cuda.synchronize()
        y = Y[:n].cpu().numpy().astype(np.float64)
        U0 = b["U0"].cpu().numpy().reshape(n, 2)
        F0 = b["F0"].cpu().numpy().reshape(n, 4)
        m = n - 2
        assert np.array_equal(U0[:m], 8.0 * y[:m, :2])
        assert np.abs(F0[:m] - y[:m, 2:] / 20.0).max() <= 1e-7 * max(1.0, np.abs(y).max())
        # the off-grid centre: the aligned prediction moved along F0 by (1, 1) px
        f = F0[-2]
        want_u = 8.0 * y[-2, :2] + np.array([f[0] + f[2], f[1] + f[3]])
        assert np.abs(U0[-2] - want_u).max() < 1e-6
        assert np.all(np.isnan(U0[-1]))
    finally:
        net.close()


def test_training_lowers_the_held_out_error():
    """A short training run on tile mosaics (every tile its own speckles and affine warp,
    labelled by IC-GN): the held-out displacement error falls well below the untrained one."""
    import aldic_b200 as A
    from aldic_b200 import train_net
    from aldic_b200.learned import ProposalNet

    net, summary = train_net.train_network(frames=12, steps=1500, batch=256, lr=2e-3, eval_frames=1)
    fresh = ProposalNet(0, max_batch=4096, seed=0)
    ctx = A.Context(0)
    try:
        Xe, Te = train_net.build_dataset(ctx, 1, 900000)
        before = train_net.evaluate(fresh, Xe, Te)
        after = summary["held_out"]
        assert after["u_px_p50"] < 0.5 * before["u_px_p50"], (before, after)
        assert summary["loss"][-1][1] < 0.3 * summary["loss"][0][1]
    finally:
        ctx.close()
        fresh.close()
        net.close()


def test_trained_network_gains_over_the_search_guess():
    """The shipped trained network on a held-out smooth-field pair (512 x 512): IC-GN from its
    guess converges where IC-GN from the integer search's guess does, to the same solution,
    with few fallbacks; its gradient guess is closer to the converged gradient than the
    search's F = 0; an untrained network's guesses often fall back."""
    import os

    import aldic_b200 as A
    from aldic_b200 import learned as L
    from aldic_b200 import synth_gpu, train_net

    if not os.path.exists(train_net.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights shipped")
    ctx = A.Context(0)
    net = L.ProposalNet(0, max_batch=4096)
    try:
        pair = synth_gpu.field_pair(999, M=512, N=512)
        M, N = pair.M, pair.N
        gx, gy, w, st, s = [21, M - 20], [21, N - 20], 32, 16, 16
        ctx.load_image_raw(0, pair.ref, gx, gy, want_stats=False, shape=(M, N))
        ctx.load_image_raw(1, pair.deff, gx, gy, want_stats=False, shape=(M, N))
        ctx.compute_gradients()
        # the reference's start: the integer search, outliers removed, inpainted, F = 0
        r = ctx.integer_search([s, s], gx, gy, w, st)
        u, v, _ = O.remove_outliers(r["u"], r["v"], 100.0)
        U0 = O.init_u0(u, v)
        li = L.LearnedInit(net, ctx, s, gx, gy, w, st, 1e-3)
        crd = li.coords.cpu().numpy().T.copy()
        f = ctx.local_icgn(A.QUADTREE, crd, U0, w, 1e-3, want_H=False)
        ok_f = (f["conv"] > 0) & (f["conv"] < 100)

        net.set_params(L.init_params(0))  # untrained
        nf0 = li.run()
        li.stream.synchronize()
        net.set_params(np.load(train_net.DEFAULT_WEIGHTS))
        nf = li.run()
        li.stream.synchronize()
        b = {k: v.cpu().numpy() for k, v in li.buf.items()}
        ok_l = (b["conv"] > 0) & (b["conv"] < 100)
        assert nf0 > 0.2 * li.n and nf <= 0.02 * li.n, (nf0, nf, li.n)
        assert ok_l[ok_f].all()
        both = ok_l & ok_f
        assert np.abs(b["U"] - f["U"]).reshape(-1, 2)[both].max() < 1e-2
        keep = ~b["fallback"]
        Fc = b["F"].reshape(-1, 4)[keep & both]
        err_net = np.median(np.abs(b["F0"].reshape(-1, 4)[keep & both] - Fc))
        err_zero = np.median(np.abs(Fc))
        assert err_net < 0.75 * err_zero, (err_net, err_zero)
        du = np.hypot(*(b["U0"].reshape(-1, 2)[keep] - b["U"].reshape(-1, 2)[keep]).T)
        assert np.median(du) < 0.5
    finally:
        net.close()
        ctx.close()


def test_pipelined_frames_equal_one_at_a_time():
    """Frames pushed through LearnedPipeline (two contexts; the host's wait for a frame's
    fallback count sits behind the next frame's launches) get, frame by frame, the results
    of LearnedInit.run on that frame alone, fallbacks included (forced by a ZNCC threshold
    at the 10th percentile of the converged subsets)."""
    import os

    import torch

    import aldic_b200 as A
    from aldic_b200 import learned as L
    from aldic_b200 import synth_gpu, train_net

    if not os.path.exists(train_net.DEFAULT_WEIGHTS):
        pytest.skip("no trained weights shipped")
    ctxs = [A.Context(0) for _ in range(3)]
    net = L.ProposalNet(0, max_batch=4096)
    try:
        net.set_params(np.load(train_net.DEFAULT_WEIGHTS))
        M = N = 512
        gx, gy, w, st, s = [21, M - 20], [21, N - 20], 32, 16, 16
        pairs = [synth_gpu.field_pair(seed, M=M, N=N) for seed in (31, 32, 33)]

        def load(ctx, p):
            ctx.load_image_raw(0, p.ref, gx, gy, want_stats=False, shape=(M, N))
            ctx.load_image_raw(1, p.deff, gx, gy, want_stats=False, shape=(M, N))
            ctx.compute_gradients()

        one = L.LearnedInit(net, ctxs[2], s, gx, gy, w, st, 1e-3)

        def run_one(p):
            with torch.cuda.stream(one.stream):
                load(ctxs[2], p)
            nf = one.run()
            one.stream.synchronize()
            return nf, {k: v.cpu().numpy() for k, v in one.buf.items()}

        _, b0 = run_one(pairs[0])
        ok = (b0["conv"] > 0) & (b0["conv"] < 100)
        zmin = float(np.quantile(b0["zncc"][ok], 0.1))
        one.zncc_min = zmin
        want = [run_one(p) for p in pairs]
        assert all(nf > 0 for nf, _ in want)
        pipe = L.LearnedPipeline(net, ctxs[:2], s, gx, gy, w, st, 1e-3, zncc_min=zmin)
        got = []

        def keep(done):
            if done is not None:
                pipe.stream.synchronize()
                got.append((done.n_fallback, {k: v.cpu().numpy() for k, v in done.buf.items()}))

        for p in pairs:
            keep(pipe.push(lambda ctx, p=p: load(ctx, p)))
        keep(pipe.flush())
        assert len(got) == len(pairs)
        for (nf_w, bw), (nf_g, bg) in zip(want, got):
            assert nf_w == nf_g
            for k in ("U0", "F0", "U", "F", "conv", "fallback"):
                assert np.array_equal(bw[k], bg[k], equal_nan=True), k
    finally:
        net.close()
        for c in ctxs:
            c.close()
