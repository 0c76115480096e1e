"""Multi-rank sharding on CPU (gloo, world size 2): every rank solves its range of subsets
and the tensor all-gather reassembles exactly the single-process result.  The per-rank
solver is the FP64 oracle here (the device path is the same call on each rank's GPU, its
results gathered as CUDA tensors over NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from aldic_b200 import shard


def test_partition_balances_cost():
    parts = shard.partition(10, 3)
    assert parts[0][0] == 0 and parts[-1][1] == 10
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    cost = np.r_[np.full(50, 4.0), np.ones(50)]
    p = shard.partition(100, 2, cost)
    tot = [cost[s:e].sum() for s, e in p]
    assert abs(tot[0] - tot[1]) <= 4.0
    assert shard.partition(0, 4) == [(0, 0)] * 4
    assert shard.partition(3, 5)[-1][1] == 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "3d-stereo-aldic_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch.distributed as dist

    import oracle as O
    from aldic_b200 import shard as S
    from aldic_b200 import synth

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sc = synth.temporal_affine(M=160, N=150, n_speckles=300)
    M, N = sc.ref.shape
    f, _ = O.normalize(sc.ref.astype(float), [1, M], [1, N])
    g, _ = O.normalize(sc.deff.astype(float), [1, M], [1, N])
    gx, gy = O.gradient(f)
    fr = O.Frame(f, g, np.ones_like(f), gx, gy)
    xs = np.arange(20, 140, 9.0)
    X, Y = np.meshgrid(xs, np.arange(20, 130, 9.0), indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel()], 1)
    tu, tv = sc.disp(coords[:, 0], coords[:, 1])
    U0 = np.stack([np.round(tu), np.round(tv)], 1).ravel()

    def solve(c, u0):
        r = O.local_icgn(fr, c, u0, 20, 1e-3, variant=1, nthreads=1)
        return {k: r[k] for k in ("U", "F", "H", "conv")}

    fields = ("U", "F", "conv", "H")
    # cost: window area x the iterations of a previous solve (uneven ranges)
    prev = solve(coords, U0)["conv"]
    got = S.sharded_local_icgn(solve, coords, U0, cost=S.icgn_cost(20, prev), fields=fields)
    full = solve(coords, U0)
    ok = all(np.array_equal(got[k].numpy(), np.asarray(full[k]), equal_nan=True) for k in fields)
    # a bare row gather with an uneven partition
    import torch

    parts = [(0, 3), (3, 10)]
    s, e = parts[rank]
    rows = S.gather_rows(torch.arange(s, e, dtype=torch.float64).reshape(-1, 1).repeat(1, 2), parts)
    ok = ok and torch.equal(rows[:, 0], torch.arange(10, dtype=torch.float64))
    q.put((rank, ok, int(len(coords))))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_icgn_matches_single_process_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(r[0] for r in res) == [0, 1]
    assert all(r[1] for r in res)
    assert res[0][2] > 100


def test_no_group_is_local():
    calls = []

    def solve(c, u0):
        calls.append(len(c))
        n = len(c)
        return {"U": np.zeros(2 * n), "F": np.zeros(4 * n), "H": np.zeros((n, 21)), "conv": np.ones(n, np.int32)}

    out = shard.sharded_local_icgn(solve, np.zeros((7, 2)), np.zeros(14))
    assert calls == [7] and out["conv"].shape == (7,)


@pytest.mark.parametrize("n,world", [(1, 2), (5, 2), (1000, 8)])
def test_partition_covers_everything(n, world):
    parts = shard.partition(n, world, np.random.default_rng(0).uniform(0.5, 2.0, n))
    seen = np.concatenate([np.arange(s, e) for s, e in parts])
    assert np.array_equal(seen, np.arange(n))
