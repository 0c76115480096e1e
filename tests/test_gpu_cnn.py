"""GPU tests of the learned initial guess's network: the tcgen05 GEMM against numpy, the
network's forward pass and gradients against the CPU restatement with the device's BF16
rounding points (oracle/cnn_oracle.py, itself pinned by finite differences on the CPU), and
Adam steps that lower the loss."""
import numpy as np
import pytest

import cnn_oracle as CO

pytestmark = pytest.mark.gpu


def _bf16_tensor(a, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev).to(torch.bfloat16)


# the last three hold several tiles per persistent CTA (148 SMs): both TMEM accumulators and
# the stage ring wrap around many times, with split-K atomics in the last
@pytest.mark.parametrize("M,N,K,splits", [(300, 32, 24, 1), (256, 64, 288, 1), (128, 16, 128, 1),
                                          (1000, 1024, 128, 1), (64, 288, 4096, 8), (32, 24, 131072, 64),
                                          (113664, 64, 736, 1), (56832, 1024, 256, 1), (20000, 128, 4096, 4)])
def test_tensor_core_gemm_matches_numpy(M, N, K, splits):
    import torch

    from aldic_b200.learned import gemm_bf16

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(M + N + K)
    a = CO.bf16(rng.normal(size=(M, K)).astype(np.float32))
    b = CO.bf16(rng.normal(size=(N, K)).astype(np.float32))
    C = torch.zeros((M, N), dtype=torch.float32, device=dev)
    gemm_bf16(_bf16_tensor(a, dev), _bf16_tensor(b, dev), C, splits=splits)
    torch.cuda.synchronize()
    want = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    err = np.abs(C.cpu().numpy() - want) / np.maximum(scale, 1e-30)
    assert err.max() < 1e-5, err.max()


def _batch(seed, B):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, 72, 72, 2)).astype(np.float32)
    X[:, :, :, 0] = 0.0
    X[:, 16:56, 16:56, 0] = rng.normal(size=(B, 40, 40))
    T = rng.normal(scale=0.5, size=(B, 6)).astype(np.float32)
    return CO.bf16(X), T


def test_network_forward_and_gradients_match_the_cpu_restatement():
    import torch

    from aldic_b200.learned import ProposalNet

    dev = torch.device("cuda:0")
    B = 32
    p = CO.init_params(1)
    X, T = _batch(2, B)
    net = ProposalNet(0, max_batch=64)
    try:
        net.set_params(p)
        assert np.array_equal(net.get_params(), p)
        x, t = _bf16_tensor(X, dev), torch.from_numpy(T).to(dev)
        y = torch.empty((B, 6), dtype=torch.float32, device=dev)
        net.forward(x, y)
        torch.cuda.synchronize()
        yr, _ = CO.forward(p, X)
        assert np.abs(y.cpu().numpy() - yr).max() <= 2e-2 * max(1.0, np.abs(yr).max())
        loss, g = net.gradients(x, t)
        lr_, gr = CO.loss_and_gradients(p, X, T)
        assert abs(loss - lr_) <= 1e-2 * lr_
        off, n = CO.layout()
        for l, (ow, ob) in enumerate(off):
            for a, b in ((ow, ob), (ob, ob + CO.ROWS[l])):
                d, r = g[a:b].astype(np.float64), gr[a:b]
                rel = np.linalg.norm(d - r) / max(np.linalg.norm(r), 1e-30)
                cos = d @ r / max(np.linalg.norm(d) * np.linalg.norm(r), 1e-30)
                assert rel < 5e-2 and cos > 0.998, (l, rel, cos)
        net.status()
    finally:
        net.close()


def test_adam_steps_lower_the_loss():
    import torch

    from aldic_b200.learned import ProposalNet

    dev = torch.device("cuda:0")
    X, T = _batch(7, 64)
    net = ProposalNet(0, max_batch=64)
    try:
        net.set_params(CO.init_params(4))
        x, t = _bf16_tensor(X, dev), torch.from_numpy(T).to(dev)
        losses = [net.train_step(x, t, 1e-3, want_loss=True) for _ in range(40)]
        assert losses[-1] < 0.5 * losses[0], losses[::8]
        net.status()
    finally:
        net.close()
