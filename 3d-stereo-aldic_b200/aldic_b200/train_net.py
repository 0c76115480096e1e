"""Train the proposal network of the learned initial guess on the GPU and write its weights.

Training data: tile mosaics (synth_gpu.tile_pair) -- every 64 x 64 tile its own speckle
pattern under its own random affine warp (|u|, |v| <= 12 px, every gradient <= 0.05), so that
each sample's texture and deformation are independent -- labelled with the method's own
converged IC-GN results from the analytic initial guess (learned.label_pair).  Optimiser: the
library's Adam kernel on minibatches, cosine learning-rate decay.  Every forward, backward and
update step runs in the library's kernels (csrc/cnn.cu, csrc/cnn_gemm.cu).

  python -m aldic_b200.train_net [--frames 2000] [--steps 60000] [--out proposal_net.npy]

writes the FP32 parameter vector (aldic_net_set_params layout) and, beside it, a JSON summary
(data and training time, loss log, errors on held-out tile frames).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import learned
from . import synth_gpu

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "proposal_net.npy")


def build_dataset(ctx, frames, seed0, tiles=32, w=32):
    """(X, T) CUDA tensors of `frames` tile mosaics of tiles x tiles samples each."""
    import torch

    Xs, Ts = [], []
    for s in range(frames):
        X, T = learned.label_pair(ctx, synth_gpu.tile_pair(seed0 + s, tiles=tiles), w=w)
        Xs.append(X)
        Ts.append(T)
    torch.cuda.synchronize()
    return torch.cat(Xs), torch.cat(Ts)


def evaluate(net, X, T):
    """Errors of the network's outputs on (X, T): u, v in px (Euclidean) and the gradient
    entries, as percentiles."""
    import torch

    n = X.shape[0] // 8 * 8
    Y = torch.empty((n, 6), dtype=torch.float32, device=X.device)
    for s in range(0, n, net.max_batch):
        e = min(s + net.max_batch, n)
        net.forward(X[s:e].contiguous(), Y[s:e])
    torch.cuda.synchronize()
    scale = torch.tensor(learned.SCALE, device=X.device)
    err = ((Y - T[:n]) / scale).abs().cpu().numpy()
    eu = np.hypot(err[:, 0], err[:, 1])
    return {"samples": int(n), "u_px_p50": float(np.median(eu)), "u_px_p90": float(np.percentile(eu, 90)),
            "u_px_p99": float(np.percentile(eu, 99)), "F_p50": float(np.median(err[:, 2:])),
            "F_p90": float(np.percentile(err[:, 2:], 90))}


def train_network(device=0, frames=2000, steps=60000, batch=256, lr=1e-3, seed=0, eval_frames=4, log=None):
    """Build the data set, train a fresh network, evaluate it on held-out tile frames.
    Returns (network, summary dict)."""
    import torch

    import aldic_b200 as A

    ctx = A.Context(device)
    try:
        t0 = time.perf_counter()
        X, T = build_dataset(ctx, frames, 1000 + 7919 * seed)
        t_data = time.perf_counter() - t0
        Xe, Te = build_dataset(ctx, eval_frames, 900000 + seed)
    finally:
        ctx.close()
    net = learned.ProposalNet(device, max_batch=max(4096, batch), seed=seed)
    t0 = time.perf_counter()
    losses = learned.train(net, X, T, steps, batch=batch, lr=lr, lr_end=lr / 100, seed=seed,
                           log_every=max(1, steps // 20))
    t_train = time.perf_counter() - t0
    summary = {"frames": frames, "samples": int(X.shape[0]), "steps": steps, "batch": batch, "lr": lr,
               "seed": seed, "data_s": t_data, "train_s": t_train, "loss": [[k, l] for k, l in losses],
               "held_out": evaluate(net, Xe, Te), "device": torch.cuda.get_device_name(device)}
    if log:
        log(summary)
    del X, T
    return net, summary


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--frames", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=60000)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    args = ap.parse_args()
    net, summary = train_network(frames=args.frames, steps=args.steps, batch=args.batch, lr=args.lr,
                                 seed=args.seed)
    np.save(args.out, net.get_params())
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "loss"}), flush=True)
    net.close()


if __name__ == "__main__":
    main()
