"""Shared inputs and the FP64 PyTorch reference of the fused normalise ->
log1p -> scale -> project map (size factor divides), used by the GPU parity
test and by the finite-difference check of the reference itself."""

import numpy as np
import torch

from crest_b200 import synth


def make_case(n=3000, d=400, k=24, max_value=10.0, seed=0, nnz_per_cell=60.0, clusters=5, dispersion=0.5):
    p = synth.make_params(n, d, clusters, dispersion, nnz_per_cell, seed=seed)
    from oracle import synth as osynth
    indptr, indices, data = osynth.generate(p)
    rng = np.random.default_rng(seed + 1)
    sf = np.exp(rng.normal(0.0, 0.3, n)).astype(np.float32)
    W = np.linalg.qr(rng.standard_normal((d, k)))[0].astype(np.float32)
    cell = np.repeat(np.arange(n), np.diff(indptr))
    l = np.log1p(data.astype(np.float64) / sf[cell])
    s1 = np.bincount(indices, l, d)
    s2 = np.bincount(indices, l * l, d)
    mean = s1 / n
    std = np.sqrt(np.maximum((s2 - n * mean * mean) / (n - 1), 0.0))
    std[std == 0] = 1.0
    wts = rng.standard_normal((n, k))
    return dict(indptr=indptr.astype(np.int64), indices=indices.astype(np.int32), values=data.astype(np.float32),
                sf=sf, W=W, mean=mean, std=std, max_value=max_value, wts=wts, n=n, d=d, k=k)


def reference(c, values, sf, W):
    """FP64 torch restatement of the map (float64 tensors, autograd-able), on
    the device of `values`."""
    n = c["n"]
    dev = values.device
    cell = torch.as_tensor(np.repeat(np.arange(n), np.diff(c["indptr"])), device=dev)
    g = torch.as_tensor(c["indices"].astype(np.int64), device=dev)
    mean = torch.as_tensor(c["mean"], device=dev)
    std = torch.as_tensor(c["std"], device=dev)
    mv = c["max_value"]
    y = values / sf[cell]
    z = (torch.log1p(y) - mean[g]) / std[g]
    b = -mean[g] / std[g]
    if mv > 0:
        z = torch.clamp(z, -mv, mv)
        b = torch.clamp(b, -mv, mv)
    s = z - b
    scores = torch.zeros((n, W.shape[1]), dtype=torch.float64, device=dev)
    scores.index_add_(0, cell, s[:, None] * W[g])
    return scores


def loss_of(scores, wts):
    return (wts * scores * scores).sum()


def ref_run(c, device="cpu"):
    values = torch.tensor(c["values"].astype(np.float64), requires_grad=True, device=device)
    sf = torch.tensor(c["sf"].astype(np.float64), requires_grad=True, device=device)
    W = torch.tensor(c["W"].astype(np.float64), requires_grad=True, device=device)
    scores = reference(c, values, sf, W)
    loss_of(scores, torch.tensor(c["wts"], device=device)).backward()
    return scores.detach().cpu(), values.grad.cpu(), sf.grad.cpu(), W.grad.cpu()


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


