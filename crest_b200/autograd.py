"""Differentiable normalise -> log1p -> scale -> project map (the fused CUDA
kernels ``crest_fused_forward`` / ``crest_fused_backward`` behind a
``torch.autograd.Function``).

For a CSR matrix over the d selected genes, per-cell size factors ``sf``
(the normalisation DIVIDES: ``y = x / sf``), loadings ``W`` (d x k) and the
fixed scale parameters ``mean`` / ``std`` / ``max_value`` of ``crest.pp.scale``:

    scores[c, :] = sum over the cell's entries of s W[g, :],
    s = clip((log1p(x / sf[c]) - mean[g]) / std[g]) - clip(-mean[g] / std[g])

Gradients flow to the stored values, the size factors and W.  The backward
recomputes log1p and the scaled values instead of keeping the dense scaled
matrix.  PyTorch is used here only as the autograd hook and for device
buffers; all arithmetic runs in the library's kernels.
"""

from __future__ import annotations

import torch

from . import _lib


def _dev_ptr(t: torch.Tensor, dtype, name: str):
    if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA tensor of {dtype}")
    return t.data_ptr()


class FusedScaleProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, size_factors, W, indptr, indices, mean, std, max_value):
        n = indptr.numel() - 1
        d, k = W.shape
        scores = torch.empty((n, k), dtype=torch.float32, device=values.device)
        args = (_dev_ptr(indptr, torch.int64, "indptr"), _dev_ptr(indices, torch.int32, "indices"),
                _dev_ptr(values, torch.float32, "values"), n, d,
                _dev_ptr(size_factors, torch.float32, "size_factors"), _dev_ptr(W, torch.float32, "W"), k,
                _dev_ptr(mean, torch.float64, "mean"), _dev_ptr(std, torch.float64, "std"), float(max_value))
        torch.cuda.current_stream().synchronize()
        _lib.call("crest_fused_forward", *args, scores.data_ptr())
        ctx.save_for_backward(values, size_factors, W, indptr, indices, mean, std)
        ctx.max_value = float(max_value)
        return scores

    @staticmethod
    def backward(ctx, grad_scores):
        values, size_factors, W, indptr, indices, mean, std = ctx.saved_tensors
        n = indptr.numel() - 1
        d, k = W.shape
        g = grad_scores.contiguous().to(torch.float32)
        grad_values = torch.empty_like(values)
        grad_sf = torch.empty_like(size_factors)
        grad_W = torch.empty_like(W)
        torch.cuda.current_stream().synchronize()
        _lib.call("crest_fused_backward", indptr.data_ptr(), indices.data_ptr(), values.data_ptr(), n, d,
                  size_factors.data_ptr(), W.data_ptr(), k, mean.data_ptr(), std.data_ptr(), ctx.max_value,
                  g.data_ptr(), grad_values.data_ptr(), grad_sf.data_ptr(), grad_W.data_ptr())
        return grad_values, grad_sf, grad_W, None, None, None, None, None


def fused_scale_project(values, size_factors, W, indptr, indices, mean, std, max_value=10.0):
    """scores (n x k, f32) of the map above; differentiable in values, size_factors and W."""
    return FusedScaleProject.apply(values, size_factors, W, indptr, indices, mean, std, max_value)
