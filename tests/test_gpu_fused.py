"""Differentiable normalise -> log1p -> scale -> project map (K7).

The CUDA forward and backward (crest_fused_forward / crest_fused_backward
behind crest_b200.autograd) are checked against an FP64 PyTorch reference of
the same map and its autograd gradient (tests/fused_case.py); that reference
gradient is itself checked against central finite differences in
tests/test_fused_reference.py.
Tolerances: scores 1e-5 and gradients 1e-4, relative in the 2-norm (the
CUDA path keeps y and log1p(y) in f32, as the reference's transform does).
"""

import numpy as np
import pytest
import torch

from crest_b200 import _lib
from crest_b200.autograd import fused_scale_project
from fused_case import loss_of, make_case, ref_run, rel

pytestmark = pytest.mark.gpu


def gpu_run(c):
    dev = torch.device("cuda")
    values = torch.tensor(c["values"], device=dev, requires_grad=True)
    sf = torch.tensor(c["sf"], device=dev, requires_grad=True)
    W = torch.tensor(c["W"], device=dev, requires_grad=True)
    scores = fused_scale_project(values, sf, W, torch.tensor(c["indptr"], device=dev),
                                 torch.tensor(c["indices"], device=dev), torch.tensor(c["mean"], device=dev),
                                 torch.tensor(c["std"], device=dev), c["max_value"])
    loss_of(scores.double(), torch.tensor(c["wts"], device=dev)).backward()
    return (scores.detach().cpu().double(), values.grad.cpu().double(), sf.grad.cpu().double(),
            W.grad.cpu().double())


@pytest.mark.parametrize("k,max_value", [(24, 10.0), (50, 10.0), (100, 10.0), (24, 0.75), (50, 0.0)])
def test_forward_and_gradients_match_fp64_reference(k, max_value):
    c = make_case(k=k, max_value=max_value)
    s_gpu, gx, gsf, gW = gpu_run(c)
    s_ref, rx, rsf, rW = ref_run(c)
    assert rel(s_gpu, s_ref) <= 1e-5
    assert rel(gx, rx) <= 1e-4
    assert rel(gsf, rsf) <= 1e-4
    assert rel(gW, rW) <= 1e-4


def test_differentiation_workload_shape():
    """The differentiation workload at its own shape: 50,000 cells x 2,000 HVG
    genes (~200 stored entries per cell), k = 50, scale max 10; the FP64
    reference runs with float64 PyTorch ops on the GPU."""
    c = make_case(n=50_000, d=2_000, k=50, max_value=10.0, seed=4, nnz_per_cell=200.0, clusters=20,
                  dispersion=0.2)
    s_gpu, gx, gsf, gW = gpu_run(c)
    s_ref, rx, rsf, rW = ref_run(c, device="cuda")
    assert rel(s_gpu, s_ref) <= 1e-5
    assert rel(gx, rx) <= 1e-4
    assert rel(gsf, rsf) <= 1e-4
    assert rel(gW, rW) <= 1e-4


def test_out_of_range_gene_id_is_rejected():
    c = make_case(n=50, d=40, k=8)
    c["indices"][3] = c["d"] + 5
    dev = torch.device("cuda")
    with pytest.raises(ValueError, match=r"gene ids in \[0, d\)"):
        fused_scale_project(torch.tensor(c["values"], device=dev), torch.tensor(c["sf"], device=dev),
                            torch.tensor(c["W"], device=dev), torch.tensor(c["indptr"], device=dev),
                            torch.tensor(c["indices"], device=dev), torch.tensor(c["mean"], device=dev),
                            torch.tensor(c["std"], device=dev), 10.0)
    assert _lib.EINVAL == -22


def test_wide_gene_set_counts_entries_with_global_atomics():
    """d above the shared-memory histogram of the backward (12,288 genes): the
    per-gene entry counts come from global atomics; the same gradients."""
    c = make_case(n=2000, d=13_000, k=24, max_value=10.0, seed=7, nnz_per_cell=300.0)
    s_gpu, gx, gsf, gW = gpu_run(c)
    s_ref, rx, rsf, rW = ref_run(c)
    assert rel(s_gpu, s_ref) <= 1e-5
    assert rel(gx, rx) <= 1e-4
    assert rel(gsf, rsf) <= 1e-4
    assert rel(gW, rW) <= 1e-4
