"""Seeded synthetic count matrices with the shapes and distributions of the
benchmark workloads (no public dataset is available offline).

Per-gene mean expression is lognormal(-2.5, 1.8); each cell belongs to one
of C clusters (uniform); each cluster multiplies 200 random genes by
lognormal(0, 0.5) fold changes; library sizes are lognormal(7.6, 0.45)
times one global scale chosen so the expected number of non-zeros per cell
hits the workload's target; counts are negative-binomial with dispersion phi
(variance mu + phi mu^2).  Genes 0..9 are named ``MT-*`` so the mito QC path
is exercised.  The count draws are made on the GPU by ``crest_synth_gpu``
(one counter-based uniform per cell and gene, defined once in
``csrc/synth_core.h``; the test oracle draws the identical matrix on host
threads from the same definition).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass(frozen=True)
class Workload:
    name: str
    n_cells: int
    n_genes: int
    n_clusters: int
    dispersion: float
    nnz_per_cell: float
    seed: int
    chunk_cells: int = 16384


WORKLOADS = {
    # plain method, small (CPU-runnable reference case)
    "pbmc3k_like": Workload("pbmc3k_like", 2_700, 32_738, 8, 0.2, 820.0, 11),
    # plain GPU drop-in at scale
    "100k": Workload("100k", 100_000, 33_538, 20, 0.15, 2_100.0, 12, 8192),
    # precision form
    "200k": Workload("200k", 200_000, 33_538, 30, 0.15, 2_100.0, 13),
    # out-of-core large (the headline workload)
    "1m": Workload("1m", 1_000_000, 36_601, 50, 0.2, 1_500.0, 15),
}


@dataclass
class Params:
    prob: np.ndarray    # (n_clusters, n_genes) relative expression, rows sum to 1
    labels: np.ndarray  # (n_cells,) int32
    lib: np.ndarray     # (n_cells,) expected total count
    dispersion: float
    seed: int


def make_params(n_cells: int, n_genes: int, n_clusters: int, dispersion: float, nnz_per_cell: float,
                seed: int, n_de: int = 200) -> Params:
    rng = np.random.default_rng(seed)
    base = rng.lognormal(-2.5, 1.8, n_genes)
    labels = rng.integers(0, n_clusters, n_cells).astype(np.int32)
    fold = np.ones((n_clusters, n_genes))
    for c in range(n_clusters):
        idx = rng.choice(n_genes, min(n_de, n_genes), replace=False)
        fold[c, idx] = rng.lognormal(0.0, 0.5, len(idx))
    prob = base[None, :] * fold
    prob /= prob.sum(axis=1, keepdims=True)
    lib0 = rng.lognormal(7.6, 0.45, n_cells)
    # global library scale: expected non-zeros per cell on a sample of cells
    m = min(n_cells, 96)
    P = prob[labels[:m]]
    L = lib0[:m, None]
    r = 1.0 / dispersion

    def expected_nnz(log_s):
        mu = np.exp(log_s) * L * P
        return float(np.mean(np.sum(-np.expm1(-r * np.log1p(dispersion * mu)), axis=1)))

    target = min(nnz_per_cell, 0.95 * n_genes)
    lo, hi = -30.0, 30.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if expected_nnz(mid) < target:
            lo = mid
        else:
            hi = mid
    lib = lib0 * np.exp(0.5 * (lo + hi))
    return Params(np.ascontiguousarray(prob), np.ascontiguousarray(labels), np.ascontiguousarray(lib),
                  float(dispersion), int(seed))


def _struct(p: Params) -> _lib.Synth:
    return _lib.Synth(len(p.labels), p.prob.shape[1], p.prob.shape[0], p.dispersion, p.seed,
                      _lib.ptr(p.prob), _lib.ptr(p.labels), _lib.ptr(p.lib))


def generate(p: Params, pinned_alloc=None):
    """Draw the counts on the GPU; returns (indptr i64, indices u32, data f32) in
    host memory with gene-sorted rows.  ``pinned_alloc`` (n, dtype) -> array may
    supply page-locked output buffers."""
    n = len(p.labels)
    s = _struct(p)
    rn = np.zeros(n, np.int64)
    _lib.call("crest_synth_gpu", C.byref(s), _lib.ptr(rn), None, None, None)
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(rn, out=indptr[1:])
    nnz = int(indptr[-1])
    if pinned_alloc is not None:
        indices = pinned_alloc(nnz, np.uint32)
        data = pinned_alloc(nnz, np.float32)
    else:
        indices = np.empty(nnz, np.uint32)
        data = np.empty(nnz, np.float32)
    _lib.call("crest_synth_gpu", C.byref(s), None, _lib.ptr(indptr), _lib.ptr(indices), _lib.ptr(data))
    return indptr, indices, data


def gene_names(n_genes: int, n_mito: int = 10):
    return [f"MT-{i}" if i < n_mito else f"G{i}" for i in range(n_genes)]


def workload_params(w: Workload, n_cells: int = None) -> Params:
    """Parameters of a named workload; with n_cells, those of its first n_cells cells
    (the same cells, labels and library sizes as in the full workload)."""
    p = make_params(w.n_cells, w.n_genes, w.n_clusters, w.dispersion, w.nnz_per_cell, w.seed)
    if n_cells is not None and n_cells < w.n_cells:
        p = Params(p.prob, p.labels[:n_cells].copy(), p.lib[:n_cells].copy(), p.dispersion, p.seed)
    return p


def make_workload(w: Workload, n_cells: int = None, **kw):
    """CSR arrays of a named workload (optionally only its first n_cells cells), drawn on the GPU."""
    return generate(workload_params(w, n_cells), **kw)
