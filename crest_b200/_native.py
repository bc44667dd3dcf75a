"""Drop-in for the reference's native module ``crest.crest`` on the
preprocessing-to-PCA path (src/py.rs:195-309, 386-399).

Same function names, positional arguments, accumulate-into-output semantics
and errors (``ValueError`` for bad arguments, ``RuntimeError`` when the
eigensolve fails), computed by the sm_100a kernels of ``libcrest_gpu.so``.
Each chunk function takes the 9-tuple of ``BioFrame.iter_ctx`` followed by its
own arguments.  ``gram_accumulate`` takes an extra keyword ``precision``
("fp64" by default, which reproduces the reference's FP64 sums; "fp32" and
"bf16x3" are the plain and product forms).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import carray, ptr

__all__ = ["qc", "gene_stats", "gram_accumulate", "pca_from_gram", "project", "group_gene_sums",
           "group_gene_totals", "t_pvalues", "knn_graph"]


def _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell):
    """src/py.rs:162-193: builds the chunk, returns (struct, keepalive, n_rows, n_vars)."""
    g = carray(genes, np.uint32, "genes")
    v = carray(values, np.float32, "values")
    if len(g) != len(v):
        raise ValueError("genes, values must have equal length")
    cm = carray(cell_map, np.int64, "cell_map")
    gm = carray(gene_map, np.int32, "gene_map")
    if cells is not None and indptr is None:
        c = carray(cells, np.uint32, "cells")
        if len(c) != len(g):
            raise ValueError("cells, genes must have equal length")
        if len(c) > 1 and bool(np.any(c[1:] < c[:-1])):
            raise ValueError("chunk must be sorted by cell")
        p = None
    elif cells is None and indptr is not None:
        p = carray(indptr, np.int64, "indptr")
        if len(p) == 0 or bool(np.any(p[1:] < p[:-1])) or int(p[-1] - p[0]) != len(g):
            raise ValueError("indptr must be non-decreasing and span the chunk")
        c = None
    else:
        raise ValueError("pass exactly one of cells / indptr")
    ch = _lib.Chunk(ptr(g), ptr(v), len(g), ptr(cm), len(cm), ptr(gm), len(gm), float(target_sum),
                    int(bool(log1p)), ptr(c), ptr(p), 0 if p is None else len(p), int(first_cell))
    n_rows = int(max(int(cm.max()) + 1, 0)) if len(cm) else 0
    n_vars = int(max(int(gm.max()) + 1, 0)) if len(gm) else 0
    return ch, (g, v, cm, gm, c, p), n_rows, n_vars


def _mut(a, dtype, name):
    a = carray(a, dtype, name)
    if not a.flags.writeable:
        raise ValueError(f"{name} must be writeable")
    return a


def gene_stats(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell, out):
    """Accumulate per-gene [sum x, sum x^2, sum expm1 x, sum expm1(x)^2, nnz] into out (n_vars, 5)."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    o = _mut(out, np.float64, "out")
    if o.size != nv * 5:
        raise ValueError("out must be (n_vars, 5)")
    _lib.call("crest_gene_stats", C.byref(ch), nv, ptr(o))


def qc(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
       flag, cell_total, cell_ngenes, cell_flag, gene_ncells, gene_total):
    """QC accumulation on raw counts (pass target_sum=0, log1p=False)."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    f = carray(flag, np.bool_, "flag")
    ct, cn, cf = (_mut(cell_total, np.float64, "cell_total"), _mut(cell_ngenes, np.uint32, "cell_ngenes"),
                  _mut(cell_flag, np.float64, "cell_flag"))
    gn, gt = _mut(gene_ncells, np.uint32, "gene_ncells"), _mut(gene_total, np.float64, "gene_total")
    if len(ct) < nr or len(cn) < nr or len(cf) < nr or len(gn) != nv or len(gt) != nv or len(f) != nv:
        raise ValueError("output sizes do not match the maps")
    _lib.call("crest_qc", C.byref(ch), ptr(f), nv, ptr(ct), ptr(cn), ptr(cf), nr, ptr(gn), ptr(gt))


def _scale(scale, mean, std, max_value, d):
    """src/py.rs:250-261."""
    if mean is not None and std is not None:
        mu, sd = carray(mean, np.float64, "mean"), carray(std, np.float64, "std")
    elif scale:
        raise ValueError("scale=True needs mean and std")
    else:
        mu = sd = None
    if scale and (len(mu) != d or len(sd) != d):
        raise ValueError("mean/std must have length d")
    return _lib.Scale(int(bool(scale)), ptr(mu) if scale else None, ptr(sd) if scale else None,
                      float(max_value)), (mu, sd)


def _check_sub(sub, nv, d):
    """src/py.rs:263-268."""
    if len(sub) != nv or (len(sub) and int(sub.max()) >= d):
        raise ValueError("sub_map must have length n_vars and values < d")


def gram_accumulate(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                    sub_map, gram, colsum, scale, mean, std, max_value, precision: str = "fp64"):
    """Accumulate the Gram matrix (upper triangle) and column sums of the (optionally scaled) submatrix."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    sm = carray(sub_map, np.int32, "sub_map")
    cs = _mut(colsum, np.float64, "colsum")
    d = len(cs)
    gr = _mut(gram, np.float64, "gram")
    if gr.size != d * d:
        raise ValueError("gram must be (d, d)")
    _check_sub(sm, nv, d)
    t, tk = _scale(scale, mean, std, max_value, d)
    if precision not in _lib.GRAM_PRECISION:
        raise ValueError(f"precision must be one of {sorted(_lib.GRAM_PRECISION)}")
    _lib.call("crest_gram_accumulate", C.byref(ch), ptr(sm), nv, C.byref(t), d, ptr(gr), ptr(cs),
              _lib.GRAM_PRECISION[precision])


def project(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
            sub_map, loadings, out, scale, mean, std, max_value):
    """out[row] += (scaled) row . loadings for one chunk (out: (n_rows, k) float32)."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    ld = np.asarray(loadings)
    if ld.ndim != 2:
        raise ValueError("loadings must be (d, k)")
    d, k = ld.shape
    sm = carray(sub_map, np.int32, "sub_map")
    ld = carray(ld, np.float64, "loadings")
    _check_sub(sm, nv, d)
    o = _mut(out, np.float32, "out")
    if o.size < nr * k:
        raise ValueError("out must be (n_rows, k)")
    t, tk = _scale(scale, mean, std, max_value, d)
    _lib.call("crest_project", C.byref(ch), ptr(sm), nv, ptr(ld), d, k, C.byref(t), ptr(o), nr)


def pca_from_gram(gram, colsum, n, k):
    """Top-k eigenpairs of the covariance implied by (gram, colsum, n).

    Returns (variance (k,), loadings (d, k), total_variance)."""
    g = carray(gram, np.float64, "gram")
    c = carray(colsum, np.float64, "colsum")
    d = len(c)
    if g.size != d * d:
        raise ValueError("gram must be (d, d)")
    n, k = int(n), int(k)
    if n < 2 or d == 0:
        raise RuntimeError("need at least 2 cells and 1 gene")
    k = min(k, d)
    vals = np.zeros(k, np.float64)
    vecs = np.zeros((d, k), np.float64)
    total = np.zeros(1, np.float64)
    st = _lib.PcaStats()
    rc = _lib.load().crest_pca_from_gram(ptr(g), ptr(c), d, n, k, ptr(vals), ptr(vecs), ptr(total), C.byref(st))
    if rc == _lib.ERUNTIME:
        raise RuntimeError(_lib.load().crest_last_error().decode(errors="replace"))
    _lib.check(rc)
    return vals, vecs, float(total[0])


def group_gene_sums(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                    group_of_row, sum, sumsq, nnz, clip=None):
    """Accumulate per (group, var) sums, sums of squares and nnz (each (n_groups, n_vars)) of the
    transformed values; ``clip`` (n_groups, n_vars) caps each value first (src/py.rs:311-338)."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    gr = carray(group_of_row, np.uint32, "group_of_row")
    s, q, z = _mut(sum, np.float64, "sum"), _mut(sumsq, np.float64, "sumsq"), _mut(nnz, np.float64, "nnz")
    if s.ndim != 2 or s.shape[1] != nv or q.shape != s.shape or z.shape != s.shape or len(gr) < nr:
        raise ValueError("sum, sumsq, nnz must be (n_groups, n_vars); group_of_row (n_rows,)")
    if bool(np.any((gr != np.iinfo(np.uint32).max) & (gr >= s.shape[0]))):
        raise ValueError("group id out of range")
    c = None
    if clip is not None:
        c = carray(clip, np.float64, "clip")
        if c.size != s.size:
            raise ValueError("clip must be (n_groups, n_vars)")
    _lib.call("crest_group_gene_sums", C.byref(ch), ptr(gr), len(gr), s.shape[0], nv, ptr(c), ptr(s), ptr(q),
              ptr(z))


def group_gene_totals(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                      group_of_row, sum):
    """Accumulate per (group, var) sums only, (n_groups, n_vars): pseudobulk aggregation (src/py.rs:340-357)."""
    ch, keep, nr, nv = _chunk(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    gr = carray(group_of_row, np.uint32, "group_of_row")
    s = _mut(sum, np.float64, "sum")
    if s.ndim != 2 or s.shape[1] != nv or len(gr) < nr:
        raise ValueError("sum must be (n_groups, n_vars); group_of_row (n_rows,)")
    if bool(np.any((gr != np.iinfo(np.uint32).max) & (gr >= s.shape[0]))):
        raise ValueError("group id out of range")
    _lib.call("crest_group_gene_totals", C.byref(ch), ptr(gr), len(gr), s.shape[0], nv, ptr(s))


def t_pvalues(t, df):
    """Two-sided p-values of Student's t, 2 * sf(|t|, df) capped at 1; NaN for a
    non-finite t or df <= 0 (src/py.rs:413-427).  Host arithmetic over one value per
    gene (scipy's Student t distribution function)."""
    from scipy.special import stdtr
    t = np.asarray(t, np.float64)
    df = np.asarray(df, np.float64)
    if t.shape != df.shape:
        raise ValueError("t, df must have equal length")
    ok = np.isfinite(t) & (df > 0)
    p = np.full(t.shape, np.nan)
    p[ok] = np.minimum(2.0 * stdtr(df[ok], -np.abs(t[ok])), 1.0)
    return p


def knn_graph(data, k, exact=None, seed=0):
    """k nearest neighbours of every row of ``data`` (n x d f32), self excluded, ascending
    distance (src/py.rs:52-72).  Returns (indices u32 (n, k'), distances f32 (n, k')) with
    k' = min(k, n - 1).  The search is always exhaustive (``exact`` and ``seed`` are
    accepted for the reference's signature; there is no approximate index)."""
    X = np.asarray(data)
    if X.ndim != 2 or X.dtype != np.float32:
        raise TypeError("data must be a 2-d float32 array")
    if not X.flags.c_contiguous:
        raise ValueError("data must be C-contiguous")
    n, d = X.shape
    kk = max(1, min(int(k), n - 1)) if n > 1 else 0
    idx = np.zeros((n, kk), np.uint32)
    dist = np.zeros((n, kk), np.float32)
    if kk:
        _lib.call("crest_knn_graph", ptr(X), n, d, int(k), ptr(idx), ptr(dist))
    return idx, dist
