"""Preprocessing on :class:`~crest_b200.core.BioFrame` (the reference's
``crest.pp``, crest/pp.py): QC metrics and filters, lazy ``normalize_total`` /
``log1p`` / ``scale``, per-gene statistics and seurat / cell_ranger highly
variable genes.

The count passes run on the GPU: CSR stores through the device-resident
whole-matrix entry points, triplet stores chunk by chunk through the
drop-in native functions (:mod:`crest_b200._native`).  The per-gene HVG math
is O(n_vars) numpy on the host, with the reference's formulas.
"""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import pandas as pd

from . import _lib, _native, dist
from .core import BioFrame

__all__ = ["calculate_qc_metrics", "filter_cells", "filter_genes", "normalize_total", "log1p", "scale",
           "gene_stats", "group_gene_sums", "highly_variable_genes", "hvg_from_stats", "neighbors",
           "connectivities", "connectivities_matrix"]


# --------------------------------------------------------------------------- QC
def _mito_flag(bf: BioFrame, mito_prefix: Optional[str]) -> np.ndarray:
    p = mito_prefix.upper() if mito_prefix else None
    return np.array([bool(p) and n.upper().startswith(p) for n in bf.var_names], dtype=bool)


def _qc_sums(bf: BioFrame, flag: np.ndarray):
    ct = np.zeros(bf.n_obs, np.float64)
    cn = np.zeros(bf.n_obs, np.uint32)
    cf = np.zeros(bf.n_obs, np.float64)
    gn = np.zeros(bf.n_vars, np.uint32)
    gt = np.zeros(bf.n_vars, np.float64)
    dm = bf.device_matrix()
    if dm is not None:
        cmap, gmap = bf._cell_map(), bf._gene_map()
        f = np.ascontiguousarray(flag, dtype=np.bool_)
        _lib.call("crest_matrix_qc", dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), _lib.ptr(f), bf.n_obs, bf.n_vars,
                  _lib.ptr(ct), _lib.ptr(cn), _lib.ptr(cf), _lib.ptr(gn), _lib.ptr(gt))
    else:
        for ctx in bf.iter_ctx(transform=False):
            _native.qc(*ctx, flag, ct, cn, cf, gn, gt)
    # per-gene sums cover the cells of every rank (identity in one process)
    return ct, cn, cf, dist.sum_host(gn), dist.sum_host(gt)


def calculate_qc_metrics(bf: BioFrame, mito_prefix: Optional[str] = "MT-", inplace: bool = True):
    """Per-cell ``total_counts``, ``n_genes_by_counts``, ``pct_counts_mt`` and per-gene
    ``n_cells_by_counts``, ``total_counts`` on the raw counts of kept cells/genes
    (crest/pp.py:25-45)."""
    ct, cn, cf, gn, gt = _qc_sums(bf, _mito_flag(bf, mito_prefix))
    pct = np.divide(cf, ct, out=np.zeros_like(ct), where=ct > 0) * 100.0
    obs = pd.DataFrame({"n_genes_by_counts": cn.astype(np.int64), "total_counts": ct, "pct_counts_mt": pct})
    var = pd.DataFrame({"n_cells_by_counts": gn.astype(np.int64), "total_counts": gt})
    if not inplace:
        return obs, var
    for c in obs.columns:
        bf.obs[c] = obs[c].to_numpy()
    for c in var.columns:
        bf.var[c] = var[c].to_numpy()
    return None


def filter_cells(bf: BioFrame, min_genes: Optional[int] = None, min_counts: Optional[float] = None,
                 max_genes: Optional[int] = None, max_counts: Optional[float] = None,
                 max_pct_mt: Optional[float] = None) -> BioFrame:
    """New BioFrame keeping cells within the thresholds (crest/pp.py:48-65)."""
    obs, _ = calculate_qc_metrics(bf, inplace=False)
    keep = np.ones(bf.n_obs, bool)
    ng, tc, mt = (obs["n_genes_by_counts"].to_numpy(), obs["total_counts"].to_numpy(),
                  obs["pct_counts_mt"].to_numpy())
    if min_genes is not None:
        keep &= ng >= min_genes
    if max_genes is not None:
        keep &= ng <= max_genes
    if min_counts is not None:
        keep &= tc >= min_counts
    if max_counts is not None:
        keep &= tc <= max_counts
    if max_pct_mt is not None:
        keep &= mt <= max_pct_mt
    return bf._subset(obs_mask=keep)


def filter_genes(bf: BioFrame, min_cells: Optional[int] = None, min_counts: Optional[float] = None,
                 max_cells: Optional[int] = None, max_counts: Optional[float] = None) -> BioFrame:
    """New BioFrame keeping genes within the thresholds, counted over kept cells (crest/pp.py:68-82)."""
    _, var = calculate_qc_metrics(bf, inplace=False)
    keep = np.ones(bf.n_vars, bool)
    nc, tc = var["n_cells_by_counts"].to_numpy(), var["total_counts"].to_numpy()
    if min_cells is not None:
        keep &= nc >= min_cells
    if max_cells is not None:
        keep &= nc <= max_cells
    if min_counts is not None:
        keep &= tc >= min_counts
    if max_counts is not None:
        keep &= tc <= max_counts
    return bf._subset(var_mask=keep)


# --------------------------------------------------------------------------- lazy transforms
def normalize_total(bf: BioFrame, target_sum: float = 1e4) -> BioFrame:
    """Scale each cell to ``target_sum`` total counts, applied lazily (crest/pp.py:86-93)."""
    if target_sum is None or target_sum <= 0:
        raise ValueError("target_sum must be positive")
    if any(op[0] == "log1p" for op in bf.ops):
        raise ValueError("normalize_total must come before log1p")
    bf.ops = [op for op in bf.ops if op[0] != "normalize_total"] + [("normalize_total", float(target_sum))]
    return bf


def log1p(bf: BioFrame) -> BioFrame:
    """Natural log(1 + x), applied lazily."""
    if not any(op[0] == "log1p" for op in bf.ops):
        bf.ops.append(("log1p",))
    return bf


def scale(bf: BioFrame, max_value: Optional[float] = 10.0) -> BioFrame:
    """Record ``sc.pp.scale(max_value)`` for :func:`crest_b200.tl.pca`, which applies it exactly
    without densifying the matrix (crest/pp.py:103-111)."""
    bf.uns["scale"] = {"max_value": float(max_value) if max_value else 0.0}
    return bf


# --------------------------------------------------------------------------- gene statistics / HVG
def gene_stats(bf: BioFrame) -> np.ndarray:
    """(n_vars, 5): sum x, sum x^2, sum expm1(x), sum expm1(x)^2, nnz of the transformed matrix."""
    out = np.zeros((bf.n_vars, 5), np.float64)
    dm = bf.device_matrix()
    if dm is not None:
        cmap, gmap = bf._cell_map(), bf._gene_map()
        target, log = bf._transform()
        _lib.call("crest_matrix_gene_stats", dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), float(target), int(log),
                  bf.n_vars, _lib.ptr(out))
    else:
        for ctx in bf.iter_ctx():
            _native.gene_stats(*ctx, out)
    return dist.sum_host(out)


def group_gene_sums(bf: BioFrame, group_of_row: np.ndarray, n_groups: int, clip: Optional[np.ndarray] = None,
                    transform: bool = True, stats: bool = True):
    """Per (group, gene) sum, sum of squares and non-zero count of the (lazily
    transformed, unless ``transform`` is False) matrix, each (n_groups, n_vars);
    ``group_of_row`` gives each cell's group (0xffffffff: none) and ``clip``
    (n_groups, n_vars) caps values first.  With ``stats=False`` only the sums."""
    G, V = int(n_groups), bf.n_vars
    grp = np.ascontiguousarray(group_of_row, dtype=np.uint32)
    if len(grp) != bf.n_obs:
        raise ValueError("group_of_row must have one entry per cell")
    if bool(np.any((grp != np.iinfo(np.uint32).max) & (grp >= G))):
        raise ValueError("group id out of range")
    s = np.zeros((G, V))
    q = np.zeros((G, V)) if stats else None
    z = np.zeros((G, V)) if stats else None
    c = None if clip is None else np.ascontiguousarray(clip, dtype=np.float64)
    if c is not None and c.shape != (G, V):
        raise ValueError("clip must be (n_groups, n_vars)")
    dm = bf.device_matrix()
    if dm is not None:
        cmap, gmap = bf._cell_map(), bf._gene_map()
        target, log = bf._transform() if transform else (0.0, False)
        _lib.call("crest_matrix_group_gene_sums", dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), float(target), int(log),
                  _lib.ptr(grp), len(grp), G, V, _lib.ptr(c), _lib.ptr(s), _lib.ptr(q), _lib.ptr(z))
    else:
        for ctx in bf.iter_ctx(transform=transform):
            if stats:
                _native.group_gene_sums(*ctx, grp, s, q, z, c)
            else:
                _native.group_gene_totals(*ctx, grp, s)
    # sums over the cells of every rank (identity in one process)
    return (dist.sum_host(s), dist.sum_host(q), dist.sum_host(z)) if stats else dist.sum_host(s)


def _mean_var(s1: np.ndarray, s2: np.ndarray, n: int):
    """Mean and ddof=1 variance from sums (crest/pp.py:123-126), clamped at 0."""
    mean = s1 / n
    var = (s2 - n * mean * mean) / (n - 1) if n > 1 else np.zeros_like(mean)
    return mean, np.maximum(var, 0.0)


def _cut_codes(x: np.ndarray, n_bins: int) -> np.ndarray:
    """Bin index of each value under ``pandas.cut(x, n_bins)``: equal-width, right-closed
    bins, the lowest edge pushed down by 0.1% of the range (crest/pp.py:129-136)."""
    lo, hi = float(np.min(x)), float(np.max(x))
    if lo == hi:
        return np.zeros(len(x), np.int64)
    edges = np.linspace(lo, hi, n_bins + 1)
    edges[0] -= (hi - lo) * 0.001
    return np.clip(np.searchsorted(edges, x, side="left") - 1, 0, n_bins - 1)


def highly_variable_genes(bf: BioFrame, n_top_genes: Optional[int] = None, flavor: str = "seurat",
                          n_bins: int = 20, min_mean: float = 0.0125, max_mean: float = 3.0,
                          min_disp: float = 0.5, max_disp: float = np.inf, subset: bool = False,
                          batch_key: Optional[str] = None, span: float = 0.3) -> BioFrame:
    """``sc.pp.highly_variable_genes`` for ``flavor="seurat"`` (log-normalised data),
    ``"cell_ranger"`` and ``"seurat_v3"`` / ``"seurat_v3_paper"`` (crest/pp.py:139-292).

    seurat / cell_ranger add var columns ``means``, ``dispersions``,
    ``dispersions_norm``, ``highly_variable``, ``mean_log``, ``std_log``,
    ``n_cells_expr`` and record the ops the log-scale mean/std were computed under
    (for ``tl.pca``).  seurat_v3 works on the raw counts whatever ops are recorded
    (``n_top_genes`` required, ``batch_key`` optional) and adds ``means``,
    ``variances``, ``variances_norm``, ``highly_variable_rank``,
    ``highly_variable_nbatches``, ``highly_variable``."""
    if flavor in ("seurat_v3", "seurat_v3_paper"):
        if n_top_genes is None:
            raise ValueError("flavor='seurat_v3' needs n_top_genes")
        cols = _hvg_seurat_v3(bf, int(n_top_genes), batch_key, span, flavor)
        for name, v in cols.items():
            bf.var[name] = v
        bf.uns["hvg"] = {"flavor": flavor}
        if subset:
            return bf._subset(var_mask=cols["highly_variable"])
        return bf
    if batch_key is not None:
        raise NotImplementedError("batch_key is supported for flavor='seurat_v3' only")
    cols = hvg_from_stats(gene_stats(bf), dist.sum_count(bf.n_obs), n_top_genes, flavor, n_bins, min_mean,
                          max_mean, min_disp, max_disp)
    for name, v in cols.items():
        bf.var[name] = v
    bf.uns["hvg"] = {"flavor": flavor, "ops": list(bf.ops)}
    if subset:
        return bf._subset(var_mask=cols["highly_variable"])
    return bf


def _hvg_seurat_v3(bf: BioFrame, n_top: int, batch_key: Optional[str], span: float, flavor: str) -> dict:
    """Variance-stabilised HVG ranking of the raw counts (seurat_v3): per batch, a
    loess trend of log10 variance on log10 mean gives each gene an expected
    standard deviation; values are clipped at mean + sd * sqrt(cells) and the
    clipped standardised variance ranks the genes.  Two GPU passes of per
    (batch, gene) sums; the rest is host arithmetic over genes."""
    from .loess import loess_fit
    V = bf.n_vars
    if batch_key is None:
        grp = np.zeros(bf.n_obs, np.uint32)
        n_b = 1
    else:
        labels = bf.obs[batch_key].astype(str).to_numpy()
        cats = np.unique(labels)
        grp = np.searchsorted(cats, labels).astype(np.uint32)
        n_b = len(cats)
    cells = dist.sum_host(np.bincount(grp, minlength=n_b).astype(np.float64))
    s, q, _ = group_gene_sums(bf, grp, n_b, transform=False)
    mean_all, var_all = _mean_var(s.sum(0), q.sum(0), dist.sum_count(bf.n_obs))
    cap = np.zeros((n_b, V))
    mean_b, sd_b = np.zeros((n_b, V)), np.zeros((n_b, V))
    for b in range(n_b):
        mean, var = _mean_var(s[b], q[b], int(cells[b]))
        varying = var > 0
        trend = np.zeros(V)
        trend[varying] = loess_fit(np.log10(mean[varying]), np.log10(var[varying]), span=span, degree=2)
        sd_b[b] = np.sqrt(10 ** trend)
        mean_b[b] = mean
        cap[b] = sd_b[b] * np.sqrt(cells[b]) + mean
    cs, cq, _ = group_gene_sums(bf, grp, n_b, clip=np.ascontiguousarray(cap), transform=False)
    norm = (1.0 / ((cells[:, None] - 1) * sd_b ** 2)) * (cells[:, None] * mean_b ** 2 + cq - 2 * cs * mean_b)
    # the per-batch rank of every gene, with numpy's default (unstable) sort as
    # scanpy uses, so exactly tied genes rank as there
    rank = np.argsort(np.argsort(-norm, axis=1), axis=1).astype(np.float32)
    in_top = (rank < n_top).sum(0)
    rank[rank >= n_top] = np.nan
    with np.errstate(all="ignore"):
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            median_rank = np.nanmedian(rank, axis=0)
    unranked_last = np.where(np.isnan(median_rank), np.inf, median_rank)
    if flavor == "seurat_v3":  # median rank, then number of batches; stable
        order = np.lexsort((-in_top, unranked_last))
    else:  # seurat_v3_paper: number of batches first
        order = np.lexsort((unranked_last, -in_top))
    hv = np.zeros(V, bool)
    hv[order[:n_top]] = True
    return {"means": mean_all, "variances": var_all, "variances_norm": norm.mean(0),
            "highly_variable_rank": median_rank, "highly_variable_nbatches": in_top.astype(np.int64),
            "highly_variable": hv}


def hvg_from_stats(st: np.ndarray, n: int, n_top_genes: Optional[int] = None, flavor: str = "seurat",
                   n_bins: int = 20, min_mean: float = 0.0125, max_mean: float = 3.0, min_disp: float = 0.5,
                   max_disp: float = np.inf) -> dict:
    """The host-side HVG math of crest/pp.py:201-292 from per-gene statistics
    ``st`` (n_vars x 5, :func:`gene_stats`) over ``n`` cells: the var columns."""
    if flavor not in ("seurat", "cell_ranger"):
        raise ValueError('flavor must be "seurat" or "cell_ranger"')
    mean_log, var_log = _mean_var(st[:, 0], st[:, 1], n)
    if flavor == "seurat":
        mean, var = _mean_var(st[:, 2], st[:, 3], n)
    else:
        mean, var = mean_log.copy(), var_log.copy()
    mean = mean.copy()
    mean[mean == 0] = 1e-12
    with np.errstate(divide="ignore", invalid="ignore"):
        disp = var / mean
    if flavor == "seurat":
        disp[disp == 0] = np.nan
        with np.errstate(divide="ignore"):
            disp = np.log(disp)
        mean = np.log1p(mean)
        codes = _cut_codes(mean, n_bins)
        nb = n_bins
    else:
        edges = np.r_[-np.inf, np.percentile(mean, np.arange(10, 105, 5)), np.inf]
        codes = np.clip(np.searchsorted(edges, mean, side="left") - 1, 0, len(edges) - 2)
        nb = len(edges) - 1

    centre = np.full(nb, np.nan)
    spread = np.full(nb, np.nan)
    for b in range(nb):
        vals = disp[(codes == b) & ~np.isnan(disp)]
        if flavor == "seurat":
            if len(vals):
                centre[b] = vals.mean()
            if len(vals) > 1:
                spread[b] = vals.std(ddof=1)
        elif len(vals):
            med = np.median(vals)
            centre[b] = med
            spread[b] = np.median(np.abs(vals - med)) / 0.6744897501960817  # MAD, normal-consistent
    if flavor == "seurat":  # single-gene bins get a normalised dispersion of 1
        single = np.isnan(spread)
        spread[single] = centre[single]
        centre[single] = 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        disp_norm = (disp - centre[codes]) / spread[codes]

    if n_top_genes is not None:
        ok = disp_norm[~np.isnan(disp_norm)]
        k = min(n_top_genes, ok.size, st.shape[0])
        cutoff = np.sort(ok)[::-1][k - 1]
        hv = np.nan_to_num(disp_norm, nan=-np.inf) >= cutoff
    else:
        dn = np.nan_to_num(disp_norm)
        hv = (mean > min_mean) & (mean < max_mean) & (dn > min_disp) & (dn < max_disp)

    std_log = np.sqrt(var_log)
    std_log[std_log == 0] = 1.0
    return {"means": mean, "dispersions": disp, "dispersions_norm": disp_norm, "highly_variable": hv,
            "mean_log": mean_log, "std_log": std_log, "n_cells_expr": st[:, 4].astype(np.int64)}


# --------------------------------------------------------------------------- neighbours
def neighbors(bf: BioFrame, n_neighbors: int = 15, n_pcs: Optional[int] = None, use_rep: str = "X_pca",
              exact: Optional[bool] = None, random_state: int = 0) -> BioFrame:
    """kNN graph of the cells on ``obsm[use_rep]`` plus UMAP fuzzy connectivities
    (``sc.pp.neighbors(method="umap")``; crest/pp.py:296-315).  ``n_neighbors``
    counts the cell itself, as in scanpy.  The neighbours are exact for every
    number of cells (exhaustive GPU search); ``exact`` and ``random_state`` are
    accepted for the reference's signature."""
    if use_rep not in bf.obsm:
        raise KeyError(f"{use_rep!r} not in obsm; run crest_b200.tl.pca first")
    X = bf.obsm[use_rep]
    if n_pcs is not None:
        X = X[:, :n_pcs]
    X = np.ascontiguousarray(X, dtype=np.float32)
    idx, dist = _native.knn_graph(X, n_neighbors - 1, exact=exact, seed=random_state)
    rows, cols, w = connectivities(idx, dist, n_neighbors)
    bf.uns["neighbors"] = {
        "params": {"n_neighbors": n_neighbors, "n_pcs": n_pcs, "use_rep": use_rep, "method": "umap"},
        "indices": idx, "distances": dist, "rows": rows, "cols": cols, "weights": w,
    }
    return bf


def connectivities(indices: np.ndarray, distances: np.ndarray, n_neighbors: int):
    """UMAP's fuzzy simplicial set of a kNN graph (McInnes, Healy & Melville 2018,
    with umap-learn's published smoothing constants): per cell, rho = distance to
    its nearest neighbour and sigma from a 64-step bisection making the memberships
    exp(-(d - rho) / sigma) of its n_neighbors - 1 neighbours sum to
    log2(n_neighbors), floored at 1e-3 of the cell's mean distance (self included
    as 0); the directed memberships are combined by fuzzy union a + b - a b.
    Returns the undirected edges (rows < cols) with their weights."""
    idx = np.asarray(indices, np.int64)
    d = np.asarray(distances, np.float64)
    n, k = d.shape
    if n == 0 or k == 0:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float32)
    target = np.log2(n_neighbors)
    pos = np.where(d > 0, d, np.inf)
    rho = pos.min(axis=1)
    rho[~np.isfinite(rho)] = 0.0
    lo, hi, mid = np.zeros(n), np.full(n, np.inf), np.ones(n)
    done = np.zeros(n, bool)
    for _ in range(64):
        gap = d - rho[:, None]
        psum = np.where(gap > 0, np.exp(-gap / mid[:, None]), 1.0).sum(axis=1)
        done |= np.abs(psum - target) < 1e-5
        act = ~done
        big = act & (psum > target)
        hi = np.where(big, mid, hi)
        small = act & ~big
        lo = np.where(small, mid, lo)
        mid = np.where(big, (lo + hi) / 2, np.where(small, np.where(np.isinf(hi), mid * 2, (lo + hi) / 2), mid))
        if done.all():
            break
    mean_all = d.sum() / (n * (k + 1))
    mean_i = d.sum(axis=1) / (k + 1)
    sigma = np.where(rho > 0, np.maximum(mid, 1e-3 * mean_i), np.maximum(mid, 1e-3 * mean_all))
    gap = d - rho[:, None]
    w = np.where(gap > 0, np.exp(-gap / sigma[:, None]), 1.0)
    src = np.repeat(np.arange(n), k)
    dst = idx.ravel()
    ok = (dst >= 0) & (dst < n) & (dst != src)
    a, b, wv = np.minimum(src, dst)[ok], np.maximum(src, dst)[ok], w.ravel()[ok]
    key = a * n + b
    order = np.argsort(key, kind="stable")
    key, wv = key[order], wv[order]
    uniq, first, count = np.unique(key, return_index=True, return_counts=True)
    w1 = wv[first]
    w2 = np.where(count > 1, wv[np.minimum(first + 1, len(wv) - 1)], 0.0)
    weight = w1 + w2 - w1 * w2
    return (uniq // n).astype(np.uint32), (uniq % n).astype(np.uint32), weight.astype(np.float32)


def connectivities_matrix(bf: BioFrame):
    """Symmetric scipy.sparse CSR connectivities (scanpy ``obsp['connectivities']``)."""
    import scipy.sparse as sp
    nb = bf.uns["neighbors"]
    n = bf.n_obs
    C = sp.coo_matrix((nb["weights"], (nb["rows"], nb["cols"])), shape=(n, n)).tocsr()
    return (C + C.T).tocsr()
