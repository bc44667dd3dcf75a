"""CPU ORACLE -- test infrastructure only.

Restatement of the reference's host-side orchestration on the hot path
(crest/core.py chunking and maps, crest/pp.py QC / filters / lazy ops /
seurat HVG, crest/tl.py PCA) over the oracle's native-module mirror.
State is a small :class:`Frame` instead of the reference's polars-backed
BioFrame; the numpy arithmetic is the reference's.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import gene_stats as _gene_stats, gram_accumulate, pca_from_gram, project, qc

DEFAULT_CHUNK_NNZ = 1 << 24


@dataclass
class Frame:
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    n_genes: int
    names: list
    cell_ids: np.ndarray = None   # kept store cells (crest/core.py obs["cell_id"])
    gene_ids: np.ndarray = None   # kept store genes (var["gene_id"])
    ops: list = field(default_factory=list)
    uns: dict = field(default_factory=dict)
    var: dict = field(default_factory=dict)
    obsm: dict = field(default_factory=dict)
    chunk_nnz: int = DEFAULT_CHUNK_NNZ
    threads: Optional[int] = None
    cells_coo: Optional[np.ndarray] = None  # when set, chunks are COO (FrameStore)

    def __post_init__(self):
        n_cells = len(self.indptr) - 1
        if self.cell_ids is None:
            self.cell_ids = np.arange(n_cells, dtype=np.int64)
        if self.gene_ids is None:
            self.gene_ids = np.arange(self.n_genes, dtype=np.int64)

    @property
    def n_obs(self):
        return len(self.cell_ids)

    @property
    def n_vars(self):
        return len(self.gene_ids)

    def subset(self, obs_mask=None, var_mask=None):
        f = Frame(self.indptr, self.indices, self.data, self.n_genes, self.names,
                  self.cell_ids if obs_mask is None else self.cell_ids[obs_mask],
                  self.gene_ids if var_mask is None else self.gene_ids[var_mask],
                  list(self.ops), dict(self.uns), {}, {}, self.chunk_nnz, self.threads, self.cells_coo)
        if var_mask is None:
            f.var = dict(self.var)
        return f

    def var_names(self):
        return [self.names[g] for g in self.gene_ids]

    # crest/core.py:244-263
    def maps(self):
        cm = np.full(len(self.indptr) - 1, -1, np.int64)
        cm[self.cell_ids] = np.arange(self.n_obs, dtype=np.int64)
        gm = np.full(self.n_genes, -1, np.int32)
        gm[self.gene_ids] = np.arange(self.n_vars, dtype=np.int32)
        return cm, gm

    def transform(self):
        target, log = 0.0, False
        for op in self.ops:
            if op[0] == "normalize_total":
                target = float(op[1])
            elif op[0] == "log1p":
                log = True
        return target, log

    # crest/core.py:54-62 (CSR) and :97-105 (triplets)
    def chunks(self):
        if self.cells_coo is not None:
            cells = self.cells_coo
            n = len(cells)
            lo = 0
            while lo < n:
                hi = min(lo + self.chunk_nnz, n)
                if hi < n:
                    hi = int(np.searchsorted(cells, cells[hi - 1], side="right"))
                yield self.indices[lo:hi], self.data[lo:hi], cells[lo:hi], None, 0
                lo = hi
            return
        n = len(self.indptr) - 1
        start = 0
        while start < n:
            target = self.indptr[start] + self.chunk_nnz
            end = int(np.searchsorted(self.indptr, target, side="right")) - 1
            end = min(max(end, start + 1), n)
            lo, hi = int(self.indptr[start]), int(self.indptr[end])
            yield self.indices[lo:hi], self.data[lo:hi], None, self.indptr[start:end + 1], start
            start = end

    def ctx(self, transform=True):
        cm, gm = self.maps()
        target, log = self.transform() if transform else (0.0, False)
        for g, v, c, p, first in self.chunks():
            yield (np.ascontiguousarray(g, np.uint32), np.ascontiguousarray(v, np.float32), cm, gm, target, log,
                   None if c is None else np.ascontiguousarray(c, np.uint32),
                   None if p is None else np.ascontiguousarray(p, np.int64), int(first))


# --------------------------------------------------------------- crest/pp.py
def qc_metrics(f: Frame, mito_prefix="MT-"):
    names = f.var_names()
    flag = np.array([bool(mito_prefix) and n.upper().startswith(mito_prefix.upper()) for n in names], bool)
    ct, cn, cf = np.zeros(f.n_obs), np.zeros(f.n_obs, np.uint32), np.zeros(f.n_obs)
    gn, gt = np.zeros(f.n_vars, np.uint32), np.zeros(f.n_vars)
    for c in f.ctx(transform=False):
        qc(*c, flag, ct, cn, cf, gn, gt, threads=f.threads)
    pct = np.divide(cf, ct, out=np.zeros_like(ct), where=ct > 0) * 100.0
    return {"n_genes_by_counts": cn.astype(np.int64), "total_counts": ct, "pct_counts_mt": pct}, \
        {"n_cells_by_counts": gn.astype(np.int64), "total_counts": gt}


def filter_cells(f: Frame, min_genes=None, min_counts=None, max_genes=None, max_counts=None, max_pct_mt=None):
    obs, _ = qc_metrics(f)
    keep = np.ones(f.n_obs, bool)
    if min_genes is not None:
        keep &= obs["n_genes_by_counts"] >= min_genes
    if max_genes is not None:
        keep &= obs["n_genes_by_counts"] <= max_genes
    if min_counts is not None:
        keep &= obs["total_counts"] >= min_counts
    if max_counts is not None:
        keep &= obs["total_counts"] <= max_counts
    if max_pct_mt is not None:
        keep &= obs["pct_counts_mt"] <= max_pct_mt
    return f.subset(obs_mask=keep)


def filter_genes(f: Frame, min_cells=None, min_counts=None, max_cells=None, max_counts=None):
    _, var = qc_metrics(f)
    keep = np.ones(f.n_vars, bool)
    if min_cells is not None:
        keep &= var["n_cells_by_counts"] >= min_cells
    if max_cells is not None:
        keep &= var["n_cells_by_counts"] <= max_cells
    if min_counts is not None:
        keep &= var["total_counts"] >= min_counts
    if max_counts is not None:
        keep &= var["total_counts"] <= max_counts
    return f.subset(var_mask=keep)


def normalize_total(f: Frame, target_sum=1e4):
    f.ops = [op for op in f.ops if op[0] != "normalize_total"] + [("normalize_total", float(target_sum))]


def log1p(f: Frame):
    if not any(op[0] == "log1p" for op in f.ops):
        f.ops.append(("log1p",))


def scale(f: Frame, max_value=10.0):
    f.uns["scale"] = {"max_value": float(max_value) if max_value else 0.0}


def gene_stats(f: Frame):
    out = np.zeros((f.n_vars, 5))
    for c in f.ctx():
        _gene_stats(*c, out, threads=f.threads)
    return out


def mean_var(s1, s2, n):
    mean = s1 / n
    var = (s2 - n * mean * mean) / (n - 1) if n > 1 else np.zeros_like(mean)
    return mean, np.maximum(var, 0.0)


def cut_codes(x, n_bins):
    lo, hi = float(np.min(x)), float(np.max(x))
    if lo == hi:
        return np.zeros(len(x), np.int64)
    edges = np.linspace(lo, hi, n_bins + 1)
    edges[0] -= (hi - lo) * 0.001
    return np.clip(np.searchsorted(edges, x, side="left") - 1, 0, n_bins - 1)


def hvg_from_stats(st, n, n_top_genes=None, flavor="seurat", n_bins=20, min_mean=0.0125, max_mean=3.0,
                   min_disp=0.5, max_disp=np.inf):
    """crest/pp.py:227-287 on a gene_stats table."""
    mean_log, var_log = mean_var(st[:, 0], st[:, 1], n)
    if flavor == "seurat":
        mean, var = mean_var(st[:, 2], st[:, 3], n)
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
        codes = cut_codes(mean, n_bins)
        nb = n_bins
    else:
        edges = np.r_[-np.inf, np.percentile(mean, np.arange(10, 105, 5)), np.inf]
        codes = np.clip(np.searchsorted(edges, mean, side="left") - 1, 0, len(edges) - 2)
        nb = len(edges) - 1
    avg = np.full(nb, np.nan)
    dev = np.full(nb, np.nan)
    for b in range(nb):
        d = disp[(codes == b) & ~np.isnan(disp)]
        if flavor == "seurat":
            if len(d):
                avg[b] = d.mean()
            if len(d) > 1:
                dev[b] = d.std(ddof=1)
        elif len(d):
            med = np.median(d)
            avg[b] = med
            dev[b] = np.median(np.abs(d - med)) / 0.6744897501960817
    if flavor == "seurat":
        one = np.isnan(dev)
        dev[one] = avg[one]
        avg[one] = 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        disp_norm = (disp - avg[codes]) / dev[codes]
    if n_top_genes is not None:
        x = disp_norm[~np.isnan(disp_norm)]
        k = min(n_top_genes, x.size, len(disp_norm))
        cutoff = np.sort(x)[::-1][k - 1]
        hv = np.nan_to_num(disp_norm, nan=-np.inf) >= cutoff
    else:
        dn = np.nan_to_num(disp_norm)
        hv = (mean > min_mean) & (mean < max_mean) & (dn > min_disp) & (dn < max_disp)
    std_log = np.sqrt(var_log)
    std_log[std_log == 0] = 1.0
    return {"means": mean, "dispersions": disp, "dispersions_norm": disp_norm, "highly_variable": hv,
            "mean_log": mean_log, "std_log": std_log, "n_cells_expr": st[:, 4].astype(np.int64)}


def highly_variable_genes(f: Frame, **kw):
    st = gene_stats(f)
    cols = hvg_from_stats(st, f.n_obs, **kw)
    f.var.update(cols)
    f.uns["hvg"] = {"ops": list(f.ops)}
    return cols


# --------------------------------------------------------------- crest/tl.py
def pca(f: Frame, n_comps=50, use_highly_variable=None, scale=None, max_value=None, gram_fn=None):
    """crest/tl.py:37-91; ``gram_fn`` may replace the FP64 oracle Gram (e.g. to test
    reduced-precision Gram matrices through the same epilogue)."""
    if use_highly_variable is None:
        use_highly_variable = "highly_variable" in f.var
    mask = np.asarray(f.var["highly_variable"], bool) if use_highly_variable else np.ones(f.n_vars, bool)
    d = int(mask.sum())
    if scale is None:
        scale = "scale" in f.uns
    if max_value is None:
        max_value = f.uns.get("scale", {}).get("max_value", 10.0) if scale else 0.0
    gmap = np.full(f.n_vars, -1, np.int32)
    gmap[mask] = np.arange(d, dtype=np.int32)
    mean = std = None
    if scale:
        if f.uns.get("hvg", {}).get("ops") == f.ops and "mean_log" in f.var:
            mean, std = np.asarray(f.var["mean_log"]), np.asarray(f.var["std_log"])
        else:
            st = gene_stats(f)
            mean, var = mean_var(st[:, 0], st[:, 1], f.n_obs)
            std = np.sqrt(var)
            std[std == 0] = 1.0
        mean, std = np.ascontiguousarray(mean[mask], np.float64), np.ascontiguousarray(std[mask], np.float64)
    n = f.n_obs
    gram = np.zeros((d, d))
    colsum = np.zeros(d)
    for c in f.ctx():
        gram_accumulate(*c, gmap, gram, colsum, scale, mean, std, float(max_value or 0.0), threads=f.threads)
    if gram_fn is not None:
        gram, colsum = gram_fn(gram, colsum)
    k = min(n_comps, d, n - 1)
    variance, loadings, total = pca_from_gram(gram, colsum, n, k)
    shift = (colsum / n) @ loadings
    X = np.empty((n, k), np.float32)
    X[:] = -shift.astype(np.float32)
    for c in f.ctx():
        project(*c, gmap, loadings, X, scale, mean, std, float(max_value or 0.0), threads=f.threads)
    f.obsm["X_pca"] = X
    f.uns["pca"] = {"variance": variance, "variance_ratio": variance / total, "loadings": loadings,
                    "shift": shift, "mean": mean, "std": std, "gram": gram, "colsum": colsum}
    return f


def principal_angles_deg(A, B):
    """Principal angles (degrees) between the column spaces of A and B, after centring
    (QR of both, singular values of Qa^T Qb; the reference's accuracy harness)."""
    A = np.asarray(A, np.float64) - np.asarray(A, np.float64).mean(0)
    B = np.asarray(B, np.float64) - np.asarray(B, np.float64).mean(0)
    qa, _ = np.linalg.qr(A)
    qb, _ = np.linalg.qr(B)
    s = np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), -1.0, 1.0)
    return np.degrees(np.arccos(s))


def subspace_angles_deg(U, V):
    """Principal angles between column spaces of U and V without centring."""
    qa, _ = np.linalg.qr(np.asarray(U, np.float64))
    qb, _ = np.linalg.qr(np.asarray(V, np.float64))
    s = np.clip(np.linalg.svd(qa.T @ qb, compute_uv=False), -1.0, 1.0)
    return np.degrees(np.arccos(s))


# --------------------------------------------------------------- crest/tl.py rank_genes_groups
def rank_genes_groups(f: Frame, labels, n_genes=100):
    """crest/tl.py:205-288, method "t-test": per (group, gene) sums over chunks
    (group_gene_sums), then Welch's t, log fold change, p-values and BH per group.
    ``labels`` holds one label (or None) per kept cell.  Returns a dict of columns."""
    import re
    from . import group_gene_sums, t_pvalues

    def nat(s):
        return [int(t) if t.isdigit() else t for t in re.split(r"(\d+)", s)]

    labels = [None if x is None else str(x) for x in labels]
    cats = sorted({x for x in labels if x is not None}, key=nat)
    code = {c: i for i, c in enumerate(cats)}
    none = np.iinfo(np.uint32).max
    grp = np.array([code.get(x, none) if x is not None else none for x in labels], dtype=np.uint32)
    G, V = len(cats), f.n_vars
    sizes = np.bincount(grp[grp != none], minlength=G).astype(np.float64)
    N = sizes.sum()
    s, q, z = np.zeros((G, V)), np.zeros((G, V)), np.zeros((G, V))
    for c in f.ctx():
        group_gene_sums(*c, grp, s, q, z, None)
    S_all, Q_all = s.sum(0), q.sum(0)
    names = np.array(f.var_names(), dtype=object)
    k = V if n_genes is None else min(n_genes, V)
    cols = {"group": [], "names": [], "scores": [], "logfoldchanges": [], "pvals": [], "pvals_adj": []}
    for i, cat in enumerate(cats):
        n1, n2 = sizes[i], N - sizes[i]
        m1 = s[i] / n1
        m2 = (S_all - s[i]) / n2
        logfc = np.log2((np.expm1(m1) + 1e-9) / (np.expm1(m2) + 1e-9))
        v1 = np.maximum((q[i] - n1 * m1 ** 2) / (n1 - 1), 0)
        v2 = np.maximum(((Q_all - q[i]) - n2 * m2 ** 2) / (n2 - 1), 0)
        a, b = v1 / n1, v2 / n2
        with np.errstate(divide="ignore", invalid="ignore"):
            sc = (m1 - m2) / np.sqrt(a + b)
            df = (a + b) ** 2 / (a ** 2 / (n1 - 1) + b ** 2 / (n2 - 1))
        df = np.where(np.isnan(df), 1.0, df)
        pv = t_pvalues(np.ascontiguousarray(sc), np.ascontiguousarray(df))
        sc = np.where(np.isnan(sc), 0.0, sc)
        pv = np.where(np.isnan(pv), 1.0, pv)
        n = len(pv)
        order = np.argsort(pv)
        ranked = pv[order] * n / np.arange(1, n + 1)
        adj = np.minimum.accumulate(ranked[::-1])[::-1]
        padj = np.empty(n)
        padj[order] = np.minimum(adj, 1.0)
        top = np.argsort(-sc, kind="stable")[:k]
        cols["group"] += [cat] * k
        cols["names"] += list(names[top].astype(str))
        cols["scores"] += list(sc[top])
        cols["logfoldchanges"] += list(logfc[top])
        cols["pvals"] += list(pv[top])
        cols["pvals_adj"] += list(padj[top])
    return {key: np.asarray(v) for key, v in cols.items()}
