"""Tools on :class:`~crest_b200.core.BioFrame`: exact streamed PCA of the
(optionally scaled) matrix via its Gram matrix (the reference's ``crest.tl.pca``,
crest/tl.py:24-91)."""

from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib, _native, dist
from .core import BioFrame
from .pp import _mean_var, gene_stats, group_gene_sums

__all__ = ["pca"]


def _scale_params(bf: BioFrame, mask: np.ndarray):
    """Per-gene log-scale mean/std (ddof=1) for the current ops, cached by HVG (crest/tl.py:24-34)."""
    cached = bf.uns.get("hvg", {}).get("ops") == bf.ops and "mean_log" in bf.var.columns
    if cached:
        mean, std = bf.var["mean_log"].to_numpy(), bf.var["std_log"].to_numpy()
    else:
        st = gene_stats(bf)
        mean, var = _mean_var(st[:, 0], st[:, 1], dist.sum_count(bf.n_obs))
        std = np.sqrt(var)
        std[std == 0] = 1.0
    return np.ascontiguousarray(mean[mask], np.float64), np.ascontiguousarray(std[mask], np.float64)


class PcaPlan:
    """A ``crest_pca`` handle: FP64 Gram accumulators in HBM, eigensolve and projection."""

    def __init__(self, d: int, precision: str = "bf16x3"):
        if precision not in _lib.GRAM_PRECISION:
            raise ValueError(f"gram_precision must be one of {sorted(_lib.GRAM_PRECISION)}")
        h = C.c_void_p()
        _lib.call("crest_pca_create", C.byref(h), int(d), _lib.GRAM_PRECISION[precision])
        self.handle, self.d, self.k = h, int(d), 0

    def accumulate(self, dm, cmap, gmap, target, log, sub_map, n_vars, scale):
        _lib.call("crest_pca_accumulate", self.handle, dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), float(target),
                  int(log), _lib.ptr(sub_map), int(n_vars), C.byref(scale))

    def reset(self):
        _lib.call("crest_pca_reset", self.handle)
        self.k = 0

    def accumulators(self):
        g, c = C.c_void_p(), C.c_void_p()
        _lib.call("crest_pca_accumulators", self.handle, C.byref(g), C.byref(c))
        return g.value, c.value

    def gram(self) -> np.ndarray:
        """The FP64 Gram accumulator (d, d); its upper triangle holds the sums."""
        g = np.zeros((self.d, self.d), np.float64)
        _lib.call("crest_pca_gram", self.handle, _lib.ptr(g))
        return g

    def solve(self, n: int, k: int):
        _lib.call("crest_pca_solve", self.handle, int(n), int(k))
        self.k = int(k)

    def results(self):
        v = np.zeros(self.k, np.float64)
        L = np.zeros((self.d, self.k), np.float64)
        t = np.zeros(1, np.float64)
        c = np.zeros(self.d, np.float64)
        _lib.call("crest_pca_results", self.handle, _lib.ptr(v), _lib.ptr(L), _lib.ptr(t), _lib.ptr(c))
        return v, L, float(t[0]), c

    def project(self, dm, cmap, gmap, target, log, sub_map, n_vars, scale, n_rows, out=None, device_ptr=None):
        if device_ptr is not None:
            _lib.call("crest_pca_project", self.handle, dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), float(target),
                      int(log), _lib.ptr(sub_map), int(n_vars), C.byref(scale), int(n_rows), C.c_void_p(device_ptr),
                      _lib.MEM_DEVICE)
            return None
        if out is None:
            out = np.empty((n_rows, self.k), np.float32)
        _lib.call("crest_pca_project", self.handle, dm.handle, _lib.ptr(cmap), _lib.ptr(gmap), float(target),
                  int(log), _lib.ptr(sub_map), int(n_vars), C.byref(scale), int(n_rows), _lib.ptr(out),
                  _lib.MEM_HOST)
        return out

    def stats(self) -> dict:
        s = _lib.PcaStats()
        _lib.call("crest_pca_stats_get", self.handle, C.byref(s))
        return {"gram_ms": s.gram_ms, "solve_ms": s.solve_ms, "project_ms": s.project_ms, "eig_iters": s.eig_iters,
                "eig_converged": bool(s.eig_converged), "eig_residual": s.eig_residual}

    def close(self):
        if self.handle is not None and self.handle.value:
            _lib.load().crest_pca_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pca(bf: BioFrame, n_comps: int = 50, use_highly_variable: Optional[bool] = None,
        scale: Optional[bool] = None, max_value: Optional[float] = None,
        gram_precision: str = "bf16x3") -> BioFrame:
    """Principal components of the selected genes from their covariance, without
    ever materialising the dense (scaled) matrix.

    One pass accumulates the gene x gene Gram matrix of the selected genes
    (``gram_precision``: "bf16x3" split-BF16 tensor-core products, "fp32" plain
    FP32, "fp64" the reference's FP64 sums), an FP64 eigensolve on the GPU gives
    the loadings and a second pass projects the cells.  With scaling the result
    equals ``sc.pp.scale(max_value) + sc.tl.pca`` on the dense matrix, which is
    never formed.  Adds ``obsm['X_pca']``, ``varm['PCs']``, ``uns['pca']``.
    """
    if use_highly_variable is None:
        use_highly_variable = "highly_variable" in bf.var.columns
    mask = (bf.var["highly_variable"].to_numpy().astype(bool) if use_highly_variable
            else np.ones(bf.n_vars, bool))
    d = int(mask.sum())
    if d < 2:
        raise ValueError("need at least 2 genes for PCA")
    if d > 20_000:
        raise ValueError(f"{d} genes: select highly variable genes first (Gram PCA is O(genes^2) memory)")
    if scale is None:
        scale = "scale" in bf.uns
    if max_value is None:
        max_value = bf.uns.get("scale", {}).get("max_value", 10.0) if scale else 0.0
    sub = np.full(bf.n_vars, -1, np.int32)
    sub[mask] = np.arange(d, dtype=np.int32)
    mean = std = None
    if scale:
        mean, std = _scale_params(bf, mask)
    mv = float(max_value or 0.0)
    n_local = bf.n_obs
    n = dist.sum_count(n_local)  # cells over all ranks (the covariance's n)
    k = min(n_comps, d, n - 1)

    dm = bf.device_matrix()
    stats = None
    if dm is not None:
        cmap, gmap = bf._cell_map(), bf._gene_map()
        target, log = bf._transform()
        t = _lib.Scale(int(bool(scale)), _lib.ptr(mean) if scale else None, _lib.ptr(std) if scale else None, mv)
        plan = PcaPlan(d, gram_precision)
        try:
            plan.accumulate(dm, cmap, gmap, target, log, sub, bf.n_vars, t)
            if dist.active():  # one sum of the FP64 accumulators before the replicated solve
                g_dev, c_dev = plan.accumulators()
                dist.sum_device(g_dev, d * d)
                dist.sum_device(c_dev, d)
            plan.solve(n, k)
            variance, loadings, total, colsum = plan.results()
            X = plan.project(dm, cmap, gmap, target, log, sub, bf.n_vars, t, n_local)
            stats = plan.stats()
        finally:
            plan.close()
        shift = (colsum / n) @ loadings
    else:
        gram = np.zeros((d, d), np.float64)
        colsum = np.zeros(d, np.float64)
        for ctx in bf.iter_ctx():
            _native.gram_accumulate(*ctx, sub, gram, colsum, scale, mean, std, mv, precision=gram_precision)
        gram, colsum = dist.sum_host(gram), dist.sum_host(colsum)
        variance, loadings, total = _native.pca_from_gram(gram, colsum, n, k)
        del gram
        shift = (colsum / n) @ loadings
        X = np.empty((n_local, k), np.float32)
        X[:] = -shift.astype(np.float32)
        for ctx in bf.iter_ctx():
            _native.project(*ctx, sub, loadings, X, scale, mean, std, mv)

    pcs = np.zeros((bf.n_vars, k), np.float32)
    pcs[mask] = loadings
    bf.obsm["X_pca"] = X
    bf.varm["PCs"] = pcs
    bf.uns["pca"] = {"variance": variance, "variance_ratio": variance / total,
                     "params": {"scale": bool(scale), "max_value": max_value,
                                "use_highly_variable": bool(use_highly_variable), "gram_precision": gram_precision},
                     "projection": {"genes": [g for g, m in zip(bf.var_names, mask) if m], "loadings": loadings,
                                    "mean": mean, "std": std, "shift": shift, "ops": list(bf.ops)}}
    if stats is not None:
        bf.uns["pca"]["timings"] = stats
    return bf


# --------------------------------------------------------------------------- differential expression
def _natural_key(label: str):
    """Sort key putting "2" before "10" (digits compared as numbers)."""
    import re
    return [int(t) if t.isdigit() else t for t in re.split(r"(\d+)", label)]


def _bh(p: np.ndarray) -> np.ndarray:
    """Benjamini-Hochberg adjusted p-values (step-up, capped at 1)."""
    n = len(p)
    order = np.argsort(p)
    scaled = p[order] * n / np.arange(1, n + 1)
    adj = np.minimum.accumulate(scaled[::-1])[::-1]
    out = np.empty(n)
    out[order] = np.minimum(adj, 1.0)
    return out


def rank_genes_groups(bf: BioFrame, groupby: str, method: str = "t-test", groups="all",
                      n_genes: Optional[int] = 100):
    """Each group against all other cells with a Welch t-test on the (lazily
    normalised / log-transformed) matrix, as the reference's
    ``crest.tl.rank_genes_groups(method="t-test")`` (crest/tl.py:205-288): the
    per (group, gene) sums come from one GPU pass (group_gene_sums); means,
    variances, Welch's statistic and degrees of freedom, log fold changes, p-values
    and Benjamini-Hochberg adjustment are O(groups x genes) host arithmetic.
    Returns a long DataFrame (group, names, scores, logfoldchanges, pvals,
    pvals_adj) with the top ``n_genes`` genes per group by score, also kept in
    ``uns['rank_genes_groups']``."""
    import pandas as pd
    if method != "t-test":
        raise NotImplementedError("only method='t-test' is provided (the Wilcoxon rank test is not on this path)")
    labels = bf.obs[groupby].astype(str).where(bf.obs[groupby].notna(), None).to_numpy()
    cats = sorted({x for x in labels if x is not None}, key=_natural_key)
    if groups != "all":
        keep = set(groups)
        cats = [c for c in cats if c in keep]
    index = {c: i for i, c in enumerate(cats)}
    none = np.iinfo(np.uint32).max
    grp = np.array([index.get(x, none) if x is not None else none for x in labels], dtype=np.uint32)
    G = len(cats)
    sizes = dist.sum_host(np.bincount(grp[grp != none], minlength=G).astype(np.float64))
    N = sizes.sum()
    s, q, _ = group_gene_sums(bf, grp, G)
    s_all, q_all = s.sum(0), q.sum(0)
    names = np.array(bf.var_names, dtype=object)
    k = bf.n_vars if n_genes is None else min(n_genes, bf.n_vars)
    frames = []
    for i, c in enumerate(cats):
        n1, n2 = sizes[i], N - sizes[i]
        m1 = s[i] / n1
        m2 = (s_all - s[i]) / n2
        lfc = np.log2((np.expm1(m1) + 1e-9) / (np.expm1(m2) + 1e-9))
        v1 = np.maximum((q[i] - n1 * m1 ** 2) / (n1 - 1), 0)
        v2 = np.maximum(((q_all - q[i]) - n2 * m2 ** 2) / (n2 - 1), 0)
        a, b = v1 / n1, v2 / n2
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (m1 - m2) / np.sqrt(a + b)
            df = (a + b) ** 2 / (a ** 2 / (n1 - 1) + b ** 2 / (n2 - 1))
        df = np.where(np.isnan(df), 1.0, df)
        pv = _native.t_pvalues(t, df)
        t = np.where(np.isnan(t), 0.0, t)
        pv = np.where(np.isnan(pv), 1.0, pv)
        padj = _bh(pv)
        top = np.argsort(-t, kind="stable")[:k]
        frames.append(pd.DataFrame({"group": [c] * k, "names": names[top].astype(str), "scores": t[top],
                                    "logfoldchanges": lfc[top], "pvals": pv[top], "pvals_adj": padj[top]}))
    out = pd.concat(frames, ignore_index=True) if frames else pd.DataFrame()
    bf.uns["rank_genes_groups"] = {"params": {"groupby": groupby, "method": method, "reference": "rest"},
                                   "groups": cats, "table": out}
    return out
