"""Generate golden vectors by running the reference's own, unmodified Python
orchestration (crest/core.py, crest/pp.py, crest/tl.py of harshameghadri/CREST)
on the seeded synthetic workloads.

The reference's compiled module ``crest.crest`` (Rust, PyO3) cannot be built
here and polars is not installed, so two stand-ins are injected:

* ``crest.crest``  -> the oracle's native-module mirror (oracle/__init__.py),
  the C restatement of src/kernels.rs with the same Python signatures;
* ``polars``       -> the minimal DataFrame/Series surface the hot path uses,
  backed by numpy (FakePolars below).

Everything else -- maps, chunking, QC thresholds, lazy ops, the seurat HVG
arithmetic, the PCA epilogue -- is the reference's code.  The outputs pin the
oracle's own restatement of that orchestration (tests/test_golden.py).

Run from the repository root, giving the path of a checkout of the
reference:  python tests/golden/make_golden.py <reference checkout>
"""

from __future__ import annotations

import os
import sys
import types

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = None  # the reference checkout, from the command line
OUT = os.path.dirname(os.path.abspath(__file__))
THREADS = 4  # rayon thread count emulated by the oracle (fixes the per-gene sum order)
DE_TOP = 25  # genes per group kept in the differential-expression fixture
V3_TOP = 200  # seurat_v3 HVG count of the fixture


# ------------------------------------------------------------------ fake polars
class Series:
    def __init__(self, name, values=None):
        if values is None and not isinstance(name, str):
            name, values = "", name
        self.name = name
        self.v = np.asarray(values)

    def to_numpy(self):
        return self.v

    def cast(self, _t):
        return Series(self.name, self.v.astype(str))

    def to_list(self):
        return self.v.tolist()

    def fill_nan(self, value):
        v = self.v.astype(object)
        v[np.isnan(self.v.astype(float))] = value
        return Series(self.name, v)

    def __len__(self):
        return len(self.v)

    def __eq__(self, other):
        return Series(self.name, self.v == (other.v if isinstance(other, Series) else other))

    def all(self):
        return bool(np.all(self.v))


class DataFrame:
    def __init__(self, data=None):
        self.cols = {}
        if isinstance(data, dict):
            for k, v in data.items():
                self.cols[k] = np.asarray(v)
        elif isinstance(data, (list, tuple)):
            for s in data:
                self.cols[s.name] = np.asarray(s.v)

    @property
    def height(self):
        return len(next(iter(self.cols.values()))) if self.cols else 0

    @property
    def columns(self):
        return list(self.cols)

    def __getitem__(self, k):
        return Series(k, self.cols[k])

    def with_columns(self, *series):
        d = DataFrame()
        d.cols = dict(self.cols)
        items = series[0] if len(series) == 1 and isinstance(series[0], (list, tuple)) else series
        for s in items:
            d.cols[s.name] = np.asarray(s.v)
        return d

    def sort(self, by, descending, nulls_last=True, maintain_order=True):
        """Stable multi-key sort; NaN / None sort after every number (polars' order)."""
        keys = []
        for name, desc in zip(by, descending):
            v = self.cols[name].astype(float)
            v = np.where(np.isnan(v), np.inf, -v if desc else v) if not desc else np.where(np.isnan(v), np.inf, -v)
            keys.append(v)
        order = np.lexsort(tuple(reversed(keys)))
        d = DataFrame()
        d.cols = {k: v[order] for k, v in self.cols.items()}
        return d

    def filter(self, mask):
        m = np.asarray(mask.v if isinstance(mask, Series) else mask, bool)
        d = DataFrame()
        d.cols = {k: v[m] for k, v in self.cols.items()}
        return d

    def drop(self, names):
        names = {names} if isinstance(names, str) else set(names)
        d = DataFrame()
        d.cols = {k: v for k, v in self.cols.items() if k not in names}
        return d

    def hstack(self, other):
        d = DataFrame()
        d.cols = dict(self.cols)
        d.cols.update(other.cols)
        return d

    def clone(self):
        d = DataFrame()
        d.cols = {k: v.copy() for k, v in self.cols.items()}
        return d


def concat(frames):
    d = DataFrame()
    d.cols = {k: np.concatenate([f.cols[k] for f in frames]) for k in frames[0].cols} if frames else {}
    return d


def install_fakes():
    pl = types.ModuleType("polars")
    pl.Series, pl.DataFrame, pl.concat = Series, DataFrame, concat
    pl.Utf8, pl.UInt32, pl.Float32, pl.Int64 = "utf8", "u32", "f32", "i64"
    sys.modules["polars"] = pl
    sys.path.insert(0, ROOT)
    import oracle
    os.environ["CREST_ORACLE_THREADS"] = str(THREADS)
    oracle.DEFAULT_THREADS = THREADS
    sys.modules["crest.crest"] = oracle
    sys.dont_write_bytecode = True
    sys.path.insert(0, REF)
    import crest  # the reference package
    return crest


def run_reference(crest, indptr, indices, data, n_genes, names, n_top, n_comps, min_genes, min_cells,
                  chunk_nnz=None, labels=None):
    bf = crest.BioFrame.from_csr(indptr, indices, data, n_genes, var=DataFrame({"gene_name": np.array(names)}))
    if chunk_nnz:
        bf.chunk_nnz = chunk_nnz
    obs0, var0 = crest.pp.calculate_qc_metrics(bf, inplace=False)
    bf = crest.pp.filter_cells(bf, min_genes=min_genes)
    bf = crest.pp.filter_genes(bf, min_cells=min_cells)
    crest.pp.normalize_total(bf, 1e4)
    crest.pp.log1p(bf)
    crest.pp.highly_variable_genes(bf, n_top_genes=n_top)
    crest.pp.scale(bf, max_value=10)
    crest.tl.pca(bf, n_comps=n_comps)
    de = {}
    if labels is not None:  # seurat_v3 HVG on the raw counts of the filtered cells, with and without batches
        raw = crest.BioFrame.from_csr(indptr, indices, data, n_genes, var=DataFrame({"gene_name": np.array(names)}))
        raw = crest.pp.filter_cells(raw, min_genes=min_genes)
        raw = crest.pp.filter_genes(raw, min_cells=min_cells)
        kept = raw.obs["cell_id"].to_numpy().astype(np.int64)
        raw.obs = raw.obs.with_columns(Series("batch", np.array([f"b{x % 3}" for x in labels[kept]])))
        for tag, key in (("v3", None), ("v3b", "batch")):
            crest.pp.highly_variable_genes(raw, flavor="seurat_v3", n_top_genes=V3_TOP, batch_key=key)
            for col in ("means", "variances", "variances_norm", "highly_variable_rank",
                        "highly_variable_nbatches", "highly_variable"):
                v = raw.var[col].to_numpy()
                de[f"{tag}_{col}"] = v.astype(float) if v.dtype == object else v
    if labels is not None:  # differential expression of the synthetic clusters (t-test, each vs rest)
        kept = bf.obs["cell_id"].to_numpy().astype(np.int64)
        bf.obs = bf.obs.with_columns(Series("cluster", np.array([f"c{x}" for x in labels[kept]])))
        tab = crest.tl.rank_genes_groups(bf, "cluster", method="t-test", n_genes=DE_TOP)
        de.update({f"de_{k}": tab[k].to_numpy() for k in ("group", "names", "scores", "logfoldchanges", "pvals",
                                                           "pvals_adj")})
        de["de_group"] = de["de_group"].astype(str)
        de["de_names"] = de["de_names"].astype(str)
    return {**de,
        "qc_n_genes_by_counts": obs0["n_genes_by_counts"].to_numpy().astype(np.int64),
        "qc_total_counts": obs0["total_counts"].to_numpy(),
        "qc_pct_counts_mt": obs0["pct_counts_mt"].to_numpy(),
        "qc_gene_n_cells": var0["n_cells_by_counts"].to_numpy().astype(np.int64),
        "qc_gene_total": var0["total_counts"].to_numpy(),
        "kept_cells": bf.obs["cell_id"].to_numpy().astype(np.int64),
        "kept_genes": bf.var["gene_id"].to_numpy().astype(np.int64),
        "means": bf.var["means"].to_numpy(),
        "dispersions": bf.var["dispersions"].to_numpy(),
        "dispersions_norm": bf.var["dispersions_norm"].to_numpy(),
        "highly_variable": bf.var["highly_variable"].to_numpy().astype(bool),
        "mean_log": bf.var["mean_log"].to_numpy(),
        "std_log": bf.var["std_log"].to_numpy(),
        "variance": bf.uns["pca"]["variance"],
        "variance_ratio": bf.uns["pca"]["variance_ratio"],
        "shift": bf.uns["pca"]["projection"]["shift"],
        "X_pca": bf.obsm["X_pca"],
        "PCs": bf.varm["PCs"],
    }


CASES = {
    # the reference test suite's fixture shape (tests/test_crest.py:13-50)
    "small": dict(kind="params", args=(1500, 600, 5, 0.5, 150.0, 0), n_top=300, n_comps=20, min_genes=50,
                  min_cells=3),
    # the CPU-runnable 2,700-cell workload (filter 200/3, HVG 2000, 50 PCs)
    "pbmc3k_like": dict(kind="workload", name="pbmc3k_like", n_top=2000, n_comps=50, min_genes=200, min_cells=3),
}


def case_labels(name):
    """Cluster label of every input cell (the generator's own assignment)."""
    sys.path.insert(0, ROOT)
    from crest_b200 import synth
    c = CASES[name]
    if c["kind"] == "params":
        return synth.make_params(*c["args"]).labels
    return synth.workload_params(synth.WORKLOADS[c["name"]]).labels


def case_input(name):
    sys.path.insert(0, ROOT)
    from crest_b200 import synth
    from oracle import synth as osynth
    c = CASES[name]
    if c["kind"] == "params":
        p = synth.make_params(*c["args"])
        indptr, indices, data = osynth.generate(p)
        n_genes = c["args"][1]
    else:
        w = synth.WORKLOADS[c["name"]]
        indptr, indices, data = osynth.make_workload(w)
        n_genes = w.n_genes
    return indptr, indices, data, n_genes, synth.gene_names(n_genes)


def loess_fixture(crest):
    """Fits of the reference's loess (crest/_loess.py) on seeded (x, y) sets:
    mean-variance clouds like seurat_v3's, a smooth curve, and data with ties."""
    from crest._loess import loess_fit
    rng = np.random.default_rng(5)
    out = {}
    x1 = rng.normal(-1.0, 1.0, 800)
    y1 = 1.2 * x1 + 0.3 * x1 ** 2 + rng.normal(0, 0.2, 800)
    x2 = np.linspace(0, 6, 300)
    y2 = np.sin(x2) + rng.normal(0, 0.05, 300)
    x3 = np.round(rng.uniform(0, 3, 500), 1)  # many exact ties
    y3 = np.exp(-x3) + rng.normal(0, 0.02, 500)
    for i, (x, y, span) in enumerate(((x1, y1, 0.3), (x2, y2, 0.5), (x3, y3, 0.3))):
        out[f"x{i}"], out[f"y{i}"], out[f"span{i}"] = x, y, np.array([span])
        out[f"fit{i}"] = loess_fit(x, y, span=span, degree=2)
    path = os.path.join(OUT, "loess.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def main():
    crest = install_fakes()
    loess_fixture(crest)
    for name, c in CASES.items():
        indptr, indices, data, n_genes, names = case_input(name)
        res = run_reference(crest, indptr, indices, data, n_genes, names, c["n_top"], c["n_comps"], c["min_genes"],
                            c["min_cells"], labels=case_labels(name))
        if name != "small":  # keep the committed fixture small
            res["X_pca"] = res["X_pca"][:256]
            res["PCs"] = res["PCs"][res["highly_variable"]][:, :10]
            for k in ("means", "dispersions"):
                del res[k]
        res["input_nnz"] = np.array([indptr[-1]])
        res["input_checksum"] = np.array([int(indices.astype(np.uint64).sum()), int(data.astype(np.float64).sum())])
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **res)
        print(path, os.path.getsize(path), "bytes;", int(res["highly_variable"].sum()), "HVG;",
              len(res["kept_cells"]), "cells")


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], "crest")):
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout (holds crest/)>")
    REF = os.path.abspath(sys.argv[1])
    main()
