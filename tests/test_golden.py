"""The oracle's restatement of the reference's Python orchestration reproduces
golden vectors made by the reference's own crest/pp.py + crest/tl.py
(tests/golden/make_golden.py), bit for bit."""

import os

import numpy as np
import pytest

import oracle
from oracle import pipeline as op

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
THREADS = 4


def load_case(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.CASES[name]
    indptr, indices, data, n_genes, names = mg.case_input(name)
    g = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    return c, (indptr, indices, data, n_genes, names), g


@pytest.mark.parametrize("name", ["small", "pbmc3k_like"])
def test_oracle_pipeline_matches_reference_golden(name):
    c, (indptr, indices, data, n_genes, names), g = load_case(name)
    assert indptr[-1] == g["input_nnz"][0], "synthetic input drifted from the fixture"
    assert int(indices.astype(np.uint64).sum()) == g["input_checksum"][0]
    f = op.Frame(indptr, indices, data, n_genes, names, threads=THREADS)
    obs0, var0 = op.qc_metrics(f)
    assert np.array_equal(obs0["n_genes_by_counts"], g["qc_n_genes_by_counts"])
    assert np.array_equal(obs0["total_counts"], g["qc_total_counts"])
    assert np.array_equal(obs0["pct_counts_mt"], g["qc_pct_counts_mt"])
    assert np.array_equal(var0["n_cells_by_counts"], g["qc_gene_n_cells"])
    assert np.array_equal(var0["total_counts"], g["qc_gene_total"])
    f = op.filter_cells(f, min_genes=c["min_genes"])
    f = op.filter_genes(f, min_cells=c["min_cells"])
    assert np.array_equal(f.cell_ids, g["kept_cells"]) and np.array_equal(f.gene_ids, g["kept_genes"])
    op.normalize_total(f, 1e4)
    op.log1p(f)
    cols = op.highly_variable_genes(f, n_top_genes=c["n_top"])
    for k in ("dispersions_norm", "mean_log", "std_log"):
        assert np.array_equal(cols[k], g[k], equal_nan=True), k
    assert np.array_equal(cols["highly_variable"], g["highly_variable"])
    op.scale(f, 10)
    op.pca(f, n_comps=c["n_comps"])
    assert np.array_equal(f.uns["pca"]["variance"], g["variance"])
    assert np.array_equal(f.uns["pca"]["variance_ratio"], g["variance_ratio"])
    X = f.obsm["X_pca"][: len(g["X_pca"])]
    assert np.array_equal(X, g["X_pca"])


@pytest.mark.parametrize("name", ["small", "pbmc3k_like"])
def test_oracle_rank_genes_groups_matches_reference_golden(name):
    """rank_genes_groups (t-test, each synthetic cluster vs the rest) of the
    reference's crest/tl.py, run on the oracle's native functions, against the
    oracle's restatement of that host arithmetic: identical tables."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c, (indptr, indices, data, n_genes, names), g = load_case(name)
    labels = mg.case_labels(name)
    f = op.Frame(indptr, indices, data, n_genes, names, threads=THREADS)
    f = op.filter_cells(f, min_genes=c["min_genes"])
    f = op.filter_genes(f, min_cells=c["min_cells"])
    op.normalize_total(f, 1e4)
    op.log1p(f)
    tab = op.rank_genes_groups(f, [f"c{x}" for x in labels[f.cell_ids]], n_genes=mg.DE_TOP)
    assert np.array_equal(tab["group"], g["de_group"])
    assert np.array_equal(tab["names"], g["de_names"])
    for k in ("scores", "logfoldchanges", "pvals", "pvals_adj"):
        assert np.array_equal(tab[k], g[f"de_{k}"]), k
