"""Per (group, gene) sums (src/kernels.rs:388-442) on the GPU against the
oracle, and rank_genes_groups (t-test) through crest_b200.tl against the
golden tables of the reference's own crest/tl.py.

Tolerances: the reference sums each (group, gene) in entry order, the GPU
with atomics in no fixed order: sums within 1e-12 relative, counts exact.
Differential-expression tables: the same genes in the same order per group,
scores / log fold changes within 1e-9 relative, p-values within 1e-6
relative (scipy's Student t in both the oracle and the product)."""

import os

import numpy as np
import pandas as pd
import pytest

import crest_b200 as cb
import oracle
from crest_b200 import _native

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def chunks(indptr, cuts):
    for a, b in zip(cuts[:-1], cuts[1:]):
        yield a, b, int(indptr[a]), int(indptr[b])


@pytest.mark.parametrize("clip", [False, True])
@pytest.mark.parametrize("coo", [False, True])
def test_group_gene_sums_match_oracle(small_counts, clip, coo):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    rng = np.random.default_rng(21)
    keep_c = rng.random(n) >= 0.1
    cm = np.full(n, -1, np.int64)
    cm[keep_c] = np.arange(keep_c.sum())
    keep_g = rng.random(n_genes) >= 0.2
    gm = np.full(n_genes, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    nr, nv, G = int(keep_c.sum()), int(keep_g.sum()), 7
    grp = rng.integers(0, G, nr).astype(np.uint32)
    grp[rng.random(nr) < 0.1] = np.iinfo(np.uint32).max  # cells without a group
    cl = rng.uniform(0.5, 3.0, (G, nv)) if clip else None
    out = [[np.zeros((G, nv)) for _ in range(3)] for _ in range(2)]
    for a, b, lo, hi in chunks(indptr, [0, 701, n]):
        g, v = indices[lo:hi], data[lo:hi]
        if coo:
            cells = np.repeat(np.arange(a, b, dtype=np.uint32), np.diff(indptr[a:b + 1]))
            args = (g, v, cm, gm, 1e4, True, cells, None, 0)
        else:
            args = (g, v, cm, gm, 1e4, True, None, np.ascontiguousarray(indptr[a:b + 1]), a)
        _native.group_gene_sums(*args, grp, *out[0], cl)
        oracle.group_gene_sums(*args, grp, *out[1], cl)
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-12, atol=1e-12)
    assert np.array_equal(out[0][2], out[1][2])
    tot = [np.zeros((G, nv)), np.zeros((G, nv))]
    p = np.ascontiguousarray(indptr)
    _native.group_gene_totals(indices, data, cm, gm, 0.0, False, None, p, 0, grp, tot[0])
    oracle.group_gene_totals(indices, data, cm, gm, 0.0, False, None, p, 0, grp, tot[1])
    assert np.array_equal(tot[0], tot[1])  # raw integer counts: exact sums


def test_group_gene_sums_rejects_bad_groups(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cm = np.arange(n, dtype=np.int64)
    gm = np.arange(n_genes, dtype=np.int32)
    s = [np.zeros((3, n_genes)) for _ in range(3)]
    bad = np.full(n, 3, np.uint32)
    with pytest.raises(ValueError, match="group id out of range"):
        _native.group_gene_sums(indices, data, cm, gm, 0.0, False, None, indptr, 0, bad, *s)
    with pytest.raises(ValueError, match="group_of_row"):
        _native.group_gene_sums(indices, data, cm, gm, 0.0, False, None, indptr, 0, bad[:10], *s)


@pytest.mark.parametrize("name", ["small", "pbmc3k_like"])
@pytest.mark.parametrize("store", ["csr", "triplets"])
def test_rank_genes_groups_matches_reference_golden(name, store):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.CASES[name]
    indptr, indices, data, n_genes, names = mg.case_input(name)
    labels = mg.case_labels(name)
    g = dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))
    var = pd.DataFrame({"gene_name": names})
    if store == "csr":
        bf = cb.BioFrame.from_csr(indptr, indices, data, n_genes, var=var)
    else:
        cells = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr)).astype(np.uint32)
        bf = cb.BioFrame.from_triplets(cells, indices, data, len(indptr) - 1, n_genes, var=var)
    bf = cb.pp.filter_cells(bf, min_genes=c["min_genes"])
    bf = cb.pp.filter_genes(bf, min_cells=c["min_cells"])
    cb.pp.normalize_total(bf, 1e4)
    cb.pp.log1p(bf)
    bf.obs["cluster"] = [f"c{x}" for x in labels[bf.obs["cell_id"].to_numpy()]]
    tab = cb.tl.rank_genes_groups(bf, "cluster", method="t-test", n_genes=mg.DE_TOP)
    assert np.array_equal(tab["group"].to_numpy().astype(str), g["de_group"])
    assert np.array_equal(tab["names"].to_numpy().astype(str), g["de_names"])
    np.testing.assert_allclose(tab["scores"].to_numpy(), g["de_scores"], rtol=1e-9)
    np.testing.assert_allclose(tab["logfoldchanges"].to_numpy(), g["de_logfoldchanges"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(tab["pvals"].to_numpy(), g["de_pvals"], rtol=1e-6, atol=1e-300)
    np.testing.assert_allclose(tab["pvals_adj"].to_numpy(), g["de_pvals_adj"], rtol=1e-6, atol=1e-300)
    assert "rank_genes_groups" in bf.uns


@pytest.mark.parametrize("name", ["small", "pbmc3k_like"])
@pytest.mark.parametrize("store", ["csr", "triplets"])
def test_seurat_v3_matches_reference_golden(name, store):
    """seurat_v3 HVG (two GPU passes of per (batch, gene) sums of the raw
    counts, the second clipped; loess trend and ranking on the host) against
    the reference's columns: the HVG set, ranks and batch counts identical,
    means / variances within 1e-12 relative, variances_norm within 1e-9."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.CASES[name]
    indptr, indices, data, n_genes, names = mg.case_input(name)
    labels = mg.case_labels(name)
    g = dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))
    var = pd.DataFrame({"gene_name": names})
    if store == "csr":
        bf = cb.BioFrame.from_csr(indptr, indices, data, n_genes, var=var)
    else:
        cells = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr)).astype(np.uint32)
        bf = cb.BioFrame.from_triplets(cells, indices, data, len(indptr) - 1, n_genes, var=var)
    bf = cb.pp.filter_cells(bf, min_genes=c["min_genes"])
    bf = cb.pp.filter_genes(bf, min_cells=c["min_cells"])
    bf.obs["batch"] = [f"b{x % 3}" for x in labels[bf.obs["cell_id"].to_numpy()]]
    for tag, key in (("v3", None), ("v3b", "batch")):
        cb.pp.highly_variable_genes(bf, flavor="seurat_v3", n_top_genes=mg.V3_TOP, batch_key=key)
        assert np.array_equal(bf.var["highly_variable"].to_numpy(), g[f"{tag}_highly_variable"])
        assert np.array_equal(bf.var["highly_variable_nbatches"].to_numpy(), g[f"{tag}_highly_variable_nbatches"])
        assert np.array_equal(bf.var["highly_variable_rank"].to_numpy(), g[f"{tag}_highly_variable_rank"],
                              equal_nan=True)
        for col in ("means", "variances"):
            np.testing.assert_allclose(bf.var[col].to_numpy(), g[f"{tag}_{col}"], rtol=1e-12)
        np.testing.assert_allclose(bf.var["variances_norm"].to_numpy(), g[f"{tag}_variances_norm"], rtol=1e-9)
