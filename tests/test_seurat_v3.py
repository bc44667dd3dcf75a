"""seurat_v3 highly variable genes (crest/pp.py:139-198) on CPU: the loess
trend against fits of the reference's own loess (tests/golden/loess.npz),
and the host ranking logic of crest_b200.pp with the per-(batch, gene) sums
taken from the oracle, against the reference's seurat_v3 columns
(tests/golden/*.npz, made by tests/golden/make_golden.py)."""

import os

import numpy as np
import pandas as pd
import pytest

import oracle
from crest_b200 import pp
from crest_b200.loess import loess_fit

HERE = os.path.dirname(os.path.abspath(__file__))


def test_loess_matches_reference_fits():
    g = dict(np.load(os.path.join(HERE, "golden", "loess.npz")))
    for i in range(3):
        fit = loess_fit(g[f"x{i}"], g[f"y{i}"], span=float(g[f"span{i}"][0]), degree=2)
        np.testing.assert_allclose(fit, g[f"fit{i}"], rtol=1e-12, atol=1e-12)


def oracle_group_sums(bf, grp, n_groups, clip=None, transform=True, stats=True):
    G, V = int(n_groups), bf.n_vars
    s, q, z = np.zeros((G, V)), np.zeros((G, V)), np.zeros((G, V))
    for ctx in bf.iter_ctx(transform=transform):
        oracle.group_gene_sums(*ctx, np.ascontiguousarray(grp, np.uint32), s, q, z, clip)
    return (s, q, z) if stats else s


@pytest.mark.parametrize("name", ["small", "pbmc3k_like"])
def test_seurat_v3_host_logic_matches_reference(name, monkeypatch):
    import importlib.util
    import crest_b200 as cb
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c = mg.CASES[name]
    indptr, indices, data, n_genes, names = mg.case_input(name)
    labels = mg.case_labels(name)
    g = dict(np.load(os.path.join(HERE, "golden", f"{name}.npz")))
    monkeypatch.setattr(pp, "group_gene_sums", oracle_group_sums)
    kept = g["kept_cells"]
    gkeep = g["kept_genes"]
    cells = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr)).astype(np.uint32)
    bf = cb.BioFrame.from_triplets(cells, indices, data, len(indptr) - 1, n_genes,
                                   var=pd.DataFrame({"gene_name": names}))
    # the golden filters (kept cells / genes) applied directly: no GPU needed here
    obs_mask = np.isin(bf.obs["cell_id"].to_numpy(), kept)
    var_mask = np.isin(bf.var["gene_id"].to_numpy(), gkeep)
    bf = bf._subset(obs_mask=obs_mask, var_mask=var_mask)
    bf.obs["batch"] = [f"b{x % 3}" for x in labels[kept]]
    for tag, key in (("v3", None), ("v3b", "batch")):
        pp.highly_variable_genes(bf, flavor="seurat_v3", n_top_genes=mg.V3_TOP, batch_key=key)
        assert np.array_equal(bf.var["highly_variable"].to_numpy(), g[f"{tag}_highly_variable"])
        assert np.array_equal(bf.var["highly_variable_nbatches"].to_numpy(), g[f"{tag}_highly_variable_nbatches"])
        assert np.array_equal(bf.var["highly_variable_rank"].to_numpy(), g[f"{tag}_highly_variable_rank"],
                              equal_nan=True)
        for col in ("means", "variances"):
            np.testing.assert_allclose(bf.var[col].to_numpy(), g[f"{tag}_{col}"], rtol=1e-12)
        np.testing.assert_allclose(bf.var["variances_norm"].to_numpy(), g[f"{tag}_variances_norm"], rtol=1e-9)
