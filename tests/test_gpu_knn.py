"""Exact kNN on the GPU (src/knn.rs) against the oracle's exhaustive search:
identical neighbour indices and bit-identical distances (same f32 operation
order as the reference's sq_dist), ties by index; edge cases of n and k."""

import numpy as np
import pytest

import oracle
from crest_b200 import _native, pp

pytestmark = pytest.mark.gpu


def clustered(n, d, seed):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-10, 10, (20, d))
    return (centres[np.arange(n) % 20] + rng.uniform(-1.5, 1.5, (n, d))).astype(np.float32)


@pytest.mark.parametrize("n,d,k", [(600, 7, 10), (5000, 50, 14), (3000, 3, 30), (2500, 64, 64), (1500, 100, 5)])
def test_knn_matches_oracle(n, d, k):
    X = clustered(n, d, n + d)
    gi, gd = _native.knn_graph(X, k)
    oi, od = oracle.knn_graph(X, k)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gd, od)
    assert not np.any(gi == np.arange(n)[:, None])  # self excluded


def test_knn_ties_and_duplicates():
    rng = np.random.default_rng(3)
    base = rng.integers(0, 3, (200, 4)).astype(np.float32)  # many exactly equal points and distances
    X = np.concatenate([base, base[:50]])
    gi, gd = _native.knn_graph(X, 12)
    oi, od = oracle.knn_graph(X, 12)
    assert np.array_equal(gi, oi) and np.array_equal(gd, od)
    # ascending distance, ties by index
    for row_i, row_d in zip(gi, gd):
        key = list(zip(row_d.tolist(), row_i.tolist()))
        assert key == sorted(key)


def test_knn_edge_sizes():
    assert _native.knn_graph(np.zeros((0, 5), np.float32), 5)[0].shape == (0, 0)
    assert _native.knn_graph(np.ones((1, 5), np.float32), 5)[0].shape == (1, 0)
    i, d = _native.knn_graph(np.array([[0, 0], [3, 4]], np.float32), 10)
    assert i.tolist() == [[1], [0]] and d.tolist() == [[5.0], [5.0]]
    with pytest.raises(ValueError):
        _native.knn_graph(np.zeros((10, 200), np.float32), 3)


def test_neighbors_on_pca_scores():
    import crest_b200 as cb
    import pandas as pd
    from crest_b200 import synth
    from oracle import synth as osynth
    w = synth.WORKLOADS["pbmc3k_like"]
    indptr, indices, data = osynth.make_workload(w)
    bf = cb.BioFrame.from_csr(indptr, indices, data, w.n_genes,
                              var=pd.DataFrame({"gene_name": synth.gene_names(w.n_genes)}))
    bf = cb.pp.filter_cells(bf, min_genes=200)
    bf = cb.pp.filter_genes(bf, min_cells=3)
    cb.pp.normalize_total(bf, 1e4)
    cb.pp.log1p(bf)
    cb.pp.highly_variable_genes(bf, n_top_genes=2000)
    cb.pp.scale(bf, max_value=10)
    cb.tl.pca(bf, n_comps=50)
    pp.neighbors(bf, n_neighbors=15)
    nb = bf.uns["neighbors"]
    oi, od = oracle.knn_graph(np.ascontiguousarray(bf.obsm["X_pca"], np.float32), 14)
    assert np.array_equal(nb["indices"], oi) and np.array_equal(nb["distances"], od)
    C = pp.connectivities_matrix(bf)
    assert abs(C - C.T).max() == 0 and C.max() <= 1.0
