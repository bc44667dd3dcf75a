"""UMAP fuzzy connectivities of a kNN graph (host arithmetic of
crest_b200.pp.connectivities): per cell the directed memberships of its
neighbours sum to log2(n_neighbors) (the smoothing target), the nearest
neighbour has membership 1, the union is symmetric with weights in (0, 1]."""

import numpy as np

import oracle
from crest_b200 import pp


def test_fuzzy_union_properties():
    rng = np.random.default_rng(4)
    X = rng.standard_normal((500, 8)).astype(np.float32)
    idx, dist = oracle.knn_graph(X, 14)
    rows, cols, w = pp.connectivities(idx, dist, 15)
    assert np.all(rows < cols) and np.all((w > 0) & (w <= 1))
    # every directed edge appears (undirected) exactly once
    pairs = set(zip(rows.tolist(), cols.tolist()))
    assert len(pairs) == len(rows)
    for i in range(0, 500, 50):
        for j in idx[i]:
            assert (min(i, j), max(i, j)) in pairs
    # rebuild the directed memberships of one row: they sum to log2(15)
    d = dist[7].astype(np.float64)
    rho = d[d > 0].min()
    lo, hi = 0.0, np.inf
    mid = 1.0
    for _ in range(64):
        s = np.where(d - rho > 0, np.exp(-(d - rho) / mid), 1.0).sum()
        if abs(s - np.log2(15)) < 1e-5:
            break
        if s > np.log2(15):
            hi = mid
            mid = (lo + hi) / 2
        else:
            lo = mid
            mid = mid * 2 if np.isinf(hi) else (lo + hi) / 2
    assert abs(np.where(d - rho > 0, np.exp(-(d - rho) / mid), 1.0).sum() - np.log2(15)) < 1e-4
