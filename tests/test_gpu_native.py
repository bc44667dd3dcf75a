"""GPU parity of the per-chunk entry points (the drop-in for the reference's
native module) against the CPU oracle, on the same seeded inputs.

Bit-exact: QC outputs, per-cell transforms (log1pf), the FP64 Gram and
colsum, the projection given the same loadings.  Tolerances are stated where
the reference's own result depends on summation order (per-gene f64 sums)."""

import numpy as np
import pytest

import oracle
from crest_b200 import _native
from oracle import pipeline as op

pytestmark = pytest.mark.gpu


def chunks_of(indptr, indices, data, cuts):
    for a, b in zip(cuts[:-1], cuts[1:]):
        lo, hi = int(indptr[a]), int(indptr[b])
        yield indices[lo:hi], data[lo:hi], None, np.ascontiguousarray(indptr[a:b + 1]), a


def maps_for(n_cells, n_genes, rng, drop_cells=0.1, drop_genes=0.2):
    keep_c = rng.random(n_cells) >= drop_cells
    keep_g = rng.random(n_genes) >= drop_genes
    cm = np.full(n_cells, -1, np.int64)
    cm[keep_c] = np.arange(keep_c.sum())
    gm = np.full(n_genes, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    return cm, gm, int(keep_c.sum()), int(keep_g.sum())


def test_device_log1pf_is_bit_exact():
    rng = np.random.default_rng(1)
    vals = np.concatenate([
        np.arange(0, 20001, dtype=np.float32),
        rng.uniform(0, 1e4, 400_000).astype(np.float32),
        rng.uniform(0, 2, 200_000).astype(np.float32),
        np.float32(2.0) ** rng.uniform(-40, 60, 200_000).astype(np.float32),
        np.array([0.41421354, 0.41421357, 0.4142136, 1e-30, 3.4e38, 1e-45], np.float32),
    ]).astype(np.float32)
    n = len(vals)
    genes = np.arange(n, dtype=np.uint32)
    indptr = np.arange(n + 1, dtype=np.int64)
    cm = np.arange(n, dtype=np.int64)
    gm = np.arange(n, dtype=np.int32)
    out = np.zeros((n, 5))
    _native.gene_stats(genes, vals, cm, gm, 0.0, True, None, indptr, 0, out)
    _, _, ref = oracle.materialize(genes, vals, cm, gm, 0.0, True, None, indptr, 0)
    assert np.array_equal(out[:, 0], ref.astype(np.float64))


def test_normalised_values_bit_exact(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cm = np.arange(n, dtype=np.int64)
    gm = np.arange(n_genes, dtype=np.int32)
    # one gene per (cell, gene) slot: use cell-major unique gene ids so sums are single values
    ng = int(indptr[-1])
    genes = np.arange(ng, dtype=np.uint32)
    gm_big = np.arange(ng, dtype=np.int32)
    # total must still come from all kept genes: rows keep their own entries
    out = np.zeros((ng, 5))
    _native.gene_stats(genes, data, cm, gm_big, 1e4, True, None, indptr, 0, out)
    _, _, ref = oracle.materialize(genes, data, cm, gm_big, 1e4, True, None, indptr, 0)
    assert np.array_equal(out[:, 0], ref.astype(np.float64))
    assert np.array_equal(out[:, 4], np.ones(ng))
    del gm


@pytest.mark.parametrize("integral", [True, False])
def test_qc_matches_oracle(small_counts, integral):
    indptr, indices, data, n_genes, names = small_counts[:5]
    rng = np.random.default_rng(2)
    if not integral:
        data = (data * rng.uniform(0.5, 1.5, len(data))).astype(np.float32)
    n = len(indptr) - 1
    cm, gm, nr, nv = maps_for(n, n_genes, rng)
    flag = np.zeros(nv, bool)
    flag[:7] = True
    outs = [[np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
            for _ in range(2)]
    cuts = [0, 333, 900, n]
    for ctx in chunks_of(indptr, indices, data, cuts):
        g, v, c, p, f = ctx
        _native.qc(g, v, cm, gm, 0.0, False, c, p, f, flag, *outs[0])
        oracle.qc(g, v, cm, gm, 0.0, False, c, p, f, flag, *outs[1])
    a, b = outs
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])
    if integral:
        assert np.array_equal(a[4], b[4])
    else:
        np.testing.assert_allclose(a[4], b[4], rtol=1e-13)


def test_qc_triplet_chunks(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cells = np.repeat(np.arange(n), np.diff(indptr)).astype(np.uint32)
    rng = np.random.default_rng(3)
    cm, gm, nr, nv = maps_for(n, n_genes, rng)
    flag = np.ones(nv, bool)
    res = []
    for mod in (_native, oracle):
        o = [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
        for lo, hi in ((0, 5000), (5000, len(cells))):
            hi2 = int(np.searchsorted(cells, cells[hi - 1], side="right"))
            lo2 = int(np.searchsorted(cells, cells[lo], side="left")) if lo else 0
            mod.qc(indices[lo2:hi2], data[lo2:hi2], cm, gm, 0.0, False, cells[lo2:hi2], None, 0, flag, *o)
        res.append(o)
    for x, y in zip(*res):
        assert np.array_equal(x, y)


def test_gene_stats_matches_oracle(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cm, gm, nr, nv = maps_for(n, n_genes, np.random.default_rng(4))
    a, b = np.zeros((nv, 5)), np.zeros((nv, 5))
    for g, v, c, p, f in chunks_of(indptr, indices, data, [0, 700, n]):
        _native.gene_stats(g, v, cm, gm, 1e4, True, c, p, f, a)
        oracle.gene_stats(g, v, cm, gm, 1e4, True, c, p, f, b)
    assert np.array_equal(a[:, 4], b[:, 4])
    np.testing.assert_allclose(a[:, :4], b[:, :4], rtol=1e-12, atol=1e-300)


def _scale_params(indptr, indices, data, cm, gm, nv, d_mask):
    st = np.zeros((nv, 5))
    oracle.gene_stats(indices, data, cm, gm, 1e4, True, None, indptr, 0, st)
    n = int((cm >= 0).sum())
    mean = st[:, 0] / n
    var = np.maximum((st[:, 1] - n * mean * mean) / (n - 1), 0)
    std = np.sqrt(var)
    std[std == 0] = 1
    return np.ascontiguousarray(mean[d_mask]), np.ascontiguousarray(std[d_mask])


@pytest.mark.parametrize("scale,mv", [(True, 10.0), (True, 1.0), (False, 0.0)])
def test_gram_fp64_bit_exact(small_counts, scale, mv):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    rng = np.random.default_rng(5)
    cm, gm, nr, nv = maps_for(n, n_genes, rng)
    d_mask = rng.random(nv) < 0.4
    d = int(d_mask.sum())
    sub = np.full(nv, -1, np.int32)
    sub[d_mask] = np.arange(d, dtype=np.int32)
    mean, std = _scale_params(indptr, indices, data, cm, gm, nv, d_mask) if scale else (None, None)
    G = [np.zeros((d, d)), np.zeros((d, d))]
    cs = [np.zeros(d), np.zeros(d)]
    for g, v, c, p, f in chunks_of(indptr, indices, data, [0, 500, 1100, n]):
        _native.gram_accumulate(g, v, cm, gm, 1e4, True, c, p, f, sub, G[0], cs[0], scale, mean, std, mv,
                                precision="fp64")
        oracle.gram_accumulate(g, v, cm, gm, 1e4, True, c, p, f, sub, G[1], cs[1], scale, mean, std, mv)
    iu = np.triu_indices(d)
    assert np.array_equal(G[0][iu], G[1][iu])
    assert np.array_equal(cs[0], cs[1])


@pytest.mark.parametrize("precision,tol", [("fp32", 5e-6), ("bf16x3", 5e-6)])
def test_gram_reduced_precision(small_counts, precision, tol):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    rng = np.random.default_rng(6)
    cm, gm, nr, nv = maps_for(n, n_genes, rng, drop_cells=0.05, drop_genes=0.0)
    d_mask = np.zeros(nv, bool)
    d_mask[rng.choice(nv, 300, replace=False)] = True
    d = 300
    sub = np.full(nv, -1, np.int32)
    sub[d_mask] = np.arange(d, dtype=np.int32)
    mean, std = _scale_params(indptr, indices, data, cm, gm, nv, d_mask)
    G = [np.zeros((d, d)), np.zeros((d, d))]
    cs = [np.zeros(d), np.zeros(d)]
    for g, v, c, p, f in chunks_of(indptr, indices, data, [0, 800, n]):
        _native.gram_accumulate(g, v, cm, gm, 1e4, True, c, p, f, sub, G[0], cs[0], True, mean, std, 10.0,
                                precision=precision)
        oracle.gram_accumulate(g, v, cm, gm, 1e4, True, c, p, f, sub, G[1], cs[1], True, mean, std, 10.0)
    nk = int((cm >= 0).sum())
    # compare the centred covariances (what the eigensolve sees)
    cov = []
    for Gi, ci in zip(G, cs):
        S = np.triu(Gi) + np.triu(Gi, 1).T
        cov.append((S - np.outer(ci, ci) / nk) / (nk - 1))
    err = np.linalg.norm(cov[0] - cov[1]) / np.linalg.norm(cov[1])
    assert err < tol, err
    np.testing.assert_allclose(cs[0], cs[1], rtol=1e-10, atol=1e-9)


def test_project_bit_exact(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    rng = np.random.default_rng(7)
    cm, gm, nr, nv = maps_for(n, n_genes, rng)
    d_mask = rng.random(nv) < 0.5
    d = int(d_mask.sum())
    sub = np.full(nv, -1, np.int32)
    sub[d_mask] = np.arange(d, dtype=np.int32)
    mean, std = _scale_params(indptr, indices, data, cm, gm, nv, d_mask)
    for k in (7, 50, 70):
        L = rng.standard_normal((d, k))
        X = [np.full((nr, k), 0.25, np.float32), np.full((nr, k), 0.25, np.float32)]
        for g, v, c, p, f in chunks_of(indptr, indices, data, [0, 901, n]):
            _native.project(g, v, cm, gm, 1e4, True, c, p, f, sub, L, X[0], True, mean, std, 10.0)
            oracle.project(g, v, cm, gm, 1e4, True, c, p, f, sub, L, X[1], True, mean, std, 10.0)
        assert np.array_equal(X[0], X[1])


@pytest.mark.parametrize("d,k", [(12, 5), (150, 40), (600, 50), (2000, 50)])
def test_pca_from_gram_matches_lapack(d, k):
    rng = np.random.default_rng(d)
    n = 5000
    # a covariance with a decaying spectrum and a few close pairs
    A = rng.standard_normal((n, d)) * (np.linspace(3.0, 0.1, d) ** 1.5)[None, :]
    A = A @ np.linalg.qr(rng.standard_normal((d, d)))[0]
    gram = A.T @ A
    colsum = A.sum(0)
    v0, L0, t0 = oracle.pca_from_gram(gram, colsum, n, k)
    v1, L1, t1 = _native.pca_from_gram(gram, colsum, n, k)
    assert abs(t1 - t0) <= 1e-13 * abs(t0)
    np.testing.assert_allclose(v1, v0, rtol=1e-10, atol=1e-12 * v0[0])
    # columns: same sign convention and direction
    cos = np.abs((L0 * L1).sum(0))
    assert np.all(cos > 1 - 1e-9), cos.min()
    imax = np.argmax(np.abs(L1), axis=0)
    assert np.all(L1[imax, np.arange(k)] > 0)


def _gram_with_spectrum(lam, n, seed):
    """(gram, colsum) whose covariance has eigenvalues lam and random eigenvectors."""
    rng = np.random.default_rng(seed)
    d = len(lam)
    Q = np.linalg.qr(rng.standard_normal((d, d)))[0]
    cov = (Q * lam) @ Q.T
    cov = (cov + cov.T) / 2
    c = rng.uniform(0, 50, d)
    return (n - 1) * cov + np.outer(c, c) / n, c


@pytest.mark.parametrize("kind", ["single_cell", "decay", "rank_deficient", "flat"])
def test_pca_from_gram_spectra(kind):
    """Spectra the block solver meets: one dominant component over a tight
    cluster just above a dense bulk (scaled single-cell data), a power-law
    decay, fewer cells than genes (exact zeros) and a nearly flat spectrum."""
    rng = np.random.default_rng(7)
    d, k, n = 1200, 50, 100_000
    if kind == "single_cell":
        lam = np.concatenate([[7.35], rng.uniform(1.0306, 1.0455, 49), 0.9 + 0.13 * rng.beta(2, 1.2, d - 50)])
    elif kind == "decay":
        lam = 100.0 * np.arange(1, d + 1) ** -1.5
    elif kind == "rank_deficient":
        n = 120
        lam = np.concatenate([rng.exponential(1, n - 1) + 0.1, np.zeros(d - n + 1)])
    else:
        lam = 1 + 1e-3 * rng.standard_normal(d)
    gram, colsum = _gram_with_spectrum(lam, n, 3)
    v0, L0, t0 = oracle.pca_from_gram(gram, colsum, n, k)
    v1, L1, t1 = _native.pca_from_gram(gram, colsum, n, k)
    assert abs(t1 - t0) <= 1e-12 * abs(t0)
    assert np.max(np.abs(v1 - v0)) <= 1e-10 * v0[0]
    assert float(op.subspace_angles_deg(L0, L1).max()) <= 1e-5
    # separated components: same direction and sign
    gap = np.full(k, np.inf)
    gap[:-1] = np.minimum(gap[:-1], (v0[:-1] - v0[1:]) / v0[0])
    gap[1:] = np.minimum(gap[1:], (v0[:-1] - v0[1:]) / v0[0])
    sep = gap[:-1] >= 1e-4
    cos = (L0 * L1).sum(0)[:-1][sep]
    assert np.all(cos > 1 - 1e-9), cos.min()


def test_pca_from_gram_errors():
    with pytest.raises(RuntimeError):
        _native.pca_from_gram(np.eye(3), np.zeros(3), 1, 2)
