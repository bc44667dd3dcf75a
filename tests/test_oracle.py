"""The CPU oracle against the reference's own known-answer and property tests
(src/kernels.rs:565-633, tests/test_crest.py:54-107), restated."""

import numpy as np
import pytest

import oracle
from oracle import pipeline as op


def test_materialize_known_answer():
    """src/kernels.rs:565-578: filters + normalize_total(100) on COO and CSR."""
    cells = np.array([0, 0, 1, 2, 2], np.uint32)
    genes = np.array([0, 1, 0, 1, 2], np.uint32)
    vals = np.array([2.0, 6.0, 5.0, 1.0, 3.0], np.float32)
    cm = np.array([0, -1, 1], np.int64)
    gm = np.array([0, 1, -1], np.int32)
    r, g, x = oracle.materialize(genes, vals, cm, gm, 100.0, False, cells, None, 0)
    assert r.tolist() == [0, 0, 1]
    assert g.tolist() == [0, 1, 1]
    assert np.allclose(x, [25.0, 75.0, 100.0], atol=1e-5)
    indptr = np.array([0, 2, 3, 5], np.int64)
    r2, g2, x2 = oracle.materialize(genes, vals, cm, gm, 100.0, False, None, indptr, 0)
    assert np.array_equal(r, r2) and np.array_equal(g, g2) and np.array_equal(x, x2)


def scaled_gram_case(seed=9, n=200, d=12):
    """The data of src/kernels.rs:580-633 (density 0.35, gene 3 fixed at 50, others U(0.1, 4))."""
    rng = np.random.default_rng(seed)
    dense = np.zeros((n, d))
    rows, genes, vals = [], [], []
    for i in range(n):
        for j in range(d):
            if rng.random() < 0.35:
                x = np.float32(50.0) if j == 3 else np.float32(rng.uniform(0.1, 4.0))
                dense[i, j] = float(x)
                rows.append(i)
                genes.append(j)
                vals.append(x)
    return dense, np.array(rows, np.uint32), np.array(genes, np.uint32), np.array(vals, np.float32)


def test_scaled_gram_matches_dense_covariance():
    """src/kernels.rs:580-633: Gram-based scaled PCA eigenvalues equal the dense
    scaled/clipped/centred covariance's within 1e-9 relative, fed in two chunks."""
    n, d, mv = 200, 12, 2.0
    dense, rows, genes, vals = scaled_gram_case()
    mean = dense.mean(0)
    std = dense.std(0, ddof=1)
    gm = np.arange(d, dtype=np.int32)
    cm = np.arange(n, dtype=np.int64)
    gram = np.zeros((d, d))
    colsum = np.zeros(d)
    cut = int(np.argmax(rows >= 100))
    for lo, hi in ((0, cut), (cut, len(rows))):
        oracle.gram_accumulate(genes[lo:hi], vals[lo:hi], cm, gm, 0.0, False, rows[lo:hi], None, 0, gm, gram, colsum,
                               True, mean, std, mv)
    ev, _, _ = oracle.pca_from_gram(gram, colsum, n, 5)
    z = np.clip((dense - mean) / std, -mv, mv)
    zc = z - z.mean(0)
    ref = np.sort(np.linalg.eigvalsh(zc.T @ zc / (n - 1)))[::-1]
    for c in range(5):
        assert abs(ev[c] - ref[c]) < 1e-9 * max(ref[c], 1.0)


def test_lazy_normalisation_matches_numpy(small_counts):
    """tests/test_crest.py:77-85."""
    indptr, indices, data, n_genes, names, _ = small_counts
    n = len(indptr) - 1
    r, g, x = oracle.materialize(indices, data, np.arange(n, dtype=np.int64), np.arange(n_genes, dtype=np.int32),
                                 1e4, True, None, indptr, 0)
    Y = np.zeros((n, n_genes), np.float32)
    Y[r, g] = x
    D = np.zeros((n, n_genes))
    rows = np.repeat(np.arange(n), np.diff(indptr))
    D[rows, indices] = data
    ref = np.log1p(D / D.sum(1, keepdims=True) * 1e4)
    np.testing.assert_allclose(Y, ref, rtol=1e-5, atol=1e-5)


def _frame(counts, **kw):
    indptr, indices, data, n_genes, names = counts[:5]
    return op.Frame(indptr, indices, data, n_genes, names, threads=4, **kw)


def test_scaled_pca_matches_dense(small_counts):
    """tests/test_crest.py:88-107: implicit scale(2) + Gram PCA equals dense scale + SVD."""
    f = _frame(small_counts)
    op.normalize_total(f, 1e4)
    op.log1p(f)
    op.scale(f, 2.0)
    op.pca(f, n_comps=10, use_highly_variable=False)
    indptr, indices, data = small_counts[:3]
    n = len(indptr) - 1
    r, g, x = oracle.materialize(indices, data, np.arange(n, dtype=np.int64),
                                 np.arange(small_counts[3], dtype=np.int32), 1e4, True, None, indptr, 0)
    D = np.zeros((n, small_counts[3]))
    D[r, g] = x
    mu, sd = D.mean(0), D.std(0, ddof=1)
    sd[sd == 0] = 1
    Z = np.clip((D - mu) / sd, -2, 2)
    Z -= Z.mean(0)
    U, S, _ = np.linalg.svd(Z, full_matrices=False)
    ref = S[:10] ** 2 / (n - 1)
    np.testing.assert_allclose(f.uns["pca"]["variance"], ref, rtol=1e-6)
    ref_scores = U[:, :10] * S[:10]
    got = f.obsm["X_pca"].astype(np.float64)
    cos = np.abs((got * ref_scores).sum(0)) / np.linalg.norm(got, axis=0) / np.linalg.norm(ref_scores, axis=0)
    assert cos.min() > 0.9999


def run_pipeline(f, n_top=300, n_comps=20):
    f = op.filter_cells(f, min_genes=50)
    f = op.filter_genes(f, min_cells=3)
    op.normalize_total(f, 1e4)
    op.log1p(f)
    op.highly_variable_genes(f, n_top_genes=n_top)
    op.scale(f, 10)
    op.pca(f, n_comps=n_comps)
    return f


def test_chunking_invariance(small_counts):
    """tests/test_crest.py:54-61."""
    a = run_pipeline(_frame(small_counts))
    b = run_pipeline(_frame(small_counts, chunk_nnz=1000))
    assert np.array_equal(a.var["highly_variable"], b.var["highly_variable"])
    np.testing.assert_allclose(np.abs(a.obsm["X_pca"]), np.abs(b.obsm["X_pca"]), rtol=1e-4, atol=1e-3)


def test_triplet_and_csr_chunks_agree(small_counts):
    """tests/test_crest.py:64-74 (CSR vs triplet stores)."""
    indptr = small_counts[0]
    cells = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr)).astype(np.uint32)
    a = run_pipeline(_frame(small_counts))
    b = run_pipeline(_frame(small_counts, cells_coo=cells, chunk_nnz=50_000))
    np.testing.assert_allclose(np.abs(a.obsm["X_pca"]), np.abs(b.obsm["X_pca"]), rtol=1e-4, atol=1e-3)


def test_validation_errors_mirror_reference():
    g = np.zeros(3, np.uint32)
    v = np.ones(3, np.float32)
    cm = np.zeros(1, np.int64)
    gm = np.zeros(1, np.int32)
    out = np.zeros((1, 5))
    with pytest.raises(ValueError, match="exactly one"):
        oracle.gene_stats(g, v, cm, gm, 0.0, False, None, None, 0, out)
    with pytest.raises(ValueError, match="span the chunk"):
        oracle.gene_stats(g, v, cm, gm, 0.0, False, None, np.array([0, 2], np.int64), 0, out)
    with pytest.raises(ValueError, match="sorted by cell"):
        oracle.gene_stats(g, v, cm, gm, 0.0, False, np.array([1, 0, 0], np.uint32), None, 0, out)
    with pytest.raises(ValueError, match="n_vars, 5"):
        oracle.gene_stats(g, v, cm, gm, 0.0, False, None, np.array([0, 3], np.int64), 0, np.zeros((2, 5)))
    with pytest.raises(RuntimeError):
        oracle.pca_from_gram(np.zeros((2, 2)), np.zeros(2), 1, 1)


def test_part_split_only_changes_gene_sum_order(small_counts):
    """Emulating 1 vs 8 rayon threads changes per-gene f64 sums by rounding only."""
    f1 = _frame(small_counts)
    f1.threads = 1
    f8 = _frame(small_counts)
    f8.threads = 8
    for f in (f1, f8):
        op.normalize_total(f, 1e4)
        op.log1p(f)
    a, b = op.gene_stats(f1), op.gene_stats(f8)
    np.testing.assert_allclose(a, b, rtol=1e-12)
    assert np.array_equal(a[:, 4], b[:, 4])
