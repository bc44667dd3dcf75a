"""Gene-range sweeps of a device-resident matrix (k_sweep.cu) against the
oracle: the per-gene QC sums and gene_stats of crest_matrix_qc /
crest_matrix_gene_stats, with the entry-parallel kernels taking over for
unsorted rows and (QC) non-integral values.

Bar: QC bit-exact (integers, and f64 sums of integers); gene_stats counts
bit-exact and the f64 sums within 1e-12 relative (their order, like the
reference's per-part sums, is not fixed)."""

import numpy as np
import pytest

import oracle
from crest_b200 import _lib, core

pytestmark = pytest.mark.gpu

N_GENES = 13_000  # four gene ranges of 4096


def make(n_cells, seed, integral=True, unsorted_rows=0, beyond=0):
    """Random CSR with sorted rows: empty rows, rows denser than one
    window load (> 256 entries in a range), explicit zeros, and `beyond`
    entries whose gene id is past N_GENES (dropped by every map)."""
    rng = np.random.default_rng(seed)
    nnz = rng.integers(0, 300, n_cells)
    nnz[::17] = 0
    nnz[5::29] = rng.integers(1200, 2500, len(nnz[5::29]))
    indptr = np.concatenate([[0], np.cumsum(nnz)]).astype(np.int64)
    idx = np.empty(indptr[-1], np.uint32)
    for c in range(n_cells):
        idx[indptr[c]:indptr[c + 1]] = np.sort(rng.choice(N_GENES + 64 * (beyond > 0), nnz[c], replace=False))
    if integral:
        val = rng.negative_binomial(2, 0.3, len(idx)).astype(np.float32)
    else:
        val = rng.lognormal(0.0, 1.0, len(idx)).astype(np.float32)
        val[::11] = 0.0
    rows = np.flatnonzero(nnz > 3)[:unsorted_rows]
    for c in rows:
        seg = slice(indptr[c], indptr[c + 1])
        idx[seg] = idx[seg][::-1]
    return indptr, idx, val


def maps(n_cells, seed):
    rng = np.random.default_rng(seed)
    keep_c = rng.random(n_cells) >= 0.1
    keep_g = rng.random(N_GENES) >= 0.2
    cm = np.full(n_cells, -1, np.int64)
    cm[keep_c] = np.arange(keep_c.sum())
    gm = np.full(N_GENES, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    return cm, gm, int(keep_c.sum()), int(keep_g.sum())


def qc_both(indptr, idx, val, cm, gm, nr, nv, residency="device"):
    flag = np.zeros(nv, np.bool_)
    flag[::9] = True
    m = core.DeviceMatrix(indptr, idx, val, N_GENES, residency, chunk_cells=700)
    got = [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
    for _ in range(2):  # the second call reuses the range index
        for a in got:
            a[:] = 0
        _lib.call("crest_matrix_qc", m.handle, _lib.ptr(cm), _lib.ptr(gm), _lib.ptr(flag), nr, nv,
                  *[_lib.ptr(a) for a in got])
    m.close()
    ref = [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
    oracle.qc(idx, val, cm, gm, 0.0, False, None, indptr, 0, flag, *ref)
    return got, ref


def stats_both(indptr, idx, val, cm, gm, nv, target=1e4, log=True, residency="device", gm2=None):
    m = core.DeviceMatrix(indptr, idx, val, N_GENES, residency, chunk_cells=700)
    outs = []
    for g in (gm,) if gm2 is None else (gm, gm2, gm):  # totals re-formed when the map changes
        nvg = int(g.max()) + 1
        o = np.zeros((nvg, 5))
        _lib.call("crest_matrix_gene_stats", m.handle, _lib.ptr(cm), _lib.ptr(g), float(target), int(log), nvg,
                  _lib.ptr(o))
        r = np.zeros((nvg, 5))
        oracle.gene_stats(idx, val, cm, g, target, log, None, indptr, 0, r)
        outs.append((o, r))
    m.close()
    return outs


@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("unsorted_rows", [0, 3])
def test_qc_sweep_matches_oracle(integral, unsorted_rows):
    n = 3000
    indptr, idx, val = make(n, 1, integral, unsorted_rows, beyond=1)
    cm, gm, nr, nv = maps(n, 2)
    got, ref = qc_both(indptr, idx, val, cm, gm, nr, nv)
    for a, b in zip(got, ref):
        if a.dtype == np.float64 and not integral:
            np.testing.assert_allclose(a, b, rtol=1e-13)
        else:
            assert np.array_equal(a, b)


def test_qc_sweep_equals_streamed_matrix():
    n = 2500
    indptr, idx, val = make(n, 3)
    cm, gm, nr, nv = maps(n, 4)
    a, _ = qc_both(indptr, idx, val, cm, gm, nr, nv, "device")
    b, _ = qc_both(indptr, idx, val, cm, gm, nr, nv, "host")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("unsorted_rows", [0, 3])
@pytest.mark.parametrize("target,log", [(1e4, True), (0.0, True), (1e4, False)])
@pytest.mark.parametrize("gene_major", ["1", "0"])
def test_gene_stats_sweep_matches_oracle(unsorted_rows, target, log, gene_major, monkeypatch):
    """gene_stats from the gene-major copy (default) and from the gene-range
    sweep / entry-parallel kernels (CREST_GENE_MAJOR=0)."""
    monkeypatch.setenv("CREST_GENE_MAJOR", gene_major)
    n = 3000
    indptr, idx, val = make(n, 5, True, unsorted_rows, beyond=1)
    cm, gm, nr, nv = maps(n, 6)
    (o, r), = stats_both(indptr, idx, val, cm, gm, nv, target, log)
    assert np.array_equal(o[:, 4], r[:, 4])
    np.testing.assert_allclose(o[:, :4], r[:, :4], rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("gene_major", ["1", "0"])
def test_gene_stats_sweep_follows_gene_map_changes(gene_major, monkeypatch):
    monkeypatch.setenv("CREST_GENE_MAJOR", gene_major)
    n = 2000
    indptr, idx, val = make(n, 7, False)
    cm, gm, nr, nv = maps(n, 8)
    gm2 = gm.copy()
    gm2[gm2 % 3 == 0] = -1  # fewer kept genes: different per-cell totals
    gm2[gm2 >= 0] = np.arange((gm2 >= 0).sum(), dtype=np.int32)
    for o, r in stats_both(indptr, idx, val, cm, gm, nv, gm2=gm2):
        assert np.array_equal(o[:, 4], r[:, 4])
        np.testing.assert_allclose(o[:, :4], r[:, :4], rtol=1e-12, atol=1e-300)
