"""GPU parity of the device-resident scale + PCA pass (one CSR read into the
compact HVG form, Gram tiles and projection from it) against the oracle and
against the streamed path that reads the CSR itself; duplicate (cell, gene)
entries rejected instead of silently changing the Gram."""

import numpy as np
import pytest

import oracle
from crest_b200 import _lib, _native, tl
from crest_b200.core import DeviceMatrix

pytestmark = pytest.mark.gpu


def setup(small_counts, seed, d_frac=0.4):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    rng = np.random.default_rng(seed)
    keep_c = rng.random(n) >= 0.1
    keep_g = rng.random(n_genes) >= 0.2
    cm = np.full(n, -1, np.int64)
    cm[keep_c] = np.arange(keep_c.sum())
    gm = np.full(n_genes, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    nv = int(keep_g.sum())
    mask = rng.random(nv) < d_frac
    d = int(mask.sum())
    sub = np.full(nv, -1, np.int32)
    sub[mask] = np.arange(d, dtype=np.int32)
    st = np.zeros((nv, 5))
    oracle.gene_stats(indices, data, cm, gm, 1e4, True, None, indptr, 0, st)
    nk = int(keep_c.sum())
    mean = st[:, 0] / nk
    var = np.maximum((st[:, 1] - nk * mean * mean) / (nk - 1), 0)
    std = np.sqrt(var)
    std[std == 0] = 1
    return dict(indptr=indptr, indices=indices, data=data, n_genes=n_genes, cm=cm, gm=gm, nv=nv, d=d, sub=sub,
                mean=np.ascontiguousarray(mean[mask]), std=np.ascontiguousarray(std[mask]), nr=nk)


def plan_gram(s, residency, precision="fp64", indices=None, data=None):
    dm = DeviceMatrix(s["indptr"], s["indices"] if indices is None else indices,
                      s["data"] if data is None else data, s["n_genes"], residency, chunk_cells=400)
    scale = _lib.Scale(1, _lib.ptr(s["mean"]), _lib.ptr(s["std"]), 10.0)
    p = tl.PcaPlan(s["d"], precision)
    p.accumulate(dm, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale)
    return p, dm, scale


@pytest.mark.parametrize("residency", ["device", "host"])
def test_plan_fp64_gram_bit_exact(small_counts, residency):
    s = setup(small_counts, 3)
    p, dm, _ = plan_gram(s, residency)
    G = p.gram()
    colsum = p.results()[3]
    Go, co = np.zeros((s["d"], s["d"])), np.zeros(s["d"])
    oracle.gram_accumulate(s["indices"], s["data"], s["cm"], s["gm"], 1e4, True, None, s["indptr"], 0, s["sub"],
                           Go, co, True, s["mean"], s["std"], 10.0)
    iu = np.triu_indices(s["d"])
    assert np.array_equal(G[iu], Go[iu])
    assert np.array_equal(colsum, co)
    p.close()
    dm.close()


@pytest.mark.parametrize("k", [20, 50, 51, 100])
def test_compact_projection_equals_csr_projection(small_counts, k):
    """The same plan (same loadings) projects a device-resident matrix from the
    compact form and a streamed one from the CSR: identical scores."""
    s = setup(small_counts, 4)
    p, dm, scale = plan_gram(s, "device")
    p.solve(s["nr"], k)
    Xa = p.project(dm, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale, s["nr"])
    dh = DeviceMatrix(s["indptr"], s["indices"], s["data"], s["n_genes"], "host", chunk_cells=300)
    Xb = p.project(dh, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale, s["nr"])  # CSR streamed again
    assert np.array_equal(Xa, Xb)
    # a streamed matrix whose Gram pass packed its compact form projects from it: the same scores
    p2, dh2, _ = plan_gram(s, "host")
    p2.solve(s["nr"], k)
    assert np.array_equal(p2.results()[1], p.results()[1])
    Xc = p2.project(dh2, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale, s["nr"])
    assert np.array_equal(Xa, Xc)
    p2.close()
    dh2.close()
    # and the oracle's projection with the plan's loadings adds the same per-cell sums
    L = p.results()[1]
    Xo = np.zeros((s["nr"], k), np.float32)
    oracle.project(s["indices"], s["data"], s["cm"], s["gm"], 1e4, True, None, s["indptr"], 0, s["sub"], L, Xo,
                   True, s["mean"], s["std"], 10.0)
    Xz = np.zeros((s["nr"], k), np.float32)
    _native.project(s["indices"], s["data"], s["cm"], s["gm"], 1e4, True, None, s["indptr"], 0, s["sub"], L, Xz,
                    True, s["mean"], s["std"], 10.0)
    assert np.array_equal(Xz, Xo)
    for x in (p, dm, dh):
        x.close()


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_many_tiles_during_and_after_the_upload(small_counts, monkeypatch, precision):
    """256-cell Gram tiles: the first pass tiles the cells as their upload
    chunk arrives, a later pass tiles the resident matrix as one range; both
    give the same Gram, and the FP64 form the oracle's bit for bit."""
    monkeypatch.setenv("CREST_TILE_CELLS", "256")
    s = setup(small_counts, 15)
    p, dm, scale = plan_gram(s, "device", precision)
    G1, c1 = p.gram().copy(), p.results()[3].copy()
    p.reset()
    p.accumulate(dm, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale)
    G2, c2 = p.gram(), p.results()[3]
    iu = np.triu_indices(s["d"])
    assert np.array_equal(G1[iu], G2[iu]) and np.array_equal(c1, c2)
    if precision == "fp64":
        Go, co = oracle_gram(s)
        assert np.array_equal(G2[iu], Go[iu]) and np.array_equal(c2, co)
    p.close()
    dm.close()


def oracle_gram(s, indices=None, data=None, indptr=None):
    Go, co = np.zeros((s["d"], s["d"])), np.zeros(s["d"])
    oracle.gram_accumulate(s["indices"] if indices is None else indices, s["data"] if data is None else data,
                           s["cm"], s["gm"], 1e4, True, None, s["indptr"] if indptr is None else indptr, 0, s["sub"],
                           Go, co, True, s["mean"], s["std"], 10.0)
    return Go, co


def build_range_index(s, dm, all_mapped=False):
    """A QC pass over a device matrix builds its gene-range index, which also
    records whether every row is strictly sorted by gene.  With every cell
    and gene mapped it also learns whether all stored values are small
    non-negative integers (the extract then skips its per-entry test)."""
    if all_mapped:
        n, g = len(s["indptr"]) - 1, s["n_genes"]
        cm, gm, nr, nv = np.arange(n, dtype=np.int64), np.arange(g, dtype=np.int32), n, g
    else:
        cm, gm, nr, nv = s["cm"], s["gm"], s["nr"], s["nv"]
    flag = np.zeros(nv, np.bool_)
    out = [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
    _lib.call("crest_matrix_qc", dm.handle, _lib.ptr(cm), _lib.ptr(gm), _lib.ptr(flag), nr, nv,
              *[_lib.ptr(a) for a in out])


@pytest.mark.parametrize("indexed", [False, True, "all"])
@pytest.mark.parametrize("integral", [True, False])
def test_extract_with_and_without_order_check(small_counts, indexed, integral):
    """Strictly gene-sorted rows (known once the range index exists) skip the
    column-order check, and a QC over every cell and gene that met only small
    integers lets the extract skip its per-entry integrality test; in every
    case, and for non-integral values (the entry-order normalisation total),
    the FP64 Gram equals the oracle's."""
    s = setup(small_counts, 12)
    data = s["data"] if integral else (s["data"] * np.float32(0.37)).astype(np.float32)
    s = dict(s, data=data)
    dm = DeviceMatrix(s["indptr"], s["indices"], data, s["n_genes"], "device", chunk_cells=400)
    if indexed:
        build_range_index(s, dm, all_mapped=indexed == "all")
    scale = _lib.Scale(1, _lib.ptr(s["mean"]), _lib.ptr(s["std"]), 10.0)
    p = tl.PcaPlan(s["d"], "fp64")
    p.accumulate(dm, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale)
    Go, co = oracle_gram(s)
    iu = np.triu_indices(s["d"])
    assert np.array_equal(p.gram()[iu], Go[iu])
    assert np.array_equal(p.results()[3], co)
    p.close()
    dm.close()


def test_duplicates_rejected_after_range_index(small_counts):
    """A row holding a gene twice is sorted but not strictly: the range index
    keeps the order check on and the duplicate is still rejected."""
    s = setup(small_counts, 6)  # a seed that keeps cell 7, which holds the duplicate
    ip2, ix2, dx2 = with_duplicate(s)
    s2 = dict(s, indptr=ip2, indices=ix2, data=dx2)
    dm = DeviceMatrix(ip2, ix2, dx2, s["n_genes"], "device", chunk_cells=400)
    build_range_index(s2, dm)
    scale = _lib.Scale(1, _lib.ptr(s["mean"]), _lib.ptr(s["std"]), 10.0)
    p = tl.PcaPlan(s["d"], "fp64")
    with pytest.raises(ValueError, match="twice"):
        p.accumulate(dm, s["cm"], s["gm"], 1e4, True, s["sub"], s["nv"], scale)
    p.close()
    dm.close()


def test_extract_wide_gene_table(small_counts):
    """70,000 store genes: the int16 code table no longer leaves room for two
    blocks per SM and the byte-class extract runs; the same FP64 Gram."""
    indptr, indices, data = small_counts[:3]
    s = setup((indptr, indices, data, 70_000), 14, d_frac=0.0)
    # HVG columns among the stored genes (ids below 600)
    rng = np.random.default_rng(14)
    stored = np.flatnonzero(s["gm"][:600] >= 0)
    pick = np.sort(rng.choice(stored, 150, replace=False))
    sub = np.full(s["nv"], -1, np.int32)
    sub[s["gm"][pick]] = np.arange(150, dtype=np.int32)
    st = np.zeros((s["nv"], 5))
    oracle.gene_stats(indices, data, s["cm"], s["gm"], 1e4, True, None, indptr, 0, st)
    nk = s["nr"]
    mean = st[:, 0] / nk
    std = np.sqrt(np.maximum((st[:, 1] - nk * mean * mean) / (nk - 1), 0))
    std[std == 0] = 1
    mask = sub >= 0
    s.update(d=150, sub=sub, mean=np.ascontiguousarray(mean[mask]), std=np.ascontiguousarray(std[mask]))
    p, dm, _ = plan_gram(s, "device")
    Go, co = oracle_gram(s)
    iu = np.triu_indices(150)
    assert np.array_equal(p.gram()[iu], Go[iu])
    assert np.array_equal(p.results()[3], co)
    p.close()
    dm.close()


def shuffled_rows(s, seed):
    """The same matrix with every row's entries in a random order."""
    rng = np.random.default_rng(seed)
    ix, dx = s["indices"].copy(), s["data"].copy()
    ip = s["indptr"]
    for i in range(len(ip) - 1):
        a, b = ip[i], ip[i + 1]
        perm = a + rng.permutation(b - a)
        ix[a:b], dx[a:b] = s["indices"][perm], s["data"][perm]
    return ix, dx


@pytest.mark.parametrize("residency", ["device", "host"])
def test_unsorted_rows_without_duplicates_are_accepted(small_counts, residency):
    s = setup(small_counts, 5)
    ix, dx = shuffled_rows(s, 1)
    p0, d0, _ = plan_gram(s, residency)
    p1, d1, _ = plan_gram(s, residency, indices=ix, data=dx)
    iu = np.triu_indices(s["d"])
    # the FP64 Gram sums products in cell order: row order inside a cell only
    # changes which column a product lands in, not the order of the sums
    assert np.array_equal(p0.gram()[iu], p1.gram()[iu])
    for x in (p0, d0, p1, d1):
        x.close()


def with_duplicate(s, sorted_rows=True):
    """Cell 7's first HVG entry stored twice (one more entry in its row)."""
    ip, ix, dx = s["indptr"], s["indices"], s["data"]
    hv_store = np.where(s["gm"] >= 0)[0]
    hv_store = hv_store[s["sub"][s["gm"][hv_store]] >= 0]
    row = ix[ip[7]:ip[8]]
    j = int(ip[7] + np.where(np.isin(row, hv_store))[0][0])
    pos = j + 1 if sorted_rows else int(ip[8])  # next to the original, or at the row's end
    ix2 = np.insert(ix, pos, ix[j])
    dx2 = np.insert(dx, pos, dx[j])
    ip2 = ip.copy()
    ip2[8:] += 1
    return ip2, ix2.astype(np.uint32), dx2.astype(np.float32)


@pytest.mark.parametrize("residency", ["device", "host"])
@pytest.mark.parametrize("sorted_rows", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_duplicate_entries_are_rejected(small_counts, residency, sorted_rows, precision):
    s = setup(small_counts, 6)
    ip2, ix2, dx2 = with_duplicate(s, sorted_rows)
    s2 = dict(s, indptr=ip2, indices=ix2, data=dx2)
    with pytest.raises(ValueError, match="twice"):
        plan_gram(s2, residency, precision)


def test_duplicate_entries_rejected_per_chunk(small_counts):
    s = setup(small_counts, 7)
    ip2, ix2, dx2 = with_duplicate(s)
    G, cs = np.full((s["d"], s["d"]), 0.5), np.full(s["d"], 0.5)
    with pytest.raises(ValueError, match="twice"):
        _native.gram_accumulate(ix2, dx2, s["cm"], s["gm"], 1e4, True, None, ip2, 0, s["sub"], G, cs, True,
                                s["mean"], s["std"], 10.0, precision="fp32")
    # the caller's accumulators are left as they were
    assert np.all(G == 0.5) and np.all(cs == 0.5)


@pytest.mark.parametrize("pair", ["1", "0"])
def test_bf16x3_gram_both_syrk_forms(pbmc_counts, monkeypatch, pair):
    """The CTA-pair tensor-core SYRK (256 x 256 blocks, two cell halves) and the
    one-CTA form (128 x 128 blocks) against the FP64 Gram of the same plan API,
    d = 2000 HVG columns (36 pair blocks): centred covariances within 5e-6."""
    monkeypatch.setenv("CREST_TC_PAIR", pair)
    indptr, indices, data, n_genes = pbmc_counts[:4]
    s = setup((indptr, indices, data, n_genes), 9, d_frac=0.0)
    rng = np.random.default_rng(9)
    mask = np.zeros(s["nv"], bool)
    mask[rng.choice(s["nv"], 2000, replace=False)] = True
    sub = np.full(s["nv"], -1, np.int32)
    sub[mask] = np.arange(2000, dtype=np.int32)
    st = np.zeros((s["nv"], 5))
    oracle.gene_stats(indices, data, s["cm"], s["gm"], 1e4, True, None, indptr, 0, st)
    nk = s["nr"]
    mean = st[:, 0] / nk
    std = np.sqrt(np.maximum((st[:, 1] - nk * mean * mean) / (nk - 1), 0))
    std[std == 0] = 1
    s.update(d=2000, sub=sub, mean=np.ascontiguousarray(mean[mask]), std=np.ascontiguousarray(std[mask]))
    cov = []
    for prec in ("fp64", "bf16x3"):
        p, dm, _ = plan_gram(s, "device", prec)
        G, c = p.gram(), p.results()[3]
        S = np.triu(G) + np.triu(G, 1).T
        cov.append((S - np.outer(c, c) / nk) / (nk - 1))
        p.close()
        dm.close()
    err = np.linalg.norm(cov[1] - cov[0]) / np.linalg.norm(cov[0])
    assert err < 5e-6, err
