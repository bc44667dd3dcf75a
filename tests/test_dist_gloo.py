"""The cell-sharded (N > 1) path on CPU: two gloo ranks each hold half of the
cells, compute their per-cell partial sums with the oracle, and combine them
through crest_b200.dist (the same sums the GPU path makes: per-gene QC sums,
per-gene statistics and cell count, then the FP64 Gram / colsum / count).
The HVG set, scale parameters, Gram and PCA must equal those of one process
over all cells."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle

N_CELLS, N_GENES, N_TOP, K = 1600, 500, 120, 10


def data():
    from crest_b200 import synth
    p = synth.make_params(N_CELLS, N_GENES, 5, 0.5, 120.0, seed=11)
    from oracle import synth as osynth
    return osynth.generate(p)


def run_path(indptr, indices, values, reduce_host, reduce_count):
    """QC gene filter -> normalise/log1p -> HVG -> scale -> Gram -> PCA on the given cells."""
    from crest_b200 import pp
    n = len(indptr) - 1
    cm = np.arange(n, dtype=np.int64)
    gm_all = np.arange(N_GENES, dtype=np.int32)
    flag = np.zeros(N_GENES, bool)
    qc = [np.zeros(n), np.zeros(n, np.uint32), np.zeros(n), np.zeros(N_GENES, np.uint32), np.zeros(N_GENES)]
    oracle.qc(indices, values, cm, gm_all, 0.0, False, None, indptr, 0, flag, *qc)
    gene_ncells = reduce_host(qc[3])
    keep_g = gene_ncells >= 3
    gm = np.full(N_GENES, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    nv = int(keep_g.sum())
    st = np.zeros((nv, 5))
    oracle.gene_stats(indices, values, cm, gm, 1e4, True, None, indptr, 0, st)
    st = reduce_host(st)
    n_tot = reduce_count(n)
    cols = pp.hvg_from_stats(st, n_tot, n_top_genes=N_TOP)
    hv = cols["highly_variable"]
    d = int(hv.sum())
    sub = np.full(nv, -1, np.int32)
    sub[hv] = np.arange(d, dtype=np.int32)
    mean = np.ascontiguousarray(cols["mean_log"][hv])
    std = np.ascontiguousarray(cols["std_log"][hv])
    G, cs = np.zeros((d, d)), np.zeros(d)
    oracle.gram_accumulate(indices, values, cm, gm, 1e4, True, None, indptr, 0, sub, G, cs, True, mean, std, 10.0)
    G, cs = reduce_host(G), reduce_host(cs)
    vals, vecs, total = oracle.pca_from_gram(G, cs, n_tot, K)
    return dict(keep_g=keep_g, hv=hv, disp=cols["dispersions_norm"], mean=mean, std=std, G=G, cs=cs, vals=vals,
                vecs=vecs, n=n_tot)


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from crest_b200 import dist as cdist
        cdist.enable()
        assert cdist.active()
        indptr, indices, values = data()
        lo, hi = rank * N_CELLS // world, (rank + 1) * N_CELLS // world
        p = indptr[lo:hi + 1] - indptr[lo]
        g = np.ascontiguousarray(indices[indptr[lo]:indptr[hi]])
        v = np.ascontiguousarray(values[indptr[lo]:indptr[hi]])
        res = run_path(np.ascontiguousarray(p, np.int64), g, v, cdist.sum_host, cdist.sum_count)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), **res)
        cdist.disable()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_process(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    indptr, indices, values = data()
    ref = run_path(np.asarray(indptr, np.int64), indices, values, lambda a: a, int)
    for r in range(world):
        got = dict(np.load(tmp_path / f"rank{r}.npz"))
        assert int(got["n"]) == N_CELLS
        assert np.array_equal(got["keep_g"], ref["keep_g"])
        assert np.array_equal(got["hv"], ref["hv"])
        ok = ~np.isnan(ref["disp"])
        np.testing.assert_allclose(got["disp"][ok], ref["disp"][ok], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(got["mean"], ref["mean"], rtol=1e-12)
        np.testing.assert_allclose(got["G"], ref["G"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(got["cs"], ref["cs"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(got["vals"], ref["vals"], rtol=1e-10)
        cos = np.abs((got["vecs"] * ref["vecs"]).sum(0))
        assert np.all(cos > 1 - 1e-8)


def test_sums_are_the_identity_without_enable():
    from crest_b200 import dist as cdist
    cdist.disable()
    a = np.arange(5, dtype=np.uint32)
    assert cdist.sum_host(a) is a
    assert cdist.sum_count(7) == 7
    assert not cdist.active()


# ----------------------------------------------------------------------------
# The same through crest_b200.pp / crest_b200.tl themselves: each rank builds
# a triplet-store BioFrame over its half of the cells (triplet stores take the
# per-chunk native path), with the oracle standing in for the native module,
# so the sums at the call sites of pp (QC gene sums, gene statistics, cell
# count) and tl (scale parameters, Gram / colsum, cell count) are the ones
# exercised.  Not run on GPUs here: one GPU per call on this build's machines.
class _OracleNative:
    """The oracle behind the names pp / tl call on crest_b200._native."""

    qc = staticmethod(oracle.qc)
    gene_stats = staticmethod(oracle.gene_stats)
    project = staticmethod(oracle.project)
    pca_from_gram = staticmethod(oracle.pca_from_gram)

    @staticmethod
    def gram_accumulate(*args, precision="fp64"):
        assert precision == "fp64"
        return oracle.gram_accumulate(*args)


def pp_tl_path(indptr, indices, values, lo, hi):
    import pandas as pd
    import crest_b200 as cb
    n = hi - lo
    cells = np.repeat(np.arange(n, dtype=np.uint32), np.diff(indptr[lo:hi + 1]))
    g = indices[indptr[lo]:indptr[hi]]
    v = values[indptr[lo]:indptr[hi]]
    names = [f"MT-{i}" if i < 5 else f"G{i}" for i in range(N_GENES)]
    bf = cb.BioFrame.from_triplets(cells, g, v, n, N_GENES, var=pd.DataFrame({"gene_name": names}))
    bf.chunk_nnz = 5000
    bf = cb.pp.filter_cells(bf, min_genes=20)
    bf = cb.pp.filter_genes(bf, min_cells=3)
    cb.pp.normalize_total(bf, 1e4)
    cb.pp.log1p(bf)
    cb.pp.highly_variable_genes(bf, n_top_genes=N_TOP)
    cb.pp.scale(bf, max_value=10)
    cb.tl.pca(bf, n_comps=K, gram_precision="fp64")
    return dict(cells=bf.obs["cell_id"].to_numpy() + lo, genes=bf.var["gene_id"].to_numpy(),
                hv=bf.var["highly_variable"].to_numpy(), disp=bf.var["dispersions_norm"].to_numpy(),
                mean_log=bf.var["mean_log"].to_numpy(), X=bf.obsm["X_pca"], variance=bf.uns["pca"]["variance"],
                loadings=bf.uns["pca"]["projection"]["loadings"])


def _rank_pp(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from crest_b200 import dist as cdist, pp, tl
        pp._native = tl._native = _OracleNative
        cdist.enable()
        indptr, indices, values = data()
        lo, hi = rank * N_CELLS // world, (rank + 1) * N_CELLS // world
        np.savez(os.path.join(out_dir, f"pp{rank}.npz"), **pp_tl_path(indptr, indices, values, lo, hi))
        cdist.disable()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_through_pp_and_tl(tmp_path, monkeypatch):
    world = 2
    mp.start_processes(_rank_pp, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    from crest_b200 import pp, tl
    monkeypatch.setattr(pp, "_native", _OracleNative)
    monkeypatch.setattr(tl, "_native", _OracleNative)
    indptr, indices, values = data()
    ref = pp_tl_path(indptr, indices, values, 0, N_CELLS)
    got = [dict(np.load(tmp_path / f"pp{r}.npz")) for r in range(world)]
    assert np.array_equal(np.concatenate([x["cells"] for x in got]), ref["cells"])
    for x in got:
        assert np.array_equal(x["genes"], ref["genes"])
        assert np.array_equal(x["hv"], ref["hv"])
        ok = ~np.isnan(ref["disp"])
        np.testing.assert_allclose(x["disp"][ok], ref["disp"][ok], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(x["mean_log"], ref["mean_log"], rtol=1e-12)
        np.testing.assert_allclose(x["variance"], ref["variance"], rtol=1e-10)
        cos = np.abs((x["loadings"] * ref["loadings"]).sum(0))
        assert np.all(cos > 1 - 1e-8)
    # the ranks' scores stacked are the one-process scores (up to sign per component)
    X = np.concatenate([x["X"] for x in got]).astype(np.float64)
    R = ref["X"].astype(np.float64)
    s = np.sign((X * R).sum(0))
    np.testing.assert_allclose(X * s, R, rtol=1e-4, atol=1e-4 * np.abs(R).max())
