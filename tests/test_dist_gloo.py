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
