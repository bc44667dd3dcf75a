"""Out-of-core Parquet store (crest/core.py:108-135, 368-421): writing the
kept cells / genes as whole-cell parts and reading them back gives the same
raw triplets, parts end on cell boundaries, obs / var survive."""

import numpy as np
import pandas as pd

import crest_b200 as cb
from crest_b200 import synth
from oracle import synth as osynth


def frame():
    p = synth.make_params(700, 400, 4, 0.5, 60.0, seed=8)
    ip, ix, d = osynth.generate(p)
    bf = cb.BioFrame.from_csr(ip, ix, d, 400, var=pd.DataFrame({"gene_name": [f"G{i}" for i in range(400)]}))
    bf.obs["label"] = [f"c{x}" for x in p.labels]
    return bf._subset(obs_mask=np.arange(700) % 4 != 1, var_mask=np.arange(400) % 7 != 3)


def test_write_read_roundtrip(tmp_path):
    bf = frame()
    bf.write_parquet(tmp_path, nnz_per_part=2500)
    rb = cb.read_parquet(tmp_path, chunk_nnz=123)
    assert isinstance(rb.store, cb.ParquetStore)
    assert rb.shape == bf.shape
    assert list(rb.obs["label"]) == list(bf.obs["label"])
    assert list(rb.var["gene_name"]) == list(bf.var["gene_name"])
    src = [np.concatenate(x) for x in zip(*bf.raw_triplets())]
    parts = list(rb.store.chunks())
    assert len(parts) == len(rb.store.parts) > 2
    got = [np.concatenate([p[i] for p in parts]) for i in (2, 0, 1)]  # (cells, genes, counts)
    for a, b in zip(src, got):
        assert np.array_equal(a, b)
    ends = [p[2][-1] for p in parts[:-1]]
    starts = [p[2][0] for p in parts[1:]]
    assert all(e < s for e, s in zip(ends, starts))  # whole cells per part
    assert rb.store.nnz == len(got[0])
    # the reopened frame's own triplets are the identity map of the stored ones
    again = [np.concatenate(x) for x in zip(*rb.raw_triplets())]
    for a, b in zip(src, again):
        assert np.array_equal(a, b)
