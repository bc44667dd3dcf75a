"""Failure detection without faulting the GPU.

* A bounded pipeline wait of the tensor-core Gram runs out: a test hook
  (CREST_TC_INJECT_STALL=1) arms the last stage of each launch without
  loading it and shortens the wait limit to 5 ms.  The call must report
  CREST_ETIMEOUT (CrestError), leave the caller's accumulators untouched,
  and the next call on the same context must give the right Gram.
* A device allocation fails (CREST_INJECT_ALLOC_FAIL=N, host side): the call
  reports out-of-memory and the library keeps working afterwards.
"""

import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import oracle
from crest_b200 import _lib, _native

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def gram_case(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cm = np.arange(n, dtype=np.int64)
    gm = np.arange(n_genes, dtype=np.int32)
    rng = np.random.default_rng(12)
    d = 300
    sub = np.full(n_genes, -1, np.int32)
    sub[rng.choice(n_genes, d, replace=False)] = np.arange(d, dtype=np.int32)
    return indptr, indices, data, cm, gm, sub, d


@pytest.mark.parametrize("pair", ["1", "0"])
def test_tensor_core_wait_runs_out(small_counts, monkeypatch, pair):
    indptr, indices, data, cm, gm, sub, d = gram_case(small_counts)
    monkeypatch.setenv("CREST_TC_PAIR", pair)
    monkeypatch.setenv("CREST_TC_INJECT_STALL", "1")
    G, cs = np.full((d, d), 0.25), np.full(d, 0.25)
    with pytest.raises(_lib.CrestError, match="timed out") as ei:
        _native.gram_accumulate(indices, data, cm, gm, 1e4, True, None, indptr, 0, sub, G, cs, False, None, None,
                                0.0, precision="bf16x3")
    assert f"status {_lib.ETIMEOUT}" in str(ei.value)
    assert np.all(G == 0.25) and np.all(cs == 0.25)
    monkeypatch.delenv("CREST_TC_INJECT_STALL")
    G, cs = np.zeros((d, d)), np.zeros(d)
    _native.gram_accumulate(indices, data, cm, gm, 1e4, True, None, indptr, 0, sub, G, cs, False, None, None, 0.0,
                            precision="bf16x3")
    Go, co = np.zeros((d, d)), np.zeros(d)
    oracle.gram_accumulate(indices, data, cm, gm, 1e4, True, None, indptr, 0, sub, Go, co, False, None, None, 0.0)
    iu = np.triu_indices(d)
    assert np.linalg.norm(G[iu] - Go[iu]) / np.linalg.norm(Go[iu]) < 1e-5
    np.testing.assert_allclose(cs, co, rtol=1e-10, atol=1e-9)


def test_injected_allocation_failure():
    """In a fresh process (so no buffer exists yet) the first device allocation
    fails; the call reports out of memory and the next call works."""
    code = textwrap.dedent("""
        import sys
        import numpy as np
        sys.path.insert(0, %r)
        from crest_b200 import _lib, _native
        rng = np.random.default_rng(2)
        n, ng = 400, 300
        counts = rng.poisson(0.4, (n, ng)).astype(np.float32)
        indptr = np.zeros(n + 1, np.int64)
        indptr[1:] = np.cumsum((counts > 0).sum(1))
        genes = np.nonzero(counts)[1].astype(np.uint32)
        vals = counts[counts > 0].astype(np.float32)
        cm = np.arange(n, dtype=np.int64)
        gm = np.arange(ng, dtype=np.int32)
        out = np.zeros((ng, 5))
        try:
            _native.gene_stats(genes, vals, cm, gm, 0.0, False, None, indptr, 0, out)
            print("no failure")
            sys.exit(1)
        except _lib.CrestError as e:
            assert "out of memory (injected)" in str(e), e
            assert "status %d" in str(e), e
        assert not out.any()
        _native.gene_stats(genes, vals, cm, gm, 0.0, False, None, indptr, 0, out)
        assert np.array_equal(out[:, 4], (counts > 0).sum(0))
        print("ok")
    """) % (ROOT, _lib.ENOMEM)
    env = dict(os.environ, CREST_INJECT_ALLOC_FAIL="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr[-3000:]
