"""crest_qc_static (fixed device scratch, no allocation) against crest_qc.

Both entry points are called through the C ABI on the same chunks, twice in
a row: the outputs accumulate (+=) on the host exactly like the reference's
qc, and must agree after each call.  The tolerance is the one of the QC
parity tests: bit-exact for integral counts, 1e-13 relative for per-gene
totals of non-integral values (atomic summation order)."""

import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from crest_b200 import _lib, _native
from crest_b200._lib import ptr

pytestmark = pytest.mark.gpu


def _outputs(nr, nv):
    return [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]


def _call(name, ch, flag, nv, nr, o):
    return getattr(_lib.load(), name)(C.byref(ch), ptr(flag), nv, ptr(o[0]), ptr(o[1]), ptr(o[2]), nr,
                                      ptr(o[3]), ptr(o[4]))


@pytest.mark.parametrize("integral", [True, False])
def test_static_scratch_qc_matches_qc_twice(small_counts, integral):
    indptr, indices, data, n_genes = small_counts[:4]
    rng = np.random.default_rng(11)
    if not integral:
        data = (data * rng.uniform(0.5, 1.5, len(data))).astype(np.float32)
    n = len(indptr) - 1
    keep_c = rng.random(n) >= 0.1
    cm = np.full(n, -1, np.int64)
    cm[keep_c] = np.arange(keep_c.sum())
    keep_g = rng.random(n_genes) >= 0.2
    gm = np.full(n_genes, -1, np.int32)
    gm[keep_g] = np.arange(keep_g.sum(), dtype=np.int32)
    nr, nv = int(keep_c.sum()), int(keep_g.sum())
    flag = np.zeros(nv, bool)
    flag[:9] = True
    a, b = _outputs(nr, nv), _outputs(nr, nv)
    for lo, hi in ((0, 640), (640, n)):  # two calls in a row, accumulating
        p = np.ascontiguousarray(indptr[lo:hi + 1])
        g = np.ascontiguousarray(indices[p[0]:p[-1]])
        v = np.ascontiguousarray(data[p[0]:p[-1]])
        ch, keep, _, _ = _native._chunk(g, v, cm, gm, 0.0, False, None, p, lo)
        assert _call("crest_qc", ch, flag, nv, nr, a) == _lib.OK
        assert _call("crest_qc_static", ch, flag, nv, nr, b) == _lib.OK
        for x, y in zip(a[:4], b[:4]):
            assert np.array_equal(x, y)
        if integral:
            assert np.array_equal(a[4], b[4])
        else:
            np.testing.assert_allclose(a[4], b[4], rtol=1e-13)
    assert a[1].sum() == np.count_nonzero(data[np.isin(np.repeat(np.arange(n), np.diff(indptr)), np.flatnonzero(keep_c))
                                              & (gm[indices] >= 0)])


def test_static_scratch_rejects_oversized_chunks():
    n_cells = (1 << 16) + 1
    indptr = np.zeros(n_cells + 1, np.int64)
    g = np.zeros(0, np.uint32)
    v = np.zeros(0, np.float32)
    cm = np.arange(n_cells, dtype=np.int64)
    gm = np.arange(4, dtype=np.int32)
    ch, keep, nr, nv = _native._chunk(g, v, cm, gm, 0.0, False, None, indptr, 0)
    o = _outputs(nr, nv)
    rc = _call("crest_qc_static", ch, np.zeros(nv, bool), nv, nr, o)
    assert rc == _lib.EINVAL
    assert b"static scratch holds at most" in _lib.load().crest_last_error()


@pytest.mark.parametrize("map_len", [700, 640, 100])
def test_static_scratch_short_cell_map(small_counts, map_len):
    """cell_map shorter than first_cell + n_spans: cells past its end are
    dropped (src/kernels.rs:65-68), including a chunk that starts past it."""
    indptr, indices, data, n_genes = small_counts[:4]
    n = len(indptr) - 1
    cm = np.arange(map_len, dtype=np.int64)
    gm = np.arange(n_genes, dtype=np.int32)
    nr, nv = map_len, n_genes
    flag = np.zeros(nv, bool)
    a, b = _outputs(nr, nv), _outputs(nr, nv)
    for lo, hi in ((0, 640), (640, n)):
        p = np.ascontiguousarray(indptr[lo:hi + 1])
        g = np.ascontiguousarray(indices[p[0]:p[-1]])
        v = np.ascontiguousarray(data[p[0]:p[-1]])
        ch, keep, _, _ = _native._chunk(g, v, cm, gm, 0.0, False, None, p, lo)
        assert _call("crest_qc", ch, flag, nv, nr, a) == _lib.OK
        assert _call("crest_qc_static", ch, flag, nv, nr, b) == _lib.OK
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    row_sums = np.bincount(np.repeat(np.arange(n), np.diff(indptr)), weights=data.astype(np.float64), minlength=n)
    assert np.array_equal(a[0], row_sums[:map_len])


def test_static_scratch_bad_row_leaves_outputs_untouched(small_counts):
    indptr, indices, data, n_genes = small_counts[:4]
    p = np.ascontiguousarray(indptr[:51])
    g = np.ascontiguousarray(indices[:p[-1]])
    v = np.ascontiguousarray(data[:p[-1]])
    cm = np.arange(50, dtype=np.int64)
    gm = np.arange(n_genes, dtype=np.int32)
    ch, keep, _, _ = _native._chunk(g, v, cm, gm, 0.0, False, None, p, 0)
    o = _outputs(40, n_genes)  # rows 40..49 do not fit
    rc = _call("crest_qc_static", ch, np.zeros(n_genes, bool), n_genes, 40, o)
    assert rc == _lib.EINVAL
    assert all(not x.any() for x in o)


def test_static_scratch_allocates_nothing():
    """In a fresh process that never calls crest_qc: after the first call (which
    loads the device code), further calls leave the device's free memory as it is."""
    code = textwrap.dedent("""
        import ctypes as C, sys
        import numpy as np
        import torch
        sys.path.insert(0, %r)
        from crest_b200 import _lib, _native
        torch.cuda.init()
        rng = np.random.default_rng(3)
        n, ng = 900, 700
        counts = rng.poisson(0.3, (n, ng)).astype(np.float32)
        indptr = np.zeros(n + 1, np.int64)
        indptr[1:] = np.cumsum((counts > 0).sum(1))
        genes = np.nonzero(counts)[1].astype(np.uint32)
        vals = counts[counts > 0].astype(np.float32)
        cm = np.arange(n, dtype=np.int64)
        gm = np.arange(ng, dtype=np.int32)
        ch, keep, nr, nv = _native._chunk(genes, vals, cm, gm, 0.0, False, None, indptr, 0)
        out = [np.zeros(nr), np.zeros(nr, np.uint32), np.zeros(nr), np.zeros(nv, np.uint32), np.zeros(nv)]
        flag = np.zeros(nv, bool)
        P = _lib.ptr
        def call():
            rc = _lib.load().crest_qc_static(C.byref(ch), P(flag), nv, P(out[0]), P(out[1]), P(out[2]), nr,
                                             P(out[3]), P(out[4]))
            assert rc == 0, rc
        call()
        torch.cuda.synchronize()
        f0 = torch.cuda.mem_get_info()[0]
        for _ in range(5):
            call()
        torch.cuda.synchronize()
        f1 = torch.cuda.mem_get_info()[0]
        assert f1 == f0, (f0, f1)
        assert np.array_equal(out[0], 6 * counts.sum(1))
        print("ok")
    """) % os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-3000:]
