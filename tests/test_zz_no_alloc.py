"""crest_qc_static (fixed device scratch, no allocation) against crest_qc.

Both entry points are called through the C ABI on the same chunks, twice in
a row: the outputs accumulate (+=) on the host exactly like the reference's
qc, and must agree after each call.  The tolerance is the one of the QC
parity tests: bit-exact for integral counts, 1e-13 relative for per-gene
totals of non-integral values (atomic summation order)."""

import ctypes as C

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
