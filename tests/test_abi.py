"""C ABI checks that need no GPU: the library loads, exports every function
include/crest_gpu.h declares, validates arguments like src/py.rs, and fails
loudly (no CPU fallback) when no CUDA device is usable."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from crest_b200 import _lib, _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(crest_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.exported_symbols())


def test_version_and_device_count_need_no_gpu():
    lib = _lib.load()
    assert lib.crest_version() == 1
    assert lib.crest_device_count() >= 0


def _ctx(n_cells=3, nnz=4):
    genes = np.array([0, 1, 0, 2], np.uint32)[:nnz]
    values = np.ones(nnz, np.float32)
    cm = np.arange(n_cells, dtype=np.int64)
    gm = np.arange(3, dtype=np.int32)
    indptr = np.array([0, 2, 3, 4], np.int64)
    return genes, values, cm, gm, 0.0, False, None, indptr, 0


def test_native_validation_matches_reference_messages():
    g, v, cm, gm, t, l, c, p, f = _ctx()
    out = np.zeros((3, 5))
    with pytest.raises(ValueError, match="exactly one of cells / indptr"):
        _native.gene_stats(g, v, cm, gm, t, l, None, None, f, out)
    with pytest.raises(ValueError, match="non-decreasing and span the chunk"):
        _native.gene_stats(g, v, cm, gm, t, l, None, np.array([0, 3, 2, 4], np.int64), f, out)
    with pytest.raises(ValueError, match="sorted by cell"):
        _native.gene_stats(g, v, cm, gm, t, l, np.array([2, 1, 0, 0], np.uint32), None, f, out)
    with pytest.raises(ValueError, match=r"out must be \(n_vars, 5\)"):
        _native.gene_stats(g, v, cm, gm, t, l, c, p, f, np.zeros((2, 5)))
    with pytest.raises(ValueError, match="C-contiguous"):
        _native.gene_stats(g, v, cm, gm, t, l, c, p, f, np.zeros((3, 10))[:, ::2])
    with pytest.raises(TypeError):
        _native.gene_stats(g.astype(np.int64), v, cm, gm, t, l, c, p, f, out)
    with pytest.raises(ValueError, match="sub_map"):
        _native.gram_accumulate(g, v, cm, gm, t, l, c, p, f, np.array([0, 1, 5], np.int32), np.zeros((2, 2)),
                                np.zeros(2), False, None, None, 0.0)
    with pytest.raises(ValueError, match="needs mean and std"):
        _native.gram_accumulate(g, v, cm, gm, t, l, c, p, f, np.array([0, 1, -1], np.int32), np.zeros((2, 2)),
                                np.zeros(2), True, None, None, 10.0)
    with pytest.raises(RuntimeError, match="at least 2 cells"):
        _native.pca_from_gram(np.zeros((2, 2)), np.zeros(2), 1, 1)


@pytest.mark.skipif(_lib.device_count() > 0, reason="checks the no-GPU behaviour")
def test_compute_without_gpu_fails_loudly():
    out = np.zeros((3, 5))
    with pytest.raises(_lib.CrestError, match="no usable CUDA device"):
        _native.gene_stats(*_ctx(), out)
    assert not out.any()
