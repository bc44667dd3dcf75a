"""CPU ORACLE -- test infrastructure only.

Host-thread generator of the seeded synthetic workloads: the same matrix as
``crest_b200.synth.generate`` (GPU), from the same per-draw definition
(``crest_b200/csrc/synth_core.h``), built into ``liboracle.so`` so that tests
and the CPU baseline never load the product library for their inputs.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import lib


class _Params(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_genes", C.c_int64), ("n_clusters", C.c_int32),
                ("dispersion", C.c_double), ("seed", C.c_uint64), ("prob", C.c_void_p), ("labels", C.c_void_p),
                ("lib", C.c_void_p)]


def generate(p, threads: int = 0, pinned_alloc=None):
    """Counts of ``crest_b200.synth.Params`` p as (indptr i64, indices u32, data f32), gene-sorted rows."""
    n = len(p.labels)
    prob = np.ascontiguousarray(p.prob, dtype=np.float64)
    labels = np.ascontiguousarray(p.labels, dtype=np.int32)
    libs = np.ascontiguousarray(p.lib, dtype=np.float64)
    s = _Params(n, prob.shape[1], prob.shape[0], float(p.dispersion), int(p.seed), prob.ctypes.data,
                labels.ctypes.data, libs.ctypes.data)
    threads = threads or os.cpu_count() or 1
    rn = np.zeros(n, np.int64)
    L = lib()
    if L.oc_synth(C.byref(s), rn.ctypes.data, None, None, None, threads) != 0:
        raise ValueError("bad synthetic-count parameters")
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(rn, out=indptr[1:])
    nnz = int(indptr[-1])
    if pinned_alloc is not None:
        indices, data = pinned_alloc(nnz, np.uint32), pinned_alloc(nnz, np.float32)
    else:
        indices, data = np.empty(nnz, np.uint32), np.empty(nnz, np.float32)
    if L.oc_synth(C.byref(s), None, indptr.ctypes.data, indices.ctypes.data, data.ctypes.data, threads) != 0:
        raise ValueError("bad synthetic-count parameters")
    return indptr, indices, data


def make_workload(w, n_cells: int = None, **kw):
    """CSR arrays of a ``crest_b200.synth.Workload`` (optionally only its first n_cells cells)."""
    from crest_b200 import synth
    return generate(synth.workload_params(w, n_cells), **kw)
