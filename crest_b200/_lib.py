"""ctypes binding of ``libcrest_gpu.so`` (the C ABI in include/crest_gpu.h).

The library is built in-tree by :mod:`crest_b200.build`.  There is no CPU
fallback: if the library cannot be loaded, or no CUDA device is usable, every
compute call raises.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrest_gpu.so")

OK, ERUNTIME, ECUDA, ENOMEM, ENODEV, EINVAL, ETIMEOUT = 0, -1, -5, -12, -19, -22, -110
GRAM_PRECISION = {"fp64": 0, "fp32": 1, "bf16x3": 2}
MEM_HOST, MEM_DEVICE = 0, 1

P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32
D = C.c_double


class Chunk(C.Structure):
    """struct crest_chunk: one chunk in the reference's chunk protocol."""
    _fields_ = [
        ("genes", P), ("values", P), ("nnz", I64),
        ("cell_map", P), ("n_cell_map", I64),
        ("gene_map", P), ("n_gene_map", I64),
        ("target_sum", D), ("log1p", I32),
        ("cells", P), ("indptr", P), ("n_indptr", I64),
        ("first_cell", C.c_uint32),
    ]


class Scale(C.Structure):
    """struct crest_scale."""
    _fields_ = [("scale", I32), ("mean", P), ("std", P), ("max_value", D)]


class PcaStats(C.Structure):
    _fields_ = [("gram_ms", D), ("solve_ms", D), ("project_ms", D), ("eig_iters", I32),
                ("eig_converged", I32), ("eig_residual", D)]


class Synth(C.Structure):
    _fields_ = [("n_cells", I64), ("n_genes", I64), ("n_clusters", I32), ("dispersion", D),
                ("seed", C.c_uint64), ("prob", P), ("labels", P), ("lib", P)]


# name -> argtypes (all return int)
_SIGS = {
    "crest_version": [],
    "crest_device_count": [],
    "crest_memory_stats": [C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int32],
    "crest_set_device": [C.c_int],
    "crest_qc": [P, P, I64, P, P, P, I64, P, P],
    "crest_qc_static": [P, P, I64, P, P, P, I64, P, P],
    "crest_gene_stats": [P, I64, P],
    "crest_group_gene_sums": [P, P, I64, I64, I64, P, P, P, P],
    "crest_group_gene_totals": [P, P, I64, I64, I64, P],
    "crest_knn_graph": [P, I64, I64, I64, P, P],
    "crest_gram_accumulate": [P, P, I64, P, I64, P, P, I32],
    "crest_pca_from_gram": [P, P, I64, I64, I64, P, P, P, P],
    "crest_project": [P, P, I64, P, I64, I64, P, P, I64],
    "crest_matrix_create": [P, P, P, P, I64, I64, I32, I64],
    "crest_matrix_free": [P],
    "crest_matrix_info": [P, P, P, P],
    "crest_matrix_qc": [P, P, P, P, I64, I64, P, P, P, P, P],
    "crest_matrix_gene_stats": [P, P, P, D, I32, I64, P],
    "crest_matrix_group_gene_sums": [P, P, P, D, I32, P, I64, I64, I64, P, P, P, P],
    "crest_pca_create": [P, I64, I32],
    "crest_pca_free": [P],
    "crest_pca_accumulate": [P, P, P, P, D, I32, P, I64, P],
    "crest_pca_reset": [P],
    "crest_pca_accumulators": [P, P, P],
    "crest_pca_gram": [P, P],
    "crest_pca_solve": [P, I64, I64],
    "crest_pca_results": [P, P, P, P, P],
    "crest_pca_project": [P, P, P, P, D, I32, P, I64, P, I64, P, I32],
    "crest_pca_stats_get": [P, P],
    "crest_fused_forward": [P, P, P, I64, I64, P, P, I64, P, P, D, P],
    "crest_fused_backward": [P, P, P, I64, I64, P, P, I64, P, P, D, P, P, P, P],
    "crest_synth_gpu": [P, P, P, P, P],
    "crest_profile_enable": [C.c_int],
    "crest_profile_count": [],
    "crest_profile_entry": [C.c_int, C.c_char_p, C.c_int, P, P, P],
}

_lib = None
_lock = threading.Lock()


class CrestError(RuntimeError):
    pass


def load():
    """Load the library (building it first when it is missing and nvcc exists)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.crest_last_error.argtypes = []
        L.crest_last_error.restype = C.c_char_p
        _lib = L
        return L


def exported_symbols():
    return list(_SIGS) + ["crest_last_error"]


def check(rc: int):
    if rc == OK:
        return
    msg = (load().crest_last_error() or b"").decode(errors="replace")
    if rc == EINVAL:
        raise ValueError(msg)
    raise CrestError(f"{msg} (status {rc})")


def call(name: str, *args):
    check(getattr(load(), name)(*args))


def profile_enable(on: bool = True):
    load().crest_profile_enable(1 if on else 0)


def profile_table() -> dict:
    """{kernel: (launches, total_ms, max_ms)} of the launches timed since profile_enable."""
    L = load()
    out = {}
    for i in range(L.crest_profile_count()):
        name = C.create_string_buffer(128)
        n, t, m = C.c_longlong(), C.c_double(), C.c_double()
        check(L.crest_profile_entry(i, name, 128, C.byref(n), C.byref(t), C.byref(m)))
        out[name.value.decode()] = (int(n.value), float(t.value), float(m.value))
    return out


def device_count() -> int:
    return int(load().crest_device_count())


def require_gpu():
    if device_count() == 0:
        raise CrestError("no usable CUDA device: the CREST GPU path has no CPU fallback")


def ptr(a):
    if a is None:
        return None
    return a.ctypes.data


def carray(a, dtype, name):
    """The buffer as a C-contiguous array of `dtype`, without copying when possible."""
    a = np.asarray(a)
    if a.dtype != dtype:
        raise TypeError(f"{name} must be {np.dtype(dtype).name}, got {a.dtype}")
    if not a.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")
    return a


def memory_stats(reset_high: bool = False):
    """(bytes in use, high-water mark) of the library's device allocations."""
    u, h = C.c_int64(), C.c_int64()
    call("crest_memory_stats", C.byref(u), C.byref(h), int(bool(reset_high)))
    return u.value, h.value
