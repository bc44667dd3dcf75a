"""CPU ORACLE -- test infrastructure only.

Restates harshameghadri/CREST's CPU path for the preprocessing-to-PCA hot path:

* ``crest_oracle.c`` restates the Rust streaming kernels (src/kernels.rs
  ``qc``, ``gene_stats``, ``gram_accumulate``, ``project``, ``materialize``)
  in the reference's summation order;
* this module exposes them with the exact Python signatures of the
  reference's native module ``crest.crest`` (src/py.rs:213-309, 386-399), so
  the reference's own Python orchestration can run on top of it (see
  tests/golden/make_golden.py), and restates the host-side numpy math of
  crest/pp.py (HVG) and crest/tl.py (PCA) in :mod:`oracle.pipeline`.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product (``crest_b200``) never
does.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_SRC = os.path.join(_HERE, "crest_oracle.c")
_SYNTH_SRC = os.path.join(_HERE, "synth_cpu.c")
# the per-draw definition shared with the product's GPU generator
_SYNTH_HDR = os.path.join(os.path.dirname(_HERE), "crest_b200", "csrc", "synth_core.h")
_lib = None

# rayon::current_num_threads() of the emulated reference run; it only decides
# how cells are grouped into parts, i.e. the order of per-gene f64 sums.
DEFAULT_THREADS = int(os.environ.get("CREST_ORACLE_THREADS", os.cpu_count() or 1))


def build(force: bool = False) -> str:
    """Compile the C restatement into ``oracle/liboracle.so`` (gcc, no FMA contraction)."""
    srcs = [_SRC, _SYNTH_SRC, _SYNTH_HDR]
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs)):
        cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-I",
               os.path.dirname(_SYNTH_HDR), "-o", _LIB_PATH + ".tmp", _SRC, _SYNTH_SRC, "-lm", "-lpthread"]
        subprocess.run(cmd, check=True)
        os.replace(_LIB_PATH + ".tmp", _LIB_PATH)
    return _LIB_PATH


class _Chunk(C.Structure):
    _fields_ = [
        ("genes", C.c_void_p), ("values", C.c_void_p), ("nnz", C.c_int64),
        ("cell_map", C.c_void_p), ("n_cell_map", C.c_int64),
        ("gene_map", C.c_void_p), ("n_gene_map", C.c_int64),
        ("target_sum", C.c_double), ("log1p", C.c_int32),
        ("cells", C.c_void_p), ("indptr", C.c_void_p), ("n_indptr", C.c_int64),
        ("first_cell", C.c_uint32),
    ]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.oc_qc.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_int64]
        L.oc_gene_stats.argtypes = [P, C.c_int, P, C.c_int64]
        L.oc_gram_accumulate.argtypes = [P, C.c_int, P, C.c_int64, C.c_int, P, P, C.c_double, P, P]
        L.oc_project.argtypes = [P, C.c_int, P, C.c_int, P, P, C.c_double, P, C.c_int64, P]
        L.oc_materialize.argtypes = [P, C.c_int, P, P, P, C.c_int64]
        L.oc_materialize.restype = C.c_int64
        L.oc_synth.argtypes = [P, P, P, P, P, C.c_int]
        L.oc_group_gene_sums.argtypes = [P, P, C.c_int64, P, P, P, P]
        L.oc_knn.argtypes = [P, C.c_int64, C.c_int64, C.c_int64, P, P, C.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _c(a, dt, name):
    if not isinstance(a, np.ndarray) or a.dtype != dt:
        raise TypeError(f"{name} must be a numpy {np.dtype(dt).name} array")
    if not a.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous")
    return a


def _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell):
    """Validation of src/py.rs:162-189; returns (chunk struct, keepalive, n_rows)."""
    g = _c(genes, np.uint32, "genes")
    v = _c(values, np.float32, "values")
    if len(g) != len(v):
        raise ValueError("genes, values must have equal length")
    cm = _c(cell_map, np.int64, "cell_map")
    gm = _c(gene_map, np.int32, "gene_map")
    if cells is not None and indptr is None:
        c = _c(cells, np.uint32, "cells")
        if len(c) != len(g):
            raise ValueError("cells, genes must have equal length")
        if len(c) > 1 and np.any(c[1:] < c[:-1]):
            raise ValueError("chunk must be sorted by cell")
        p = None
    elif cells is None and indptr is not None:
        p = _c(indptr, np.int64, "indptr")
        if len(p) == 0 or np.any(p[1:] < p[:-1]) or int(p[-1] - p[0]) != len(g):
            raise ValueError("indptr must be non-decreasing and span the chunk")
        c = None
    else:
        raise ValueError("pass exactly one of cells / indptr")
    ch = _Chunk(_ptr(g), _ptr(v), len(g), _ptr(cm), len(cm), _ptr(gm), len(gm), float(target_sum),
                int(bool(log1p)), _ptr(c), _ptr(p), 0 if p is None else len(p), int(first_cell))
    n_rows = int(max(cm.max() + 1, 0)) if len(cm) else 0
    return ch, (g, v, cm, gm, c, p), n_rows


def _n_var(gene_map):
    return int(max(gene_map.max() + 1, 0)) if len(gene_map) else 0


# --------------------------------------------------------------------------- native-module mirror
def qc(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
       flag, cell_total, cell_ngenes, cell_flag, gene_ncells, gene_total, threads=None):
    """src/py.rs:234-248 / src/kernels.rs:164-195."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    f = _c(flag, np.bool_, "flag")
    ct, cn, cf = _c(cell_total, np.float64, "cell_total"), _c(cell_ngenes, np.uint32, "cell_ngenes"), \
        _c(cell_flag, np.float64, "cell_flag")
    gn, gt = _c(gene_ncells, np.uint32, "gene_ncells"), _c(gene_total, np.float64, "gene_total")
    if len(ct) < nr or len(cn) < nr or len(cf) < nr or len(gn) != nv or len(gt) != nv or len(f) != nv:
        raise ValueError("output sizes do not match the maps")
    lib().oc_qc(C.byref(ch), threads or DEFAULT_THREADS, _ptr(f), _ptr(ct), _ptr(cn), _ptr(cf), _ptr(gn), _ptr(gt), nv)


def gene_stats(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell, out, threads=None):
    """src/py.rs:221-232 / src/kernels.rs:144-160."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    o = _c(out, np.float64, "out")
    if o.size != nv * 5:
        raise ValueError("out must be (n_vars, 5)")
    lib().oc_gene_stats(C.byref(ch), threads or DEFAULT_THREADS, _ptr(o), nv)


def _transform(scale, mean, std, max_value, d):
    if mean is not None and std is not None:
        mu, sd = _c(mean, np.float64, "mean"), _c(std, np.float64, "std")
    elif scale:
        raise ValueError("scale=True needs mean and std")
    else:
        mu = sd = None
    if scale and (len(mu) != d or len(sd) != d):
        raise ValueError("mean/std must have length d")
    return mu, sd


def _check_sub(sub, nv, d):
    if len(sub) != nv or (len(sub) and sub.max() >= d):
        raise ValueError("sub_map must have length n_vars and values < d")


def gram_accumulate(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                    sub_map, gram, colsum, scale, mean, std, max_value, threads=None):
    """src/py.rs:270-287 / src/kernels.rs:227-309 (FP64 Gram, upper triangle)."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    sm = _c(sub_map, np.int32, "sub_map")
    cs = _c(colsum, np.float64, "colsum")
    d = len(cs)
    gr = _c(gram, np.float64, "gram")
    if gr.size != d * d:
        raise ValueError("gram must be (d, d)")
    _check_sub(sm, nv, d)
    mu, sd = _transform(scale, mean, std, max_value, d)
    lib().oc_gram_accumulate(C.byref(ch), threads or DEFAULT_THREADS, _ptr(sm), d, int(bool(scale)), _ptr(mu), _ptr(sd),
                             float(max_value), _ptr(gr), _ptr(cs))


def project(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
            sub_map, loadings, out, scale, mean, std, max_value, threads=None):
    """src/py.rs:289-309 / src/kernels.rs:352-371."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    if loadings.ndim != 2:
        raise ValueError("loadings must be (d, k)")
    d, k = loadings.shape
    sm = _c(sub_map, np.int32, "sub_map")
    ld = _c(loadings, np.float64, "loadings")
    _check_sub(sm, nv, d)
    o = _c(out, np.float32, "out")
    if o.size < nr * k:
        raise ValueError("out must be (n_rows, k)")
    mu, sd = _transform(scale, mean, std, max_value, d)
    lib().oc_project(C.byref(ch), threads or DEFAULT_THREADS, _ptr(sm), int(bool(scale)), _ptr(mu), _ptr(sd),
                     float(max_value), _ptr(ld), k, _ptr(o))


def materialize(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell):
    """src/py.rs:213-219 / src/kernels.rs:123-139."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    cap = len(genes)
    r, g, x = np.empty(cap, np.uint32), np.empty(cap, np.uint32), np.empty(cap, np.float32)
    n = lib().oc_materialize(C.byref(ch), 1, _ptr(r), _ptr(g), _ptr(x), cap)
    return r[:n].copy(), g[:n].copy(), x[:n].copy()


def group_gene_sums(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                    group_of_row, sum, sumsq, nnz, clip=None):
    """src/py.rs:311-338 / src/kernels.rs:388-442."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    gr = _c(group_of_row, np.uint32, "group_of_row")
    s, q, z = _c(sum, np.float64, "sum"), _c(sumsq, np.float64, "sumsq"), _c(nnz, np.float64, "nnz")
    if s.ndim != 2 or s.shape[1] != nv or q.shape != s.shape or z.shape != s.shape or len(gr) < nr:
        raise ValueError("sum, sumsq, nnz must be (n_groups, n_vars); group_of_row (n_rows,)")
    if np.any((gr != np.iinfo(np.uint32).max) & (gr >= s.shape[0])):
        raise ValueError("group id out of range")
    c = None if clip is None else _c(clip, np.float64, "clip")
    if c is not None and c.size != s.size:
        raise ValueError("clip must be (n_groups, n_vars)")
    lib().oc_group_gene_sums(C.byref(ch), _ptr(gr), nv, _ptr(c), _ptr(s), _ptr(q), _ptr(z))


def group_gene_totals(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell,
                      group_of_row, sum):
    """src/py.rs:340-357."""
    ch, keep, nr = _view(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)
    nv = _n_var(gene_map)
    gr = _c(group_of_row, np.uint32, "group_of_row")
    s = _c(sum, np.float64, "sum")
    if s.ndim != 2 or s.shape[1] != nv or len(gr) < nr:
        raise ValueError("sum must be (n_groups, n_vars); group_of_row (n_rows,)")
    if np.any((gr != np.iinfo(np.uint32).max) & (gr >= s.shape[0])):
        raise ValueError("group id out of range")
    lib().oc_group_gene_sums(C.byref(ch), _ptr(gr), nv, None, _ptr(s), None, None)


def t_pvalues(t, df):
    """src/py.rs:413-427 (statrs StudentsT): 2 * sf(|t|, df) capped at 1, NaN for a
    non-finite t or df <= 0; scipy's Student t here."""
    from scipy import stats
    t = np.asarray(t, np.float64)
    df = np.asarray(df, np.float64)
    ok = np.isfinite(t) & (df > 0)
    p = np.full(t.shape, np.nan)
    p[ok] = np.minimum(2.0 * stats.t.sf(np.abs(t[ok]), df[ok]), 1.0)
    return p


def knn_graph(data, k, exact=None, seed=0, threads=None):
    """src/py.rs:52-72 / src/knn.rs: exact k nearest neighbours (self excluded),
    (indices u32 (n, k'), distances f32 (n, k')), k' = min(k, n - 1)."""
    X = _c(np.asarray(data), np.float32, "data")
    n, d = X.shape
    kk = max(1, min(int(k), n - 1)) if n > 1 else 0
    idx = np.zeros((n, kk), np.uint32)
    dist = np.zeros((n, kk), np.float32)
    if kk:
        lib().oc_knn(_ptr(X), n, d, kk, _ptr(idx), _ptr(dist), threads or DEFAULT_THREADS)
    return idx, dist


def pca_from_gram(gram, colsum, n, k):
    """src/kernels.rs:313-348 with LAPACK (numpy ``eigh``, upper triangle) standing in for
    faer's ``self_adjoint_eigen``.  Returns (variance (k,), loadings (d, k), total)."""
    g = _c(gram, np.float64, "gram")
    c = _c(colsum, np.float64, "colsum")
    d = len(c)
    if g.size != d * d:
        raise ValueError("gram must be (d, d)")
    if n < 2 or d == 0:
        raise RuntimeError("need at least 2 cells and 1 gene")
    G = g.reshape(d, d)
    up = np.triu(G)
    sym = up + np.triu(G, 1).T
    nf = float(n)
    cov = (sym - np.outer(c, c) / nf) / (nf - 1.0)
    total = float(np.trace(cov))
    w, U = np.linalg.eigh(cov, UPLO="U")
    k = min(int(k), d)
    vals = np.maximum(w[::-1][:k], 0.0)
    V = U[:, ::-1][:, :k].copy()
    for j in range(k):
        col = V[:, j]
        i = int(np.argmax(np.abs(col)))  # first index of the largest |loading|
        if col[i] < 0:
            V[:, j] = -col
    return vals, np.ascontiguousarray(V), total
