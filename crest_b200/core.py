"""BioFrame: a single-cell dataset processed in cell-sorted chunks.

Mirrors the reference's data model (crest/core.py): raw counts are never
modified; cell/gene filters are kept as ``obs``/``var`` tables over the same
store and ``normalize_total``/``log1p`` are recorded in ``ops`` and applied
inside the kernels.  ``obs``/``var`` are pandas DataFrames here (the
reference uses polars, which this package does not depend on).

Stores:

* :class:`CSRStore` - CSR raw counts (``indptr`` i64, ``indices`` u32,
  ``data`` f32).  Whole-matrix passes run on a device-resident copy
  (:meth:`CSRStore.device_matrix`) or stream pinned host chunks.
* :class:`FrameStore` - COO ``(cell_id, gene_id, count)`` triplets sorted by
  cell, processed chunk by chunk through the per-chunk native functions.
* :class:`ParquetStore` - the same triplets on disk as Parquet parts, read one
  part at a time (out of core) with the next part decoded in the background.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterator, Optional, Tuple, Union

import numpy as np
import pandas as pd

from . import _lib

DEFAULT_CHUNK_NNZ = 1 << 24


class DeviceMatrix:
    """A ``crest_matrix`` handle: the CSR matrix in HBM (residency "device") or
    streamed from host memory in chunks of ``chunk_cells`` cells ("host")."""

    def __init__(self, indptr, indices, data, n_genes: int, residency: str = "device", chunk_cells: int = 16384):
        _lib.require_gpu()
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int64)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(data, dtype=np.float32)
        if self.indptr[0] != 0:
            base = self.indptr[0]
            self.indptr = self.indptr - base
        self.n_cells = len(self.indptr) - 1
        self.n_genes = int(n_genes)
        self.residency = residency
        h = C.c_void_p()
        res = _lib.MEM_DEVICE if residency == "device" else _lib.MEM_HOST
        _lib.call("crest_matrix_create", C.byref(h), _lib.ptr(self.indptr), _lib.ptr(self.indices),
                  _lib.ptr(self.data), self.n_cells, self.n_genes, res, int(chunk_cells))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.load().crest_matrix_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CSRStore:
    """Raw counts in memory as CSR (cells x genes), about 8 bytes per non-zero."""

    def __init__(self, indptr: np.ndarray, indices: np.ndarray, data: np.ndarray, n_genes: int):
        self.indptr = np.asarray(indptr, dtype=np.int64)
        self.indices = np.ascontiguousarray(indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(data, dtype=np.float32)
        self.n_cells = len(self.indptr) - 1
        self.n_genes = int(n_genes)
        self._dev = None
        self.residency = "device"
        self.chunk_cells = 16384

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def chunks(self, chunk_nnz: int = DEFAULT_CHUNK_NNZ):
        """(genes, values, cells, indptr, first_cell) views cut at ~chunk_nnz entries
        (crest/core.py:54-62)."""
        n = self.n_cells
        start = 0
        while start < n:
            target = self.indptr[start] + chunk_nnz
            end = int(np.searchsorted(self.indptr, target, side="right")) - 1
            end = min(max(end, start + 1), n)
            lo, hi = int(self.indptr[start]), int(self.indptr[end])
            yield self.indices[lo:hi], self.data[lo:hi], None, self.indptr[start:end + 1], start
            start = end

    def device_matrix(self) -> DeviceMatrix:
        if self._dev is None:
            self._dev = DeviceMatrix(self.indptr, self.indices, self.data, self.n_genes, self.residency,
                                     self.chunk_cells)
        return self._dev

    def nbytes(self) -> int:
        return self.indptr.nbytes + self.indices.nbytes + self.data.nbytes


class FrameStore:
    """Raw counts as ``(cell_id, gene_id, count)`` triplets sorted by cell (crest/core.py:69-105)."""

    def __init__(self, cells, genes, counts, n_cells: int, n_genes: int):
        cells = np.asarray(cells, dtype=np.uint32)
        genes = np.asarray(genes, dtype=np.uint32)
        counts = np.asarray(counts, dtype=np.float32)
        if len(cells) > 1 and np.any(cells[1:] < cells[:-1]):
            order = np.argsort(cells, kind="stable")
            cells, genes, counts = cells[order], genes[order], counts[order]
        self._cells = np.ascontiguousarray(cells)
        self._genes = np.ascontiguousarray(genes)
        self._vals = np.ascontiguousarray(counts)
        self.n_cells, self.n_genes = int(n_cells), int(n_genes)

    @property
    def nnz(self) -> int:
        return len(self._cells)

    def chunks(self, chunk_nnz: int = DEFAULT_CHUNK_NNZ):
        n = len(self._cells)
        lo = 0
        while lo < n:
            hi = min(lo + chunk_nnz, n)
            if hi < n:  # extend to the end of the current cell
                hi = int(np.searchsorted(self._cells, self._cells[hi - 1], side="right"))
            yield self._genes[lo:hi], self._vals[lo:hi], self._cells[lo:hi], None, 0
            lo = hi


class ParquetStore:
    """Raw counts on disk, out of core: a directory of ``part-*.parquet`` files of
    ``(cell_id, gene_id, count)`` rows, each file holding whole cells in cell
    order (crest/core.py:108-135).  One chunk is one file; while the GPU works
    on a chunk, a reader thread already decodes the next file, so disk and
    decompression overlap the device passes.  Made by
    :meth:`BioFrame.write_parquet`, opened with :func:`read_parquet`."""

    def __init__(self, path, n_cells: int, n_genes: int):
        from pathlib import Path
        self.path = Path(path)
        self.parts = sorted(self.path.glob("part-*.parquet"))
        if not self.parts:
            raise FileNotFoundError(f"no part-*.parquet files in {self.path}")
        self.n_cells, self.n_genes = int(n_cells), int(n_genes)

    @property
    def nnz(self) -> int:
        import pyarrow.parquet as pq
        return int(sum(pq.ParquetFile(p).metadata.num_rows for p in self.parts))

    @staticmethod
    def _read(part):
        import pyarrow.parquet as pq
        t = pq.read_table(part, columns=["cell_id", "gene_id", "count"])
        col = {name: t.column(name).to_numpy() for name in ("cell_id", "gene_id", "count")}
        return (np.ascontiguousarray(col["gene_id"], dtype=np.uint32),
                np.ascontiguousarray(col["count"], dtype=np.float32),
                np.ascontiguousarray(col["cell_id"], dtype=np.uint32))

    def chunks(self, chunk_nnz: int = DEFAULT_CHUNK_NNZ):
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=1) as pool:
            nxt = pool.submit(self._read, self.parts[0])
            for i in range(len(self.parts)):
                genes, values, cells = nxt.result()
                if i + 1 < len(self.parts):
                    nxt = pool.submit(self._read, self.parts[i + 1])
                yield genes, values, cells, None, 0


Store = Union[CSRStore, FrameStore, ParquetStore]


@dataclass
class BioFrame:
    """A single-cell dataset: raw counts plus annotations (the reference's BioFrame,
    crest/core.py:141-309)."""

    store: Store
    obs: pd.DataFrame
    var: pd.DataFrame
    obsm: dict = field(default_factory=dict)
    varm: dict = field(default_factory=dict)
    uns: dict = field(default_factory=dict)
    ops: list = field(default_factory=list)
    chunk_nnz: int = DEFAULT_CHUNK_NNZ

    # ---- construction
    @classmethod
    def from_csr(cls, indptr, indices, data, n_genes: int, obs=None, var=None) -> "BioFrame":
        return cls._with_store(CSRStore(indptr, indices, data, n_genes), obs, var)

    @classmethod
    def from_scipy(cls, X, obs=None, var=None) -> "BioFrame":
        X = X.tocsr()
        X.sort_indices()
        return cls.from_csr(X.indptr, X.indices, X.data, X.shape[1], obs, var)

    @classmethod
    def from_triplets(cls, cells, genes, counts, n_cells: Optional[int] = None, n_genes: Optional[int] = None,
                      obs=None, var=None) -> "BioFrame":
        cells = np.asarray(cells)
        genes = np.asarray(genes)
        n_cells = n_cells if n_cells is not None else (len(obs) if obs is not None else int(cells.max()) + 1)
        n_genes = n_genes if n_genes is not None else (len(var) if var is not None else int(genes.max()) + 1)
        return cls._with_store(FrameStore(cells, genes, counts, n_cells, n_genes), obs, var)

    @classmethod
    def _with_store(cls, store: Store, obs, var) -> "BioFrame":
        if obs is None:
            obs = pd.DataFrame({"cell_id": np.arange(store.n_cells, dtype=np.uint32)})
        else:
            obs = pd.DataFrame(obs).reset_index(drop=True)
            if "cell_id" not in obs.columns:
                obs["cell_id"] = np.arange(len(obs), dtype=np.uint32)
        if var is None:
            var = pd.DataFrame({"gene_id": np.arange(store.n_genes, dtype=np.uint32)})
        else:
            var = pd.DataFrame(var).reset_index(drop=True)
            if "gene_id" not in var.columns:
                var["gene_id"] = np.arange(len(var), dtype=np.uint32)
        if len(obs) != store.n_cells or len(var) != store.n_genes:
            raise ValueError(f"obs/var sizes {len(obs)}/{len(var)} do not match store {store.n_cells}/{store.n_genes}")
        return cls(store=store, obs=obs, var=var)

    # ---- shape / names
    @property
    def n_obs(self) -> int:
        return len(self.obs)

    @property
    def n_vars(self) -> int:
        return len(self.var)

    @property
    def shape(self) -> Tuple[int, int]:
        return self.n_obs, self.n_vars

    @property
    def var_names(self) -> list:
        for c in ("gene_name", "gene_symbols", "gene_ids"):
            if c in self.var.columns:
                return [str(x) for x in self.var[c].tolist()]
        return [str(x) for x in self.var["gene_id"].tolist()]

    def __repr__(self) -> str:
        pending = [o[0] for o in self.ops]
        lines = [f"<BioFrame: {self.n_obs:,} cells, {self.n_vars:,} genes, store={type(self.store).__name__}, "
                 f"lazy ops={pending if pending else 'none'}>"]
        for label, keys in (("obs", self.obs.columns), ("var", self.var.columns), ("obsm", self.obsm),
                            ("varm", self.varm), ("uns", self.uns)):
            if len(keys):
                lines.append(f"  {label}: " + ", ".join(map(str, keys)))
        return "\n".join(lines)

    # ---- maps from store ids to current rows (crest/core.py:244-263)
    def _cell_map(self) -> np.ndarray:
        m = np.full(self.store.n_cells, -1, dtype=np.int64)
        m[self.obs["cell_id"].to_numpy().astype(np.int64)] = np.arange(self.n_obs, dtype=np.int64)
        return m

    def _gene_map(self) -> np.ndarray:
        m = np.full(self.store.n_genes, -1, dtype=np.int32)
        m[self.var["gene_id"].to_numpy().astype(np.int64)] = np.arange(self.n_vars, dtype=np.int32)
        return m

    def _transform(self) -> Tuple[float, bool]:
        target, log = 0.0, False
        for op in self.ops:
            if op[0] == "normalize_total":
                if log:
                    raise ValueError("normalize_total after log1p is not supported")
                target = float(op[1])
            elif op[0] == "log1p":
                log = True
        return target, log

    def iter_ctx(self, transform: bool = True) -> Iterator[tuple]:
        """Argument tuples of the per-chunk native functions:
        ``(genes, values, cell_map, gene_map, target_sum, log1p, cells, indptr, first_cell)``."""
        cmap, gmap = self._cell_map(), self._gene_map()
        target, log = self._transform() if transform else (0.0, False)
        for genes, values, cells, indptr, first in self.store.chunks(self.chunk_nnz):
            yield (np.ascontiguousarray(genes, dtype=np.uint32), np.ascontiguousarray(values, dtype=np.float32),
                   cmap, gmap, target, log,
                   None if cells is None else np.ascontiguousarray(cells, dtype=np.uint32),
                   None if indptr is None else np.ascontiguousarray(indptr, dtype=np.int64), int(first))

    def device_matrix(self) -> Optional[DeviceMatrix]:
        """Whole-matrix device handle for CSR stores, ``None`` for triplet stores."""
        return self.store.device_matrix() if isinstance(self.store, CSRStore) else None

    # ---- subsetting
    # uns entries whose contents are indexed by cells: stale once cells are dropped
    _PER_CELL_UNS = ("neighbors",)

    def _subset(self, obs_mask=None, var_mask=None) -> "BioFrame":
        """A view keeping the masked cells / genes; the store is shared, no counts are copied."""
        def pick(frame, mask):
            return frame if mask is None else frame.loc[np.asarray(mask, bool)].reset_index(drop=True)

        def pick_rows(arrays, mask):
            return dict(arrays) if mask is None else {key: a[np.asarray(mask, bool)] for key, a in arrays.items()}

        uns = {key: v for key, v in self.uns.items() if obs_mask is None or key not in self._PER_CELL_UNS}
        return BioFrame(self.store, pick(self.obs, obs_mask), pick(self.var, var_mask), pick_rows(self.obsm, obs_mask),
                        pick_rows(self.varm, var_mask), uns, list(self.ops), self.chunk_nnz)

    def filter_cells(self, mask) -> "BioFrame":
        """Keep cells where the boolean mask holds."""
        return self._subset(obs_mask=np.asarray(mask, dtype=bool))

    def filter_genes(self, mask) -> "BioFrame":
        """Keep genes where the boolean mask holds."""
        return self._subset(var_mask=np.asarray(mask, dtype=bool))

    def raw_triplets(self) -> Iterator[tuple]:
        """Raw counts of the kept cells / genes with their current row / column ids,
        chunk by chunk: ``(rows u32, cols u32, counts f32)``, cell-sorted."""
        cmap, gmap = self._cell_map(), self._gene_map()
        for genes, values, cells, indptr, first in self.store.chunks(self.chunk_nnz):
            if cells is None:
                cells = first + np.repeat(np.arange(len(indptr) - 1, dtype=np.int64), np.diff(indptr))
            cells = np.asarray(cells, dtype=np.int64)
            ok = cells < len(cmap)
            rows = np.full(len(cells), -1, np.int64)
            rows[ok] = cmap[cells[ok]]
            g = np.asarray(genes, dtype=np.int64)
            okg = g < len(gmap)
            cols = np.full(len(g), -1, np.int64)
            cols[okg] = gmap[g[okg]]
            keep = (rows >= 0) & (cols >= 0)
            yield rows[keep].astype(np.uint32), cols[keep].astype(np.uint32), np.asarray(values, np.float32)[keep]

    def write_parquet(self, path, nnz_per_part: int = 1 << 23) -> None:
        """Write the raw counts of the kept cells / genes (current ids) as a Parquet
        directory of whole-cell parts of about ``nnz_per_part`` stored values, with
        ``obs.parquet`` / ``var.parquet`` (crest/core.py:368-392)."""
        from pathlib import Path
        import pyarrow as pa
        import pyarrow.parquet as pq
        path = Path(path)
        path.mkdir(parents=True, exist_ok=True)
        for old in path.glob("part-*.parquet"):
            old.unlink()
        pending, n_pending, part = [], 0, 0

        def flush():
            nonlocal pending, n_pending, part
            if pending:
                cols = [np.concatenate([p[i] for p in pending]) for i in range(3)]
                table = pa.table({"cell_id": cols[0], "gene_id": cols[1], "count": cols[2]})
                pq.write_table(table, path / f"part-{part:05d}.parquet", compression="zstd")
                part += 1
            pending, n_pending = [], 0

        for r, g, v in self.raw_triplets():
            lo = 0
            while lo < len(r):
                hi = min(lo + nnz_per_part - n_pending, len(r))
                if hi < len(r):  # a part ends where a cell ends
                    hi = int(np.searchsorted(r, r[hi - 1], side="right"))
                pending.append((r[lo:hi], g[lo:hi], v[lo:hi]))
                n_pending += hi - lo
                lo = hi
                if n_pending >= nnz_per_part:
                    flush()
        flush()
        obs = self.obs.copy()
        obs["cell_id"] = np.arange(self.n_obs, dtype=np.uint32)
        var = self.var.copy()
        var["gene_id"] = np.arange(self.n_vars, dtype=np.uint32)
        pq.write_table(pa.Table.from_pandas(obs, preserve_index=False), path / "obs.parquet")
        pq.write_table(pa.Table.from_pandas(var, preserve_index=False), path / "var.parquet")

    def copy(self) -> "BioFrame":
        return BioFrame(self.store, self.obs.copy(), self.var.copy(), dict(self.obsm), dict(self.varm),
                        dict(self.uns), list(self.ops), self.chunk_nnz)


def read_parquet(path, chunk_nnz: int = DEFAULT_CHUNK_NNZ) -> BioFrame:
    """Open a Parquet directory written by :meth:`BioFrame.write_parquet` (out of
    core: passes read one part at a time; crest/core.py:414-421)."""
    from pathlib import Path
    import pyarrow.parquet as pq
    path = Path(path)
    obs = pq.read_table(path / "obs.parquet").to_pandas()
    var = pq.read_table(path / "var.parquet").to_pandas()
    bf = BioFrame._with_store(ParquetStore(path, len(obs), len(var)), obs, var)
    bf.chunk_nnz = chunk_nnz
    return bf
