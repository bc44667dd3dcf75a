"""crest_b200 -- B200-native (sm_100a) implementation of CREST's chunked
preprocessing-to-PCA path behind the reference's ``crest.pp`` / ``crest.tl``
API: CSR QC sums, lazy normalize_total + log1p, seurat HVG statistics, the
exact scale-inside-PCA Gram over the HVG columns (FP64 / FP32 / split-BF16
tensor cores), FP64 centring and eigensolve, and the score projection.
"""

__version__ = "0.1.0"

from .core import BioFrame, CSRStore, FrameStore, ParquetStore, DeviceMatrix, read_parquet  # noqa: F401
from . import pp, tl  # noqa: F401

__all__ = ["BioFrame", "CSRStore", "FrameStore", "ParquetStore", "DeviceMatrix", "read_parquet", "pp", "tl",
           "__version__"]
