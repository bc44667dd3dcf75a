"""Cell-sharded runs over several processes, one GPU each.

Every rank holds a :class:`~crest_b200.core.BioFrame` over its own cells
(the same genes everywhere).  The path shards by cells: QC, gene statistics,
Gram partials and the projection are per cell.  Three sums over ranks make
the result that of one process over all cells:

1. per-gene QC sums (``filter_genes`` counts cells over all ranks);
2. per-gene statistics and the cell count (HVG selection, scale mean/std);
3. the FP64 Gram, its column sums and the cell count (PCA), once, before
   the eigensolve, which then runs replicated on every rank.

Enable with :func:`enable` after ``torch.distributed.init_process_group``
("nccl" for device buffers on GPUs, "gloo" for host-only use); the functions
of :mod:`crest_b200.pp` and :mod:`crest_b200.tl` then reduce at those points.
Every rank must call them in the same order.  Without :func:`enable` all
sums are the identity.
"""

from __future__ import annotations

import numpy as np

_group = None
_enabled = False


class DevArray:
    """``__cuda_array_interface__`` view of ``n`` f64 values at a device address."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3}


def enable(group=None) -> None:
    """Reduce over the ranks of ``group`` (default: the world) from now on."""
    global _group, _enabled
    import torch.distributed as dist
    if not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    _group, _enabled = group, dist.get_world_size(group) > 1


def disable() -> None:
    global _group, _enabled
    _group, _enabled = None, False


def active() -> bool:
    return _enabled


def _nccl() -> bool:
    import torch.distributed as dist
    return dist.get_backend(_group) == "nccl"


def sum_host(a: np.ndarray) -> np.ndarray:
    """Element-wise sum over ranks of a host array (float64 arithmetic; exact
    for integer counts below 2^53); returns an array of ``a``'s dtype."""
    if not _enabled:
        return a
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).copy())
    if _nccl():
        t = t.cuda()
        dist.all_reduce(t, group=_group)
        t = t.cpu()
    else:
        dist.all_reduce(t, group=_group)
    return t.numpy().astype(a.dtype, copy=False)


def sum_count(n: int) -> int:
    """Total of an integer over ranks (cells kept on each rank)."""
    if not _enabled:
        return int(n)
    return int(round(float(sum_host(np.array([n], np.float64))[0])))


def sum_device(ptr: int, n: int) -> None:
    """In-place sum over ranks of ``n`` f64 values in device memory."""
    if not _enabled or n == 0:
        return
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(DevArray(ptr, n), device="cuda")
    if _nccl():
        dist.all_reduce(t, group=_group)
    else:
        h = t.cpu()
        dist.all_reduce(h, group=_group)
        t.copy_(h)
    torch.cuda.synchronize()
