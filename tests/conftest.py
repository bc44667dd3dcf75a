import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _gpu_count():
    try:
        from crest_b200 import _lib
        return _lib.device_count()
    except Exception:
        return 0


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly when selected on a machine without a GPU: no skipping
    pass


@pytest.fixture(scope="session")
def small_counts():
    """1,500 cells x 600 genes, 5 clusters, NB counts, MT- genes (the reference's test fixture shape)."""
    from crest_b200 import synth
    p = synth.make_params(1500, 600, 5, 0.5, 150.0, seed=0)
    from oracle import synth as osynth
    indptr, indices, data = osynth.generate(p)
    return indptr, indices, data, 600, synth.gene_names(600), p.labels


@pytest.fixture(scope="session")
def pbmc_counts():
    """The small CPU-runnable workload: 2,700 cells x 32,738 genes, 8 clusters, ~820 nnz/cell."""
    from crest_b200 import synth
    w = synth.WORKLOADS["pbmc3k_like"]
    from oracle import synth as osynth
    indptr, indices, data = osynth.make_workload(w)
    return indptr, indices, data, w.n_genes, synth.gene_names(w.n_genes)
