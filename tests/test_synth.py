import numpy as np

from crest_b200 import synth


def test_generator_is_deterministic_and_thread_invariant():
    p = synth.make_params(300, 2000, 4, 0.2, 120.0, seed=3)
    a = synth.generate(p, threads=1)
    b = synth.generate(p, threads=7)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_generator_hits_nnz_target_and_sorted_rows():
    p = synth.make_params(2000, 5000, 6, 0.2, 300.0, seed=5)
    indptr, indices, data = synth.generate(p)
    per_cell = np.diff(indptr)
    assert abs(per_cell.mean() / 300.0 - 1.0) < 0.15
    assert np.all(data >= 1) and np.all(data == np.round(data))
    for i in range(0, 2000, 97):
        row = indices[indptr[i]:indptr[i + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)
    assert indices.max() < 5000


def test_subset_of_cells_matches_prefix():
    w = synth.Workload("t", 500, 1000, 3, 0.2, 100.0, 9)
    full = synth.make_workload(w)
    part = synth.make_workload(w, n_cells=200)
    assert np.array_equal(part[0], full[0][:201])
    nnz = part[0][-1]
    assert np.array_equal(part[1], full[1][:nnz]) and np.array_equal(part[2], full[2][:nnz])
