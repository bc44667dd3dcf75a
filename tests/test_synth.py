import numpy as np
import pytest

from crest_b200 import synth
from oracle import synth as osynth


def test_generator_is_deterministic_and_thread_invariant():
    p = synth.make_params(300, 2000, 4, 0.2, 120.0, seed=3)
    a = osynth.generate(p, threads=1)
    b = osynth.generate(p, threads=7)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_generator_hits_nnz_target_and_sorted_rows():
    p = synth.make_params(2000, 5000, 6, 0.2, 300.0, seed=5)
    indptr, indices, data = osynth.generate(p)
    per_cell = np.diff(indptr)
    assert abs(per_cell.mean() / 300.0 - 1.0) < 0.15
    assert np.all(data >= 1) and np.all(data == np.round(data))
    for i in range(0, 2000, 97):
        row = indices[indptr[i]:indptr[i + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)
    assert indices.max() < 5000


def test_subset_of_cells_matches_prefix():
    w = synth.Workload("t", 500, 1000, 3, 0.2, 100.0, 9)
    full = osynth.make_workload(w)
    part = osynth.make_workload(w, n_cells=200)
    assert np.array_equal(part[0], full[0][:201])
    nnz = part[0][-1]
    assert np.array_equal(part[1], full[1][:nnz]) and np.array_equal(part[2], full[2][:nnz])


def test_zero_shortcut_keeps_the_counts():
    """The draw skips exp/log1p when the uniform lies clearly below 1 - mu <= P(0);
    a plain restatement of the full inverse-CDF draw gives the same counts."""
    from math import exp, log1p
    p = synth.make_params(40, 400, 3, 0.3, 60.0, seed=21)
    indptr, indices, data = osynth.generate(p)
    dense = np.zeros((40, 400))
    for c in range(40):
        dense[c, indices[indptr[c]:indptr[c + 1]]] = data[indptr[c]:indptr[c + 1]]

    def mix(x):
        m = (1 << 64) - 1
        x = (x + 0x9e3779b97f4a7c15) & m
        x = ((x ^ (x >> 30)) * 0xbf58476d1ce4e5b9) & m
        x = ((x ^ (x >> 27)) * 0x94d049bb133111eb) & m
        return x ^ (x >> 31)

    phi, r = p.dispersion, 1.0 / p.dispersion
    for c in range(40):
        for g in range(0, 400, 7):
            key = (mix(p.seed ^ mix((c * 0xd1b54a32d192ed03 + 0x8cb92ba72f3d8dd7) & ((1 << 64) - 1)))
                   + g * 0xaef17502108ef2d9) & ((1 << 64) - 1)
            u = (mix(key) >> 11) * 2.0 ** -53
            mu = p.lib[c] * p.prob[p.labels[c], g]
            pm = phi * mu
            p0 = exp(-r * log1p(pm))
            k, pk, cdf = 0, p0, p0
            if u >= p0:
                q = pm / (1 + pm)
                while cdf <= u:
                    k += 1
                    pk *= (k - 1 + r) / k * q
                    cdf += pk
            assert dense[c, g] == k, (c, g)


@pytest.mark.gpu
def test_gpu_generator_matches_host_generator():
    """The GPU generator and the oracle's host-thread generator draw the same matrix."""
    w = synth.Workload("t", 3000, 20000, 6, 0.2, 900.0, 17)
    a = synth.make_workload(w)
    b = osynth.make_workload(w)
    for x, y in zip(a, b):
        assert x.dtype == y.dtype and np.array_equal(x, y)
