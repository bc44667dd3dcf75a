"""Local quadratic regression of one predictor, as R ``loess`` / netlib
``dloess`` compute it with their defaults (Cleveland & Grosse 1991,
"Computational methods for local regression"): ``surface="interpolate"``,
tricube weights, Gaussian family (no robustness iterations).

Fitting at every data point is replaced by fits at the vertices of a k-d tree
over the predictor: an interval holding more than ``floor(n * span * cell)``
points is cut at its median point (moved off runs of equal values), and the
curve between two neighbouring vertices is the cubic Hermite interpolant of
the fitted values and slopes at both ends.  Each vertex fit is a weighted
least-squares polynomial over the ``floor(n * span)`` nearest points with
tricube weights of distance / (largest of those distances).

Host-side, O(vertices x n) numpy: it runs once per batch on the per-gene
(log mean, log variance) points of the seurat_v3 variance model.
"""

from __future__ import annotations

import numpy as np


def _vertex_fit(x: np.ndarray, y: np.ndarray, at: float, n_near: int, span: float, degree: int):
    """(value, slope) at `at` of the tricube-weighted degree-`degree` fit over the
    n_near points nearest to it."""
    dist2 = (x - at) ** 2
    idx = np.argpartition(dist2, n_near - 1)[:n_near]
    reach2 = dist2[idx].max() * max(1.0, span)
    if reach2 <= 0.0:  # every neighbour sits on the vertex
        return float(y[idx].mean()), 0.0
    inside = idx[dist2[idx] < reach2]
    w = (1.0 - (dist2[inside] / reach2) ** 1.5) ** 3
    t = x[inside] - at
    basis = np.vander(t, degree + 1, increasing=True)
    root_w = np.sqrt(w)
    coef = np.linalg.lstsq(basis * root_w[:, None], y[inside] * root_w, rcond=None)[0]
    return float(coef[0]), (float(coef[1]) if degree >= 1 else 0.0)


def _vertices(x: np.ndarray, max_points: int) -> np.ndarray:
    """Sorted vertices of the k-d tree over x (cells of at most max_points points)."""
    lo, hi = float(x.min()), float(x.max())
    pad = 0.005 * max(hi - lo, 1e-10 * max(abs(lo), abs(hi)) + 1e-30)
    lo, hi = lo - pad, hi + pad
    xs = np.sort(x)
    cuts = [lo, hi]
    todo = [(0, len(xs) - 1, lo, hi)]  # inclusive index range of the cell's points and its bounds
    while todo:
        first, last, left, right = todo.pop()
        if last - first + 1 <= max_points:
            continue
        mid = (first + last + 2) // 2 - 1  # the median point (upper of two, 1-based convention)
        # cut between two different values: try mid, mid+1, mid-1, mid+2, ... within the cell
        step = 0
        while first <= mid + step < last:
            if xs[mid + step] == xs[mid + step + 1]:
                step = -step if step > 0 else 1 - step
            else:
                mid += step
                break
        cut = float(xs[mid])
        if cut == left or cut == right:
            continue
        cuts.append(cut)
        todo.append((first, mid, left, cut))
        todo.append((mid + 1, last, cut, right))
    return np.unique(np.asarray(cuts))


def loess_fit(x, y, span: float = 0.75, degree: int = 2, cell: float = 0.2) -> np.ndarray:
    """Fitted values of the loess curve of y on x at the data points."""
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(x)
    if n == 0:
        return np.zeros(0)
    n_near = min(n, int(np.floor(n * span + 1e-5)))
    if n_near <= 0:
        raise ValueError("span is too small")
    verts = _vertices(x, int(np.floor(n * span * cell)))
    fit = np.array([_vertex_fit(x, y, v, n_near, span, degree) for v in verts])
    val, slope = fit[:, 0], fit[:, 1]
    j = np.clip(np.searchsorted(verts, x, side="left") - 1, 0, len(verts) - 2)
    a, b = verts[j], verts[j + 1]
    h = b - a
    u = (x - a) / h
    # cubic Hermite basis on [a, b]
    h00 = (1 - u) ** 2 * (1 + 2 * u)
    h01 = u ** 2 * (3 - 2 * u)
    h10 = u * (1 - u) ** 2
    h11 = -(u ** 2) * (1 - u)
    return h00 * val[j] + h01 * val[j + 1] + (h10 * slope[j] + h11 * slope[j + 1]) * h
