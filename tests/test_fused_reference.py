"""The FP64 reference of the fused map (tests/fused_case.py) against central
finite differences (eps = 1e-3, f64), away from the clip boundary: this pins
the reference gradient that the CUDA backward is compared with."""

import numpy as np
import torch

from fused_case import loss_of, make_case, ref_run, reference


def test_fp64_reference_gradient_matches_finite_differences():
    c = make_case(n=400, d=120, k=8, max_value=0.75, seed=3)
    _, rx, rsf, rW = ref_run(c)
    rng = np.random.default_rng(5)
    eps = 1e-3
    wts = torch.tensor(c["wts"])

    def f(values, sf, W):
        with torch.no_grad():
            return float(loss_of(reference(c, values, sf, W), wts))

    base = [torch.tensor(c["values"].astype(np.float64)), torch.tensor(c["sf"].astype(np.float64)),
            torch.tensor(c["W"].astype(np.float64))]
    # z of every entry, to keep finite differences away from the clip boundary
    cell = np.repeat(np.arange(c["n"]), np.diff(c["indptr"]))
    g = c["indices"]
    z = (np.log1p(c["values"] / c["sf"][cell]) - c["mean"][g]) / c["std"][g]
    margin = np.abs(np.abs(z) - c["max_value"])
    safe = np.flatnonzero(margin > 0.05)
    checks = [(0, int(i)) for i in rng.choice(safe, 12, replace=False)]
    nonempty = np.diff(c["indptr"]) > 0
    cell_margin = np.full(c["n"], -1.0)
    cell_margin[nonempty] = np.minimum.reduceat(margin, c["indptr"][:-1][nonempty])
    cells_safe = np.flatnonzero(cell_margin > 0.05)
    checks += [(1, int(i)) for i in rng.choice(cells_safe, 6, replace=False)]
    checks += [(2, (int(rng.integers(c["d"])), int(rng.integers(c["k"])))) for _ in range(6)]
    grads = [rx, rsf, rW]
    for which, idx in checks:
        plus = [t.clone() for t in base]
        minus = [t.clone() for t in base]
        plus[which][idx] += eps
        minus[which][idx] -= eps
        fd = (f(*plus) - f(*minus)) / (2 * eps)
        an = float(grads[which][idx])
        scale = float(torch.linalg.norm(grads[which])) / np.sqrt(grads[which].numel())
        assert abs(fd - an) <= 1e-4 * max(abs(an), scale), (which, idx, fd, an)


