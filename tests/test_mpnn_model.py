"""CPU checks of the learned-preconditioner network model (oracle/mpnn_oracle.py).

* the analytic gradient of the exact (unrounded) model against central finite
  differences, 1e-6 relative per parameter group;
* with BF16 rounding of the dense-product operands the gradient stays within
  1e-2 of the exact one (the rounding the tensor-core kernels apply);
* the blocks are symmetric with eigenvalues at least a_i / 2.
"""
import numpy as np
import pytest

import mpnn_oracle as Q
from conftest import rel_err


def _graph(N=24, seed=3):
    r = np.random.default_rng(seed)
    nbr = np.full((N, Q.KN), -1)
    for i in range(N):
        k = r.integers(4, Q.KN + 1)
        nbr[i, :k] = r.choice([j for j in range(N) if j != i], k, replace=False)
    v = r.normal(size=(N, Q.KN, 3))
    nvec = v / np.linalg.norm(v, axis=2, keepdims=True) * (nbr[..., None] >= 0)
    d = r.uniform(2.0, 6.0, (N, Q.KN))
    mu = 2 + 4 * np.arange(Q.NR) / (Q.NR - 1)
    rbf = np.exp(-0.5 * ((d[..., None] - mu) / 0.35) ** 2) * (nbr[..., None] >= 0)
    w = []
    for name, shp in Q.LAYOUT:
        w.append(r.normal(0, 0.3 if name.startswith("W") else 0.1, shp).reshape(-1))
    z = r.normal(size=(N, 3))
    t = r.normal(size=(N, 3)) * 0.3
    return np.concatenate(w), nbr, nvec, rbf, z, t


def test_gradient_finite_differences():
    w, nbr, nvec, rbf, z, t = _graph()
    _, g, _ = Q.loss_grad(w, nbr, nvec, rbf, z, t, bf16=False)
    r = np.random.default_rng(0)
    o = 0
    for name, shp in Q.LAYOUT:
        n = int(np.prod(shp))
        idx = o + r.choice(n, min(n, 6), replace=False)
        fd = []
        for k in idx:
            h = 1e-6 * max(1.0, abs(w[k]))
            wp, wm = w.copy(), w.copy()
            wp[k] += h
            wm[k] -= h
            lp = Q.loss_grad(wp, nbr, nvec, rbf, z, t, bf16=False)[0]
            lm = Q.loss_grad(wm, nbr, nvec, rbf, z, t, bf16=False)[0]
            fd.append((lp - lm) / (2 * h))
        assert rel_err(g[idx], np.array(fd)) < 1e-6, name
        o += n


def test_bf16_gradient_close_to_exact():
    w, nbr, nvec, rbf, z, t = _graph()
    _, ge, _ = Q.loss_grad(w, nbr, nvec, rbf, z, t, bf16=False)
    _, gb, _ = Q.loss_grad(w, nbr, nvec, rbf, z, t, bf16=True)
    assert rel_err(gb, ge) < 1e-2


def test_blocks_symmetric_positive():
    w, nbr, nvec, rbf, _, _ = _graph()
    c = Q.forward(w, nbr, nvec, rbf)
    G = c["G"]
    assert np.allclose(G, G.transpose(0, 2, 1))
    ev = np.linalg.eigvalsh(G)
    assert np.all(ev >= 0.5 * c["a"][:, None] - 1e-12)
