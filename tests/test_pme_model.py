"""CPU checks of the particle-mesh mobility model (oracle/pme_oracle.py).

* its Ewald sum (any split parameter, calcHI's overlap and self-block
  conventions) against oracle/bd_oracle.c's dense bdo_calc_hi_ewald, which is
  pinned to the reference's calcHI: agreement to the dense sum's own
  convergence, 1e-5 relative, in the first half of the lattice period.  In
  the second half calcHI halves its split parameter, and its k-vector box
  (kvectors, shear/src/main26.c:1557-1600), sized from the cell edges, no
  longer holds every k inside its cutoff once the cell is strongly skewed:
  there the dense sum is 1e-4 to 2e-3 from the converged one, which the
  model (and the CUDA particle-mesh path) follow instead;
* its smooth-PME sum (grid 1.5 L, order 8, cutoff 10, split 0.4) against
  that Ewald sum, 1e-5 relative, in shear and in planar extension at several
  points of the lattice period;
* the default grid rule at its accuracy bound (12.9 L / rc points: split
  parameter 4 / rc times spacing 0.31 at L = 30, rc = 12.9, K = 30): within
  5e-6 of the converged Ewald sum over the lattice period of both flows
  (3.3e-6 at most on these systems);
* the Gauss-reduced cell spans the same lattice.
"""
import numpy as np
import pytest

import bd_b200 as B
import oracle as O
import pme_oracle as P
from conftest import rel_err


def _system(flow, t, Nb=25, Nc=8, L=30.0, seed=31):
    x, y, z = B.random_chains(Nb, Nc, L, seed + t, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    s = o.s
    if flow == 1:
        xl, yl = x * s.cth - y * s.sth, x * s.sth + y * s.cth
    else:
        xl, yl = x, y
    return o, (x, y, z), np.stack([xl, yl, z], 1)


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 4000), (1, 2000), (1, 4500)])
def test_ewald_model_vs_dense_oracle(flow, t):
    o, (x, y, z), pos = _system(flow, t)
    M = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    v = np.random.default_rng(1).normal(size=(o.N, 3))
    ar = P.ref_alpha(t, o.s.tp, o.s.L2yp)
    H = P.cell(list(o.s.L1), list(o.s.L2), 30.0)
    got = P.ewald_apply(H, pos, v, alpha=ar) - v @ P.self_offdiag(H, ar).T
    assert rel_err(got.reshape(-1), M @ v.reshape(-1)) < 1e-5


@pytest.mark.parametrize("flow,t", [(0, 6000), (1, 8000)])
def test_pme_model_vs_ewald_model(flow, t):
    o, _, pos = _system(flow, t)
    v = np.random.default_rng(2).normal(size=(o.N, 3))
    ar = P.ref_alpha(t, o.s.tp, o.s.L2yp)
    H = P.reduced_cell(list(o.s.L1), list(o.s.L2), 30.0)
    ref = P.ewald_apply(H, pos, v, alpha=ar, tol_exp=30.0) - v @ P.self_offdiag(H, ar, 30.0).T
    got = P.pme_apply(H, pos, v, K=45, p=8, alpha=0.4, rc=10.0, alpha_ref=ar)
    assert rel_err(got, ref) < 1e-5


@pytest.mark.parametrize("flow", [0, 1])
@pytest.mark.parametrize("frac", [0.0, 0.25, 0.5, 0.7, 0.9])
def test_default_grid_rule_accuracy(flow, frac):
    L, rc = 30.0, 12.9
    K = B.pme_default_grid(L, rc)
    assert K == 30 and abs(4.0 / rc * L / K - 0.31) < 1e-3
    o = O.Oracle(flow, 25, 8, L, 0.2, 5e-4)
    t = int(frac * o.s.tp)
    o, _, pos = _system(flow, t, seed=41)
    v = np.random.default_rng(5).normal(size=(o.N, 3))
    ar = P.ref_alpha(t, o.s.tp, o.s.L2yp)
    H = P.reduced_cell(list(o.s.L1), list(o.s.L2), L)
    ref = P.ewald_apply(H, pos, v, alpha=ar, tol_exp=30.0) - v @ P.self_offdiag(H, ar, 30.0).T
    got = P.pme_apply(H, pos, v, K=K, p=8, alpha=4.0 / rc, rc=rc, alpha_ref=ar)
    assert rel_err(got, ref) < 5e-6


@pytest.mark.parametrize("flow,t", [(0, 7000), (1, 5000)])
def test_reduced_cell_same_lattice(flow, t):
    o = O.Oracle(flow, 25, 8, 30.0, 0.2, 5e-4)
    o.lattice(t)
    H = P.cell(list(o.s.L1), list(o.s.L2), 30.0)
    R = P.reduced_cell(list(o.s.L1), list(o.s.L2), 30.0)
    U = np.linalg.solve(H, R)  # integer unimodular change of basis
    assert np.allclose(U, np.rint(U), atol=1e-9) and abs(abs(np.linalg.det(np.rint(U))) - 1) < 1e-9
    w = P._widths(R)
    assert w.min() >= 0.86 * 30.0 - 1e-9
