"""The north-star mobility path on the GPU (no reference counterpart; the
oracle is the project's FP64 restatement and a dense eigendecomposition):

* the Ewald-summed RPY tensor for every pair against oracle/bd_oracle.c's
  bdo_calc_hi_ewald, FP64, 1e-10 relative;
* M v against the dense product, FP64 1e-10 and FP32-stored tiles 1e-6;
* the Lanczos sqrt(M) z at tolerance 1e-6 (the solve stops when the geometric
  tail of its successive changes, an estimate of the iterate's own error, is
  below the tolerance) against numpy.linalg.eigh's square root: 1e-6
  relative with FP64 tiles; with FP32-stored tiles the operator itself is off
  by about 1e-7, so 2e-6;
* a few hundred Krylov Brownian steps run without error and keep every FENE
  bond inside qmax.
"""
import numpy as np
import pytest

import bd_b200 as B
import oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _system(flow, Nb, Nc, L, seed):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    return x, y, z


def _prepared(flow, t, precision="fp64", Nb=25, Nc=20, L=30.0, seed=31):
    x, y, z = _system(flow, Nb, Nc, L, seed + t)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, mobility="ewald",
                                precision=precision, noise="philox"))
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    c.set_positions(x, y, z)
    c.set_time(t, t)
    c.update_lattice(t)
    c.calc_hi()
    return c, o, (x, y, z)


def upper_and_diag(M, N):
    Bk = M.reshape(N, N, 3, 3)
    iu = np.triu_indices(N, 1)
    return Bk[iu], np.array([[Bk[i, i, a, a] for a in range(3)] for i in range(N)])


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 3000), (1, 0), (1, 3000)])
def test_ewald_mobility_vs_oracle(flow, t):
    c, o, (x, y, z) = _prepared(flow, t)
    M = o.calc_hi_ewald(x, y, z)
    ub, db = upper_and_diag(c.mobility(), o.N)
    ur, dr = upper_and_diag(M, o.N)
    assert rel_err(ub, ur) < 1e-10 and rel_err(db, dr) < 1e-10


@pytest.mark.parametrize("flow", [0, 1])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-6)])
def test_mobility_product(flow, precision, tol):
    c, o, (x, y, z) = _prepared(flow, 1000, precision)
    Mf = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    v = np.random.default_rng(3).normal(size=3 * o.N)
    assert rel_err(c.mobility_apply(v), Mf @ v) < tol


@pytest.mark.parametrize("flow", [0, 1])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("fp32", 2e-6)])
def test_lanczos_sqrt_vs_eigh(flow, precision, tol):
    c, o, (x, y, z) = _prepared(flow, 500, precision)
    Mf = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    zz = np.random.default_rng(7).normal(size=3 * o.N)
    ref, lmin = O.sqrtm_apply(Mf, zz)
    assert lmin > 0
    got, iters = c.lanczos_sqrt(zz)
    assert 2 <= iters < 80
    assert rel_err(got, ref) < tol, (iters, rel_err(got, ref))
    st = c.lanczos_stats()
    assert st["calls"] == 1 and st["maxed"] == 0 and st["negative"] == 0


@pytest.mark.parametrize("flow", [0, 1])
def test_krylov_steps_stable(flow):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = _system(flow, Nb, Nc, L, 41)
    q = B.random_charges(Nb, Nc, 0.5, 43)
    # FENE k = 30 in both flows (the shear tree's forced k = 200 is for its
    # Hookean spring; shear_kappas_override keeps the configured k)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.01, 5e-4, mobility="ewald", precision="fp32",
                                noise="philox", MStep=100, Ncharges=len(q),
                                shear_kappas_override=1))
    c.set_positions(x, y, z)
    c.set_charges(q)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.inverse_coords()
    c.step_lanczos(0, 250, True)
    px = np.stack(c.positions())
    assert np.all(np.isfinite(px))
    st = c.lanczos_stats()
    assert st["calls"] == 250 and st["maxed"] == 0
    assert st["iterations"] / st["calls"] < 60
