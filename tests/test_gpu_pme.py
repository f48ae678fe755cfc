"""The matrix-free particle-mesh mobility (BD_MOB_PME) on the GPU.

No reference counterpart; checked against

* oracle/pme_oracle.py's pme_apply with the same grid, order, split and
  cutoff (the same discretisation), FP64, 1e-11 relative: this pins the
  spreading, transforms, influence tensor, interpolation, pair list, overlap
  convention and self-block convention to rounding;
* oracle/bd_oracle.c's dense Ewald mobility (bdo_calc_hi_ewald) at the
  default discretisation, 2e-5 relative (the dense sum itself is converged to
  about 3e-6, the particle-mesh sum to a few 1e-6), in the first half of the
  lattice period, where the dense sum's k-vector box holds every k inside
  its cutoff; in the second half the particle-mesh sum is checked against
  the converged Ewald model of oracle/pme_oracle.py;
* FP32 storage of grids, transforms, influence and pair tensors (FP64
  accumulation) against the FP64 path, 1e-5 relative;
* the square root: Lanczos sqrt(M) z at tolerance 1e-6 with the FP64 PME
  product against numpy.linalg.eigh of the PME operator itself (assembled
  column by column from the same product), 1e-6 relative (the Krylov gate);
  and against eigh of the dense Ewald matrix, 3e-5 (the gate plus the
  particle-mesh discretisation);
* the noise blocks' multi-vector product (bd_mobility_apply_block: right-hand
  sides packed in complex pairs, in-place complex transforms, influence on
  the full spectrum) against one product per vector (real-to-complex
  transforms), FP64 1e-12, FP32 2e-6, and FP32 blocks against FP64 single
  products 1e-5, with an odd number of vectors (a lone right-hand side in the
  last pair);
* a few hundred Krylov Brownian steps with the PME mobility run without error;
* pair rows past the default cap (600 beads within 5 of each other) grown
  and built again, an explicit cap overflowing reported as an error;
* the cutoff autotuner of the Python binding times every candidate that
  fits the box and returns the fastest.
"""
import numpy as np
import pytest

import bd_b200 as B
import oracle as O
import pme_oracle as P
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _prepared(flow, t, Nb=25, Nc=20, L=30.0, seed=31, **pme):
    x, y, z = B.random_chains(Nb, Nc, L, seed + t, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, mobility="pme", noise="philox",
                                **pme))
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    c.set_positions(x, y, z)
    c.set_time(t, t)
    c.update_lattice(t)
    c.calc_hi()
    return c, o, (x, y, z)


def _lab_cell(o, x, y, z, L):
    s = o.s
    if s.flow == 1:
        xl, yl = x * s.cth - y * s.sth, x * s.sth + y * s.cth
    else:
        xl, yl = x, y
    return np.stack([xl, yl, z], 1), P.reduced_cell(list(s.L1), list(s.L2), L)


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 3000), (1, 1000), (1, 7000)])
def test_pme_matches_cpu_model(flow, t):
    K, p, rc, alpha = 32, 6, 10.0, 0.35
    c, o, (x, y, z) = _prepared(flow, t, Nb=25, Nc=8, pme_grid=K, pme_order=p, pme_rc=rc,
                                pme_alpha=alpha)
    pos, H = _lab_cell(o, x, y, z, 30.0)
    v = np.random.default_rng(5).normal(size=(o.N, 3))
    ar = P.ref_alpha(t, o.s.tp, o.s.L2yp)
    ref = P.pme_apply(H, pos, v, K, p, alpha, rc, alpha_ref=ar)
    got = c.mobility_apply(v.reshape(-1)).reshape(o.N, 3)
    assert rel_err(got, ref) < 1e-11


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 3000), (1, 1000), (1, 4500)])
def test_pme_vs_dense_ewald(flow, t):
    c, o, (x, y, z) = _prepared(flow, t)
    Mf = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    v = np.random.default_rng(3).normal(size=3 * o.N)
    err = rel_err(c.mobility_apply(v), Mf @ v)
    assert err < 2e-5, err


@pytest.mark.parametrize("flow,t", [(0, 6000), (1, 8000)])
def test_pme_vs_converged_ewald(flow, t):
    c, o, (x, y, z) = _prepared(flow, t, Nb=25, Nc=8)
    pos, H = _lab_cell(o, x, y, z, 30.0)
    v = np.random.default_rng(4).normal(size=(o.N, 3))
    ar = P.ref_alpha(t, o.s.tp, o.s.L2yp)
    ref = P.ewald_apply(H, pos, v, alpha=ar, tol_exp=30.0) - v @ P.self_offdiag(H, ar, 30.0).T
    err = rel_err(c.mobility_apply(v.reshape(-1)), ref.reshape(-1))
    assert err < 1e-5, err


@pytest.mark.parametrize("flow", [0, 1])
def test_pme_lanczos_vs_eigh(flow):
    c, o, (x, y, z) = _prepared(flow, 500)
    Mf = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    zz = np.random.default_rng(7).normal(size=3 * o.N)
    ref, lmin = O.sqrtm_apply(Mf, zz)
    assert lmin > 0
    got, iters = c.lanczos_sqrt(zz)
    assert 2 <= iters < 80
    assert rel_err(got, ref) < 3e-5, (iters, rel_err(got, ref))
    # the operator the solve sees: symmetric to rounding
    Mp = np.stack([c.mobility_apply(e) for e in np.eye(3 * o.N)], 1)
    assert rel_err(Mp, Mp.T) < 1e-12
    ref_p, lmin_p = O.sqrtm_apply(0.5 * (Mp + Mp.T), zz)
    assert lmin_p > 0
    assert rel_err(got, ref_p) < 1e-6, (iters, rel_err(got, ref_p))


@pytest.mark.parametrize("flow,t", [(0, 3000), (1, 4500)])
def test_pme_fp32_storage(flow, t):
    c64, o, (x, y, z) = _prepared(flow, t)
    c32, _, _ = _prepared(flow, t, precision="fp32")
    v = np.random.default_rng(9).normal(size=3 * o.N)
    ref = c64.mobility_apply(v)
    err = rel_err(c32.mobility_apply(v), ref)
    assert err < 1e-5, err
    Mf = O.full_mobility(o.calc_hi_ewald(x, y, z), o.N)
    assert rel_err(c32.mobility_apply(v), Mf @ v) < 2e-5


@pytest.mark.parametrize("precision,K,tol", [("fp32", 64, 2e-6), ("fp32", 40, 2e-6),
                                             ("fp64", 64, 1e-12)])
@pytest.mark.parametrize("flow,t", [(0, 3000), (1, 7000)])
def test_block_product_matches_single(precision, K, tol, flow, t):
    c, o, _ = _prepared(flow, t, precision=precision, pme_grid=K, noise_block=8)
    V = np.random.default_rng(7).normal(size=(7, 3 * o.N))
    got = c.mobility_apply_block(V)
    errs = [rel_err(got[r], c.mobility_apply(V[r])) for r in range(7)]
    assert max(errs) < tol, errs
    if precision == "fp32":
        c64, _, _ = _prepared(flow, t, pme_grid=K)
        errs = [rel_err(got[r], c64.mobility_apply(V[r])) for r in range(7)]
        assert max(errs) < 1e-5, errs


def _clustered(precision="fp64", **pme):
    """600 beads uniform within 5 of the centre of a box of 30: with cutoff
    12.9 each has 599 others within the cutoff, past the default cap of 512
    pairs per row."""
    Nb, Nc, L = 25, 24, 30.0
    r = np.random.default_rng(17).uniform(-5.0, 5.0, size=(3, Nb * Nc))
    c = B.Context(B.make_params(0, Nb, Nc, L, 0.2, 5e-4, mobility="pme", noise="philox",
                                precision=precision, pme_grid=32, pme_order=6, pme_rc=12.9,
                                pme_alpha=0.3, **pme))
    c.set_positions(*r)
    c.set_time(0, 0)
    c.update_lattice(0)
    return c, r


def test_pair_rows_grow_past_the_default_cap():
    """With the default cap the rows that overflow it are grown and built
    again: the product matches the CPU model of the same discretisation, and
    the FP32 block product (its own pair data) matches the FP64 product."""
    c, r = _clustered()
    c.calc_hi()
    o = O.Oracle(0, 25, 24, 30.0, 0.2, 5e-4)
    o.lattice(0)
    pos, H = _lab_cell(o, r[0], r[1], r[2], 30.0)
    v = np.random.default_rng(5).normal(size=(600, 3))
    ref = P.pme_apply(H, pos, v, 32, 6, 0.3, 12.9, alpha_ref=P.ref_alpha(0, o.s.tp, o.s.L2yp))
    got = c.mobility_apply(v.reshape(-1)).reshape(600, 3)
    assert rel_err(got, ref) < 1e-11
    c32, _ = _clustered("fp32", noise_block=4)
    c32.calc_hi()
    V = np.random.default_rng(6).normal(size=(4, 1800))
    out = c32.mobility_apply_block(V)
    assert max(rel_err(out[k], c.mobility_apply(V[k])) for k in range(4)) < 1e-5


def test_explicit_pair_cap_overflow_is_an_error():
    c, _ = _clustered(pme_max_pairs=64)
    with pytest.raises(B.BDError, match="overflow"):
        c.calc_hi()
        c.mobility_apply(np.ones(1800))


def test_cutoff_autotuner_times_every_candidate_that_fits():
    """bd_b200.autotune_pme_cutoff times the block product of each candidate
    cutoff up to 0.43 L (20 is skipped in a box of 30) on the device and
    returns the fastest; the contexts it was given are closed."""
    made = []

    def make(rc):
        c, _, _ = _prepared(0, 0, precision="fp32", pme_rc=rc, noise_block=4)
        made.append(c)
        return c

    best, times = B.autotune_pme_cutoff(make, 30.0, 4, candidates=(10.0, 12.5, 20.0))
    assert sorted(times) == [10.0, 12.5]
    assert best == min(times, key=times.get)
    assert all(v > 0 for v in times.values())
    assert len(made) == 2 and all(c.h is None for c in made)


def test_pme_rejects_dense_download():
    c, o, _ = _prepared(0, 0, Nb=10, Nc=4)
    with pytest.raises(B.BDError):
        c.mobility()


@pytest.mark.parametrize("flow", [0, 1])
def test_pme_krylov_steps_stable(flow):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = B.random_chains(Nb, Nc, L, 41, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    q = B.random_charges(Nb, Nc, 0.5, 43)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.01, 5e-4, mobility="pme", noise="philox",
                                MStep=100, Ncharges=len(q), shear_kappas_override=1, srpy=10))
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
