"""Ensembles of replicas (bd_batch_*) and the grid autotuner (no reference
counterpart).

* Replicas of different sizes and flows advanced concurrently by a batch end
  bit-identical to the same replicas advanced one after another (dense exact
  Ewald mobility, FP64: every reduction has a fixed order);
* with the particle-mesh mobility (atomic spreading) they agree to 1e-9
  relative after a few steps, also with noise blocks (every replica solving
  several steps' displacements per Krylov run while the others capture and
  replay their own iterations);
* the autotuned grid is a 2^a 3^b 5^c size within [1.29 L, 1.25 x 1.29 L].
"""
import numpy as np
import pytest

import bd_b200 as B

pytestmark = pytest.mark.gpu

SYSTEMS = [(0, 25, 8, 20.0), (1, 20, 15, 24.0), (1, 25, 20, 30.0)]


def _ctx(flow, Nb, Nc, L, seed, mobility, precision, noise_block=1):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    q = B.random_charges(Nb, Nc, 0.5, seed + 1)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.01, 5e-4, mobility=mobility,
                                precision=precision, noise="philox", philox_seed=seed,
                                Ncharges=len(q), shear_kappas_override=1, MStep=5, srpy=5,
                                noise_block=noise_block))
    c.set_positions(x, y, z)
    c.set_charges(q)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.inverse_coords()
    return c


def _run(mobility, precision, nsteps, noise_block=1):
    solo = []
    for k, (f, Nb, Nc, L) in enumerate(SYSTEMS):
        c = _ctx(f, Nb, Nc, L, 50 + k, mobility, precision, noise_block)
        c.step_lanczos(0, nsteps, True)
        solo.append(np.stack(c.positions()))
    ctxs = [_ctx(f, Nb, Nc, L, 50 + k, mobility, precision, noise_block)
            for k, (f, Nb, Nc, L) in enumerate(SYSTEMS)]
    b = B.Batch(ctxs)
    b.step_lanczos(0, nsteps, True)
    b.close()
    return solo, [np.stack(c.positions()) for c in ctxs]


def test_batch_matches_sequential_dense():
    solo, batch = _run("ewald", "fp64", 12)
    for a, b in zip(solo, batch):
        assert np.array_equal(a, b)


def test_batch_matches_sequential_pme():
    solo, batch = _run("pme", "fp64", 4)
    for a, b in zip(solo, batch):
        assert np.linalg.norm(a - b) <= 1e-9 * np.linalg.norm(a)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_noise_blocks(precision):
    solo, batch = _run("pme", precision, 12, noise_block=4)
    tol = 1e-9 if precision == "fp64" else 1e-5
    for a, b in zip(solo, batch):
        assert np.linalg.norm(a - b) <= tol * np.linalg.norm(a)


@pytest.mark.parametrize("L", [22.0, 60.0, 110.0])
def test_autotuned_grid(L):
    K = B.autotune_pme_grid(L, "fp32")
    r = K
    for f in (2, 3, 5):
        while r % f == 0:
            r //= f
    assert r == 1 and np.ceil(1.29 * L) <= K <= np.ceil(1.25 * np.ceil(1.29 * L))
