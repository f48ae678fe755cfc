"""Lanczos iterations replayed from a captured CUDA graph give the results of
the same kernels launched one by one: bit-identical with the dense FP64
mobility (every reduction has a fixed order), 1e-12 with the particle-mesh
mobility (atomic spreading), with and without a preconditioner, and over
Brownian steps that rebuild the mobility (which drops and recaptures the
graph)."""
import numpy as np
import pytest

import bd_b200 as B

pytestmark = pytest.mark.gpu


def _ctx(mobility, flow=1, Nb=25, Nc=20, L=30.0, seed=3):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.05, 5e-4, mobility=mobility, noise="philox",
                                precision="fp64", shear_kappas_override=1, srpy=3))
    c.set_positions(x, y, z)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.calc_hi()
    return c


@pytest.mark.parametrize("mobility,tol", [("ewald", 0.0), ("pme", 1e-12)])
@pytest.mark.parametrize("precond", ["none", "segment"])
def test_graph_replay_matches_direct(mobility, tol, precond):
    z = np.random.default_rng(4).normal(size=3 * 500)
    out = []
    for graphs in (False, True):
        c = _ctx(mobility)
        c.enable_graphs(graphs)
        if precond != "none":
            c.set_preconditioner(precond, 5)
        a, it = c.lanczos_sqrt(z)
        b, it2 = c.lanczos_sqrt(z)  # second call replays the captured graph
        out.append((a, b, it, it2))
    (a0, b0, i0, j0), (a1, b1, i1, j1) = out
    assert i0 == i1 and j0 == j1
    for u, v in ((a0, a1), (b0, b1)):
        assert np.linalg.norm(u - v) <= tol * np.linalg.norm(u)


@pytest.mark.parametrize("mobility,tol", [("ewald", 0.0), ("pme", 1e-9)])
def test_graph_steps_match_direct(mobility, tol):
    res = []
    for graphs in (False, True):
        c = _ctx(mobility)
        c.enable_graphs(graphs)
        c.inverse_coords()
        c.step_lanczos(0, 8, False)
        res.append(np.stack(c.positions()))
    assert np.linalg.norm(res[0] - res[1]) <= tol * np.linalg.norm(res[0])
