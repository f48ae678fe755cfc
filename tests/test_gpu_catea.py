"""CA-TEA sampling on the GPU against the reference's own ewaldBin / CATEA
(oracle/_ref, compiled from the reference sources): eps and rowsum 1e-10
relative, the running beta / C sums and counts of CATEA 1e-10, and the
decomp file of printTEA's format read back."""
import os
import tempfile

import numpy as np
import pytest

import bd_b200 as B
import oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _pair(flow, t, Nb=25, Nc=8, L=20.0, seed=3):
    if not O.ref_available(flow):
        pytest.skip("reference library not built")
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    edot, dt = 0.05, 5e-4
    c = B.Context(B.make_params(flow, Nb, Nc, L, edot, dt))
    c.set_positions(x, y, z)
    c.set_time(t, t)
    c.update_lattice(t)
    r = O.RefSim(flow, Nb, Nc, L, edot, dt)
    r.set_t(t)
    r.update_lattice(t)
    r.set_pos(x, y, z)
    return c, r


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 7000), (1, 0), (1, 5200)])
def test_ewald_bin_matches_reference(flow, t):
    c, r = _pair(flow, t)
    eps, rs = c.ewald_bin()
    eps_r, rs_r = r.ewald_bin()
    assert abs(eps - eps_r) <= 1e-10 * abs(eps_r)
    assert rel_err(rs, rs_r) < 1e-10


@pytest.mark.parametrize("flow", [0, 1])
def test_catea_running_sums_and_decomp(flow):
    c, r = _pair(flow, 0)
    with tempfile.TemporaryDirectory() as d:
        for strain in (0.3, 0.7, 0.35):
            c.catea(strain)
            brun, crun, gw = r.catea(strain, os.path.join(d, "beta.txt"))
        n, b, Cc = c.catea_averages()
        assert np.array_equal(n, gw)
        nz = gw > 0
        assert rel_err(b[nz], brun[nz] / gw[nz]) < 1e-10
        assert rel_err(Cc[nz], crun[nz] / (8 * gw[nz][:, None])) < 1e-10
        path = os.path.join(d, "DC.txt")
        c.write_decomp(path, 123)
        lines = open(path).read().split("\n")
        assert lines[0] == "123"
        rows = [list(map(float, l.split())) for l in lines[1:] if l.strip()]
        k = 0
        for i in range(21):
            assert int(rows[k][0]) == i and int(rows[k][1]) == gw[i]
            assert abs(rows[k][2] - (b[i] if gw[i] else 0.0)) <= 1e-11 * max(1.0, abs(b[i]))
            k += 1 + 25
