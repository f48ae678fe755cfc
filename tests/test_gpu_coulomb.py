"""Ewald-summed Coulomb forces and energy on the GPU (no reference
counterpart; the reference's Debye-Hueckel path is covered by the parity
tests).  Against oracle/coulomb_oracle.py's converged Ewald sum on the same
lattice: forces 1e-5 and energy 1e-6 relative, for charge-balanced
polyanion/polycation chains (+-1) and for a net-charged system, in shear and
planar extension, at two points of the lattice period."""
import numpy as np
import pytest

import bd_b200 as B
import coulomb_oracle as CO
import oracle as O
import pme_oracle as P
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _run(flow, t, signed, Nb=25, Nc=20, L=30.0, seed=11):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    track = B.random_charges(Nb, Nc, 0.5, seed + 1)
    qk = np.where((track // Nb) % 2 == 0, 1.0, -1.0) if signed else np.ones(len(track))
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, coulomb="ewald", noise="philox",
                                Ncharges=len(track)))
    c.set_positions(x, y, z)
    c.set_charges(track)
    c.set_charge_values(qk)
    c.set_time(t, t)
    c.update_lattice(t)
    c.reset_force()
    c.coulomb_force()
    f = np.stack(c.forces(), 1)
    E = c.coulomb_energy()
    s = o.s
    if flow == 1:
        xl, yl = x * s.cth - y * s.sth, x * s.sth + y * s.cth
    else:
        xl, yl = x, y
    pos = np.stack([xl, yl, z], 1)[track]
    Fo, Eo = CO.ewald_coulomb(P.cell(list(s.L1), list(s.L2), L), pos, qk, 2.0)
    return f, track, Fo, E, Eo


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 2000), (1, 0), (1, 1500)])
def test_ewald_coulomb_balanced(flow, t):
    f, track, Fo, E, Eo = _run(flow, t, True)
    assert rel_err(f[track], Fo) < 1e-5
    mask = np.ones(len(f), bool)
    mask[track] = False
    assert np.all(f[mask] == 0)
    assert abs(E["total"] - Eo) < 1e-6 * abs(Eo)


def test_ewald_coulomb_net_charge():
    f, track, Fo, E, Eo = _run(0, 0, False)
    assert rel_err(f[track], Fo) < 1e-5
    assert abs(E["total"] - Eo) < 1e-6 * abs(Eo)
