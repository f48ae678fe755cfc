"""The project's oracles for the paths the reference does not have, pinned to
published constants (CPU; the GPU counterparts are in test_gpu_pins.py).

* Ewald Coulomb (oracle/coulomb_oracle.py): the rock-salt lattice, unit
  charges at unit nearest-neighbour distance, has the Madelung energy
  -M lambda_B / r0 per ion pair with M = 1.747564594633 (NaCl; e.g. Kittel,
  Introduction to Solid State Physics, ch. 3).  Checked on the 8-ion
  conventional cell and on a 216-ion supercell with another Ewald split.
* Ewald-summed RPY mobility (oracle/pme_oracle.py's ewald_apply, the
  converged sum the particle-mesh product is checked against): one sphere of
  radius a per cubic cell of side l, i.e. a simple cubic array dragged
  uniformly, has the mobility 1 - 2.837297 (a/l) + (4 pi/3)(a/l)^3 + ...
  of the isolated sphere (Hasimoto, J. Fluid Mech. 5, 317 (1959): drag
  1 / (1 - 1.7601 c^(1/3) + c ...) with c = (4 pi/3)(a/l)^3; the constant
  2.837297 as in Zick and Homsy, J. Fluid Mech. 115, 13 (1982)).  The
  pairwise RPY sum carries the leading periodic correction exactly; its
  cubic term differs from the exact Stokes solution's at 1e-3 of itself
  (about 3.5e-6 of the mobility at l = 10a), so the constant is pinned from
  a fit and the mobility to 5e-7 for l >= 20a.
"""
import math

import numpy as np

import coulomb_oracle as C
import pme_oracle as P

MADELUNG_NACL = 1.747564594633
HASIMOTO_SC = 2.837297


def _rocksalt(n):
    g = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    q = np.array([(-1.0) ** int(i + j + k) for i, j, k in g])
    return g, q


def test_coulomb_oracle_madelung_conventional_cell():
    pos, q = _rocksalt(2)
    F, E = C.ewald_coulomb(2.0 * np.eye(3), pos, q, 1.0)
    assert abs(-E / 4 - MADELUNG_NACL) < 1e-10
    assert np.abs(F).max() < 1e-10  # every ion at a centre of symmetry


def test_coulomb_oracle_madelung_supercell_other_split():
    pos, q = _rocksalt(6)
    lb = 2.0
    F, E = C.ewald_coulomb(6.0 * np.eye(3), pos, q, lb, alpha=0.9)
    assert abs(-E / (len(q) / 2) / lb - MADELUNG_NACL) < 1e-10
    assert np.abs(F).max() < 1e-10


def _self_mobility(l):
    return P.ewald_apply(l * np.eye(3), np.zeros((1, 3)), np.array([[1.0, 0.0, 0.0]]))[0]


def test_rpy_ewald_hasimoto_cubic_array():
    Ls = np.array([10.0, 14.0, 20.0, 28.0, 40.0, 56.0, 80.0])
    m = []
    for l in Ls:
        u = _self_mobility(l)
        assert abs(u[1]) < 1e-12 and abs(u[2]) < 1e-12
        m.append(u[0])
        if l >= 20:
            assert abs(u[0] - (1 - HASIMOTO_SC / l + (4 * math.pi / 3) / l ** 3)) < 5e-7, l
    c = (1 - np.array(m)) * Ls  # = 2.837297 - c3 / l^2 + ...
    c0, c3 = np.linalg.lstsq(np.stack([np.ones_like(Ls), -1 / Ls ** 2], 1), c, rcond=None)[0]
    assert abs(c0 - HASIMOTO_SC) < 1e-5, c0
    assert abs(c3 - 4 * math.pi / 3) < 1e-2, c3
