"""The GPU paths without a reference counterpart, pinned to published
constants through the C ABI (the CPU oracles are pinned to the same constants
in test_published_pins.py).

* Ewald Coulomb (bd_coulomb_force / bd_coulomb_energy, particle-mesh
  reciprocal part): unit charges on a rock-salt lattice of nearest-neighbour
  distance s have the energy -(N/2) M lambda_B / s, M = 1.747564594633
  (NaCl), to 5e-6 relative (the particle-mesh reciprocal sum on the default
  grid; 1.4e-6 measured at spacing 1.6), and no force (every ion is a centre
  of symmetry).
* Particle-mesh RPY mobility (bd_mobility_apply, FP64): n^3 beads on a simple
  cubic lattice of spacing l, all pushed along x, move with the mobility of
  Hasimoto's cubic array, 1 - 2.837297 (a/l) + (4 pi/3)(a/l)^3, and with the
  converged Ewald sum of the oracle for the same lattice: to 3e-5 (under a
  uniform force every bead's particle-mesh error adds coherently: 1.6e-5
  measured at l = 10a on the default grid; the pairwise RPY sum's cubic term
  is 3.5e-6 off the exact Stokes value there).
"""
import math

import numpy as np
import pytest

import bd_b200 as B
import pme_oracle as P

pytestmark = pytest.mark.gpu

MADELUNG_NACL = 1.747564594633
HASIMOTO_SC = 2.837297


def _lattice(n, s):
    g = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    return (g + 0.5) * s


@pytest.mark.parametrize("n,s,lb", [(8, 2.0, 2.0), (10, 1.6, 1.0)])
def test_ewald_coulomb_madelung(n, s, lb):
    pos = _lattice(n, s)
    N = len(pos)
    idx = np.rint(pos / s - 0.5).astype(int)
    q = np.where(idx.sum(1) % 2 == 0, 1.0, -1.0)
    L = n * s
    c = B.Context(B.make_params(0, n, n * n, L, 0.2, 5e-4, coulomb="ewald", lambda_b=lb,
                                noise="philox", Ncharges=N))
    c.set_positions(pos[:, 0], pos[:, 1], pos[:, 2])
    track = np.arange(N, dtype=np.int32)
    c.set_charges(track)
    c.set_charge_values(q)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.reset_force()
    c.coulomb_force()
    E = c.coulomb_energy()["total"]
    want = -(N / 2) * MADELUNG_NACL * lb / s
    assert abs(E - want) < 5e-6 * abs(want), (E, want)
    f = np.stack(c.forces(), 1)
    assert np.abs(f).max() < 1e-5 * lb / s ** 2
    c.close()


@pytest.mark.parametrize("n,l", [(4, 10.0), (2, 20.0), (3, 14.0)])
def test_pme_mobility_hasimoto(n, l):
    pos = _lattice(n, l)
    N = len(pos)
    L = n * l
    c = B.Context(B.make_params(0, n, n * n, L, 0.2, 5e-4, mobility="pme", noise="philox"))
    c.set_positions(pos[:, 0], pos[:, 1], pos[:, 2])
    c.set_time(0, 0)
    c.update_lattice(0)
    c.calc_hi()
    v = np.tile([1.0, 0.0, 0.0], N)
    u = c.mobility_apply(v).reshape(N, 3)
    hasimoto = 1 - HASIMOTO_SC / l + (4 * math.pi / 3) / l ** 3
    ewald = P.ewald_apply(l * np.eye(3), np.zeros((1, 3)), np.array([[1.0, 0.0, 0.0]]))[0, 0]
    assert np.abs(u[:, 0] - hasimoto).max() < 3e-5, (u[:, 0].min(), u[:, 0].max(), hasimoto)
    assert np.abs(u[:, 0] - ewald).max() < 3e-5
    assert np.abs(u[:, 1:]).max() < 1e-6
    c.close()
