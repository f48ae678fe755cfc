"""CPU checks of the Ewald Coulomb model (oracle/coulomb_oracle.py): the sum
does not depend on the split parameter (forces and energy at two splits
agree to 1e-9 relative), and the force is minus the gradient of the energy
(central differences, 1e-6 relative)."""
import numpy as np

import coulomb_oracle as C
from conftest import rel_err


def _system(N=40, L=12.0, seed=2):
    r = np.random.default_rng(seed)
    H = np.array([[L, 0.3 * L, 0], [0, L, 0], [0, 0, L]])
    pos = r.uniform(0, L, (N, 3))
    q = np.where(np.arange(N) % 2 == 0, 1.0, -1.0)
    q[0] = 1.0  # a net charge exercises the background term
    return H, pos, q


def test_split_independent():
    H, pos, q = _system()
    F1, E1 = C.ewald_coulomb(H, pos, q, 2.0, alpha=0.35)
    F2, E2 = C.ewald_coulomb(H, pos, q, 2.0, alpha=0.6)
    assert rel_err(F1, F2) < 1e-9 and abs(E1 - E2) < 1e-9 * abs(E1)


def test_force_is_gradient():
    H, pos, q = _system(N=12)
    F, _ = C.ewald_coulomb(H, pos, q, 2.0)
    h = 1e-5
    fd = np.zeros(6)
    for n, (i, a) in enumerate([(0, 0), (3, 1), (5, 2), (7, 0), (9, 1), (11, 2)]):
        p, m = pos.copy(), pos.copy()
        p[i, a] += h
        m[i, a] -= h
        fd[n] = -(C.ewald_coulomb(H, p, q, 2.0)[1] - C.ewald_coulomb(H, m, q, 2.0)[1]) / (2 * h)
    got = np.array([F[0, 0], F[3, 1], F[5, 2], F[7, 0], F[9, 1], F[11, 2]])
    assert rel_err(got, fd) < 1e-6
