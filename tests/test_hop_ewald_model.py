"""The parallel charge-hop sweep's Ewald acceptance energies, on the CPU
(oracle/hop_oracle.py; the GPU sweep is checked against the same model in
test_gpu_hop_parallel.py).  No reference counterpart: the reference's sweep
uses Debye-Hueckel energies.

* The exact energy difference the oracle keeps beside the model (every term
  from the structure factor of the state the trial sees) equals the change of
  the full Ewald energy of oracle/coulomb_oracle.py (pinned to the NaCl
  Madelung constant) over each trial, on a sweep run as one cell (fully
  sequential, so the state of every trial is known), to 1e-6 kT (the
  real-space cutoff's erfc(3.5) per pair).
* The model the GPU evaluates (mesh potential of the colour's start, the
  moved charge's own term and the cell's earlier moves from the reciprocal
  pair term near the origin, lambda_B erf(beta r)/r + r^T Q r) stays within
  1e-3 kT of the exact difference on hop cells of 7.5 in a box of 30, for a
  cubic, a sheared and a KRBC-deformed lattice: the O(r^4 / L^5) rest of the
  periodic pair term over a cell's diagonal.  The rest shrinks with the box
  (cells of 15 in a box of 60: below 5e-4 kT).
"""
import numpy as np
import pytest

import bd_b200 as B
import coulomb_oracle as CO
import hop_oracle as H
import oracle as O
import pme_oracle as P


def _sweep(flow, t, R, L=30.0, Nb=25, Nc=8, seed=5):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    track = B.random_charges(Nb, Nc, 0.5, seed + 1)
    qk = np.where((track // Nb) % 2 == 0, 1.0, -1.0)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    o.lattice(t)
    s = o.s
    x, y, z = np.array(x), np.array(y), np.array(z)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    Hc = P.reduced_cell(list(s.L1), list(s.L2), L)
    cth, sth = (s.cth, s.sth) if flow == 1 else (1.0, 0.0)
    rc = min(10.0, 0.43 * L)
    beta = 3.5 / rc
    ew = H.EwaldTerms(Hc, beta, rc, 2.0)
    flags0 = np.zeros(Nb * Nc, np.int64)
    flags0[track] = 1
    out = H.parallel_sweep(o, x, y, z, track, qk, flags0, Hc, cth, sth, R, 2.0, 0.2, 0.5, 1.0,
                           1005, 0, ewald=ew)
    lab = np.stack([x * cth - y * sth, x * sth + y * cth, z], 1)
    return out, track, qk, lab, Hc, beta


def test_exact_difference_is_the_full_energy_change():
    (tr, old, log, fl, dm, dx), track, qk, lab, Hc, beta = _sweep(0, 3000, R=16.0)
    cur = np.array(track)
    n = 0
    for k in range(len(track)):
        if log[k, 0] == 0:
            continue
        t1 = cur.copy()
        t1[k] = log[k, 1]
        dE = (CO.ewald_coulomb(Hc, lab[t1], qk, 2.0, alpha=beta)[1]
              - CO.ewald_coulomb(Hc, lab[cur], qk, 2.0, alpha=beta)[1])
        assert abs(dE - dx[k]) < 1e-6, (k, dE, dx[k])
        n += 1
        if log[k, 0] == 1:
            cur = t1
        if n >= 12:
            break
    assert n >= 12


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 3000), (1, 1500)])
def test_model_within_bound_of_exact(flow, t):
    (tr, old, log, fl, dm, dx), *_ = _sweep(flow, t, R=6.0)
    ok = ~np.isnan(dm)
    assert ok.sum() > 40 and (log[:, 0] == 1).sum() > 10
    assert np.nanmax(np.abs(dm - dx)) < 1e-3


def test_model_error_shrinks_with_the_box():
    (tr, old, log, fl, dm, dx), *_ = _sweep(1, 1500, R=15.0, L=60.0, Nc=16)
    assert (~np.isnan(dm)).sum() > 40
    assert np.nanmax(np.abs(dm - dx)) < 5e-4
