"""Parallel (independent-set) charge-hop sweep on the GPU against
oracle/hop_oracle.py, its CPU restatement with the same cells, colours,
Philox draws and Debye-Hueckel energies: final charge sites, the per-trial
log (accepted / target / move kind) and the occupancy flags agree exactly
(the energies differ only in summation order, so a decision could differ only
for a draw within round-off of its threshold).  No reference counterpart: the
reference's sequential sweep is covered bit-exactly by the parity tests."""
import numpy as np
import pytest

import bd_b200 as B
import hop_oracle as H
import oracle as O
import pme_oracle as P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flow,signed,seed", [(0, True, 5), (1, True, 6), (1, False, 7)])
def test_parallel_sweep_matches_model(flow, signed, seed):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    track = B.random_charges(Nb, Nc, 0.5, seed + 1)
    qk = np.where((track // Nb) % 2 == 0, 1.0, -1.0) if signed else np.ones(len(track))
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, noise="philox", hop="parallel",
                                hop_radius=6.0, philox_seed=1000 + seed, Ncharges=len(track),
                                barrier=0.5, barrier2=1.0))
    c.set_positions(x, y, z)
    c.set_charges(track)
    c.set_charge_values(qk)
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    px, py, pz = (np.array(a) for a in c.positions())
    _, _, flags0 = c.charges()
    c.charge_hop()
    tr, old, fl = c.charges()
    log = c.hop_log()
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    o.lattice(0)
    s = o.s
    Hc = P.reduced_cell(list(s.L1), list(s.L2), L)
    cth, sth = (s.cth, s.sth) if flow == 1 else (1.0, 0.0)
    tr_o, old_o, log_o, fl_o = H.parallel_sweep(o, px, py, pz, track, qk, flags0, Hc, cth, sth,
                                                6.0, 2.0, 1 / 5.0, 0.5, 1.0, 1000 + seed, 0)
    assert np.array_equal(log, log_o)
    assert np.array_equal(tr, tr_o)
    assert np.array_equal(fl, fl_o)
    moved = (log[:, 0] == 1).sum()
    assert moved > 0 and len(np.unique(tr)) == len(tr)
