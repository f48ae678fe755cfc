"""Parallel (independent-set) charge-hop sweep on the GPU against
oracle/hop_oracle.py, its CPU restatement with the same cells, colours and
Philox draws: final charge sites, the per-trial log (accepted / target / move
kind) and the occupancy flags agree exactly.

* Debye-Hueckel energies: the energies differ only in summation order, so a
  decision could differ only for a draw within round-off of its threshold;
  the per-trial energies are reported (NaN exactly where a move was blocked).
* Ewald energies (coulomb = BD_COULOMB_EWALD, FP64): the GPU interpolates the
  reciprocal potential from its particle-mesh grid where the oracle sums
  k-space explicitly, so each trial's energy difference agrees to 1e-5 kT
  (the mesh's accuracy); decisions agree exactly on these seeds.

No reference counterpart: the reference's sequential sweep is covered
bit-exactly by the parity tests."""
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
    de = c.hop_energies()
    assert np.array_equal(np.isnan(de), log[:, 0] == 0)


@pytest.mark.parametrize("flow,t,seed", [(0, 0, 5), (0, 3000, 6), (1, 1500, 7), (1, 0, 8)])
def test_parallel_sweep_ewald_energies_match_model(flow, t, seed):
    Nb, Nc, L, R = 25, 20, 30.0, 6.0
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    track = B.random_charges(Nb, Nc, 0.5, seed + 1)
    qk = np.where((track // Nb) % 2 == 0, 1.0, -1.0)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, noise="philox", hop="parallel",
                                coulomb="ewald", hop_radius=R, philox_seed=2000 + seed,
                                Ncharges=len(track), barrier=0.5, barrier2=1.0))
    c.set_positions(x, y, z)
    c.set_charges(track)
    c.set_charge_values(qk)
    c.set_time(t, t)
    c.update_lattice(t)
    if flow == 1:
        c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    px, py, pz = (np.array(a) for a in c.positions())
    _, _, flags0 = c.charges()
    c.charge_hop()
    tr, old, fl = c.charges()
    log = c.hop_log()
    de = c.hop_energies()
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    o.lattice(t)
    s = o.s
    Hc = P.reduced_cell(list(s.L1), list(s.L2), L)
    cth, sth = (s.cth, s.sth) if flow == 1 else (1.0, 0.0)
    rc = min(10.0, 0.43 * L)
    ew = H.EwaldTerms(Hc, 3.5 / rc, rc, 2.0)
    tr_o, old_o, log_o, fl_o, dm, dx = H.parallel_sweep(
        o, px, py, pz, track, qk, flags0, Hc, cth, sth, R, 2.0, 1 / 5.0, 0.5, 1.0, 2000 + seed,
        0, ewald=ew)
    assert np.array_equal(log, log_o)
    assert np.array_equal(tr, tr_o)
    assert np.array_equal(fl, fl_o)
    ev = ~np.isnan(dm)
    assert np.array_equal(ev, ~np.isnan(de))
    assert np.abs(de[ev] - dm[ev]).max() < 1e-5, np.abs(de[ev] - dm[ev]).max()
    assert (log[:, 0] == 1).sum() > 0 and len(np.unique(tr)) == len(tr)
