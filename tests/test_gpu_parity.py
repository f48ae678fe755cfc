"""Parity of the CUDA path (through the C ABI) with the reference.

Each case runs one reference routine's replacement on the GPU on the inputs of
a golden fixture (produced by the reference itself) and compares:
  * bit-exact: lattice, wrapped positions, neighbour rows, ran1/gasdev
    streams, charge-hop tracks and the generator position after a sweep;
  * FP64 1e-10 relative (norm-wise): forces, virial, the mobility blocks,
    the TEA and free-draining displacements;
  * 1e-9 relative: positions after several full reference steps.
Larger systems are checked against the oracle (oracle/bd_oracle.c) on seeded
inputs at sizes the oracle finishes in seconds.
"""
import json

import numpy as np
import pytest

import bd_b200 as B
import make_golden as MG
import oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu
FLOWS = [("shear", 0), ("ext", 1)]
TOL = 1e-10


def ctx_for(g, **over):
    d = json.loads(str(g["system"]))
    d.update(over)
    flow = d.pop("flow")
    p = B.make_params(flow, d.pop("Nb"), d.pop("Nc"), d.pop("L"), d.pop("edot"), d.pop("dt"),
                      **d)
    return B.Context(p), flow


def upper_and_diag(M, N):
    Bk = M.reshape(N, N, 3, 3)
    iu = np.triu_indices(N, 1)
    d = np.array([[Bk[i, i, a, a] for a in range(3)] for i in range(N)])
    return Bk[iu], d


@pytest.mark.parametrize("name,flow", FLOWS)
def test_lattice(golden, name, flow):
    g = golden(f"lattice_{name}")
    c, _ = ctx_for(g)
    assert np.array_equal(c.grid_shape(), g["bins"])
    for t, lat in zip(g["t"], g["lattice"]):
        c.update_lattice(int(t))
        assert np.array_equal(c.lattice(), lat), t


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900", "shear_bend"])
def test_pbc_neighbors_forces(golden, case):
    g = golden(f"forces_{case}")
    c, flow = ctx_for(g, kappab=float(g["kappab"]))
    t = int(g["t"])
    c.set_positions(g["x0"], g["y0"], g["z0"])
    c.set_charges(g["charges"])
    c.set_time(t)
    c.update_lattice(t)
    if flow == 1:
        c.transform_coords()
    c.apply_pbc()
    x, y, z = c.positions()
    assert np.array_equal(x, g["px"]) and np.array_equal(y, g["py"]) and np.array_equal(z, g["pz"])
    c.build_neighbors()
    cnt, rows = c.neighbors(64)
    assert np.array_equal(cnt, g["nb_count"])
    for i in range(len(cnt)):
        assert np.array_equal(rows[i, :cnt[i]], g["nb_rows"][i, :cnt[i]])
    c.reset_force()
    c.bond_force()
    assert rel_err(c.forces(), g["f_bond"]) < TOL and rel_err(c.stress(), g["s_bond"]) < TOL
    c.reset_force()
    c.ev_force()
    assert rel_err(c.forces(), g["f_ev"]) < TOL and rel_err(c.stress(), g["s_ev"]) < TOL
    c.reset_force()
    c.coulomb_force()
    assert rel_err(c.forces(), g["f_coul"]) < TOL


def _tea(c, seed, Nb):
    beta, C = MG.tea_table(Nb, 20, seed)
    for sb in range(21):
        c.set_tea(sb, beta[sb], C[sb])


def _grid(c, seed):
    shape = c.grid_shape()
    G = MG.grid_table(c.p.nt_avg, int(shape[6]), seed)
    for nt in range(c.p.nt_avg):
        c.load_grid(nt, G[nt])


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900"])
def test_calc_hi_and_tea_update(golden, case):
    g = golden(f"hi_{case}")
    c, flow = ctx_for(g)
    N, t = c.N, int(g["t"])
    gseed = int(g["grid_seed"])
    _grid(c, gseed)
    _tea(c, gseed + 1, c.p.Nb)
    c.set_positions(g["x0"], g["y0"], g["z0"])
    c.set_time(t, t)
    c.update_lattice(t)
    if flow == 1:
        c.transform_coords()
    c.apply_pbc()
    c.calc_hi()
    ub, db = upper_and_diag(c.mobility(), N)
    ur, dr = upper_and_diag(g["M"], N)
    assert rel_err(ub, ur) < TOL and rel_err(db, dr) < TOL
    c.set_forces(*g["F"])
    c.set_noise(g["R"])
    c.update_hi()
    x, y, z = c.positions()
    for a, k in zip((x, y, z), ("ux", "uy", "uz")):
        assert rel_err(a, g[k]) < TOL
    assert rel_err(c.displacements(), g["dv"]) < TOL


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900"])
def test_update_fd(golden, case):
    g = golden(f"fd_{case}")
    c, flow = ctx_for(g)
    t = int(g["t"])
    c.set_positions(g["x0"], g["y0"], g["z0"])
    c.set_time(t)
    c.update_lattice(t)
    c.set_forces(*g["F"])
    c.set_noise(g["R"])
    c.update_fd()
    x, y, z = c.positions()
    for a, k in zip((x, y, z), ("ux", "uy", "uz")):
        assert rel_err(a, g[k]) < 1e-13


@pytest.mark.parametrize("name,flow", FLOWS)
def test_gasdev_stream(golden, name, flow):
    g = golden(f"noise_{name}")
    c, _ = ctx_for(g)
    # advance the device generator past the 100 uniforms the fixture drew first
    rng = O.fresh_rng(int(g["seed"]))
    for _ in range(100):
        O.lib().bdo_ran1(rng)
    st = B.Ran1State()
    st.idum, st.idum2, st.iy = rng.idum, rng.idum2, rng.iy
    for a in range(32):
        st.iv[a] = rng.iv[a]
    st.iset, st.gset = rng.iset, rng.gset
    c.set_rng(st)
    c.get_noise()
    assert np.array_equal(c.noise(), g["R1"])
    c.get_noise()
    assert np.array_equal(c.noise(), g["R2"])


@pytest.mark.parametrize("name,flow", FLOWS)
def test_charge_hop_sequence(golden, name, flow):
    g = golden(f"hop_{name}")
    c, _ = ctx_for(g, barrier=float(g["barrier"]), barrier2=float(g["barrier2"]),
                   MStep=int(g["MStep"]))
    c.set_positions(g["px"], g["py"], g["pz"])
    c.set_charges(g["charges"])
    c.update_lattice(0)
    for s in range(len(g["tracks"])):
        c.set_time(s * 100)
        c.update_lattice(s * 100)
        c.charge_hop()
        tr, old, fl = c.charges()
        assert np.array_equal(tr, g["tracks"][s]), s
        assert np.array_equal(old, g["olds"][s]), s
        assert fl.sum() == len(tr) and np.all(fl[tr] == 1)
    # the generator sits where the reference's does after the sweeps
    ref = O.fresh_rng(0)
    st = c.rng()
    ref.idum, ref.idum2, ref.iy = st.idum, st.idum2, st.iy
    for a in range(32):
        ref.iv[a] = st.iv[a]
    tail = np.array([O.lib().bdo_ran1(ref) for _ in range(3)], np.float32)
    assert np.array_equal(tail, g["tail"])


@pytest.mark.parametrize("name,flow", FLOWS)
def test_reference_steps(golden, name, flow):
    g = golden(f"step_{name}")
    c, _ = ctx_for(g, barrier=float(g["barrier"]), barrier2=float(g["barrier2"]),
                   MStep=int(g["MStep"]))
    gseed = int(g["grid_seed"])
    _grid(c, gseed)
    _tea(c, gseed + 1, c.p.Nb)
    c.set_positions(g["x0"], g["y0"], g["z0"])
    c.set_charges(g["charges"])
    # begin_iteration: lattice(tstart), [rotate], PBC, neighbour build, [rotate back]
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.inverse_coords()
    for t in range(int(g["nsteps"])):
        c.step_reference(t, 1, True)
        assert rel_err(np.stack(c.positions()), g["pos"][t]) < 1e-9, t
        assert np.array_equal(c.charges()[0], g["tracks"][t]), t


# ---- larger systems against the oracle --------------------------------------

def _system(flow, Nb, Nc, L, seed):
    x, y, z = B.random_chains(Nb, Nc, L, seed, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(flow, x, y)
    return x, y, z


@pytest.mark.parametrize("flow,Nb,Nc,L,t", [(0, 25, 20, 30.0, 0), (0, 25, 20, 30.0, 3000),
                                            (1, 50, 16, 36.0, 0), (1, 50, 16, 36.0, 3000)])
def test_forces_neighbors_vs_oracle(flow, Nb, Nc, L, t):
    x, y, z = _system(flow, Nb, Nc, L, 7 + t)
    q = B.random_charges(Nb, Nc, 0.5, 3 + t)
    kw = dict(spring="FENE", kappas=30.0, qmax=3.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4, **kw)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, **kw))
    c.set_positions(x, y, z)
    c.set_charges(q)
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    c.set_time(t)
    c.update_lattice(t)
    o.apply_pbc(x, y, z)
    if flow == 1:
        c.transform_coords()
    c.apply_pbc()
    gx, gy, gz = c.positions()
    assert np.array_equal(gx, x) and np.array_equal(gy, y) and np.array_equal(gz, z)
    cnt, rows = o.verlet(x, y, z, 128)
    c.build_neighbors()
    gc, gr = c.neighbors(128)
    assert np.array_equal(cnt, gc)
    assert all(np.array_equal(rows[i, :cnt[i]], gr[i, :cnt[i]]) for i in range(len(cnt)))
    f, st = np.zeros((3, o.N)), np.zeros(3)
    o.bond(x, y, z, f, st)
    o.ev(x, y, z, cnt, rows, f, st)
    qq = np.zeros(o.N)
    qq[q] = 1.0
    o.coulomb(x, y, z, qq, f)
    c.reset_force()
    c.bond_force()
    c.ev_force()
    c.coulomb_force()
    assert rel_err(c.forces(), f) < TOL and rel_err(c.stress(), st) < TOL


@pytest.mark.parametrize("flow,t", [(0, 0), (0, 3000), (1, 0), (1, 3000)])
def test_mobility_vs_oracle_n500(flow, t):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = _system(flow, Nb, Nc, L, 17 + t)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4))
    G = MG.grid_table(8, o.s.nbins, 99)
    for nt in range(8):
        c.load_grid(nt, G[nt])
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    c.set_positions(x, y, z)
    c.set_time(t, t)
    c.update_lattice(t)
    c.calc_hi()
    M = o.calc_hi(x, y, z, G)
    ub, db = upper_and_diag(c.mobility(), o.N)
    ur, dr = upper_and_diag(M, o.N)
    assert rel_err(ub, ur) < TOL and rel_err(db, dr) < TOL


@pytest.mark.parametrize("flow", [0, 1])
def test_charge_hop_vs_oracle_n500(flow):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = _system(flow, Nb, Nc, L, 23)
    q = B.random_charges(Nb, Nc, 0.5, 29)
    kw = dict(barrier=0.5, barrier2=0.8, MStep=1)
    o = O.Oracle(flow, Nb, Nc, L, 0.2, 5e-4, **kw)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.2, 5e-4, seed=12345, **kw))
    o.lattice(0)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    c.set_positions(x, y, z)
    c.set_charges(q)
    c.set_time(0)
    c.update_lattice(0)
    track, old = q.copy(), q.copy()
    rng = O.fresh_rng(12345)
    for sweep in range(2):
        o.lattice(sweep)
        nacc, log = o.charge_hop(x, y, z, track, old, rng)
        c.set_time(sweep)
        c.update_lattice(sweep)
        c.charge_hop()
        assert np.array_equal(c.hop_log(), log), sweep
        tr, od, _ = c.charges()
        assert np.array_equal(tr, track) and np.array_equal(od, old), sweep


@pytest.mark.parametrize("name,flow", FLOWS)
def test_grid_table_vs_reference(golden, name, flow):
    g = golden(f"grid_{name}")
    geom = g["geom"]
    c = B.Context(B.make_params(flow, 8, 6, float(geom[0]), float(g["edot"]), 1e-3,
                                nt_avg=int(g["nt_avg"]), bin_size=float(g["bin_size"]),
                                box_volume=float(geom[1])))
    c.build_grid(float(geom[5]))
    for nt in range(int(g["nt_avg"])):
        assert rel_err(c.grid(nt), g["D"][nt]) < TOL, nt


@pytest.mark.parametrize("flow", [0, 1])
def test_grid_table_vs_oracle_c1_geometry(flow):
    """Box 30 at the bench's strain rate, all 8 frames, against the oracle."""
    L, edot = 30.0, 3.37e-3
    o = O.Oracle(flow, 25, 20, L, edot, 5e-4, nt_avg=8, bin_size=2.0)
    D, bins = o.grid(0.001, L ** 3)
    c = B.Context(B.make_params(flow, 25, 20, L, edot, 5e-4, nt_avg=8, bin_size=2.0))
    c.build_grid(0.001)
    assert np.array_equal(c.grid_shape()[:7], bins[:7])
    for nt in range(8):
        assert rel_err(c.grid(nt), D[nt]) < TOL, nt
