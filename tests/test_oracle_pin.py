"""Pins the oracle (the C restatement in oracle/bd_oracle.c) to the reference.

The golden fixtures were produced by the unmodified reference routines
(tests/golden/make_golden.py, run against oracle/_ref/).  Comparisons that the
reference decides by comparisons or integer arithmetic (lattice, wrapped
positions, neighbour rows, random streams, charge-hop outcomes) must be
bit-exact; floating-point sums agree to 1e-12 relative (both are FP64 with the
same operation order; only library-function rounding may differ).
"""
import json

import numpy as np
import pytest

import oracle as O
from conftest import rel_err

FLOWS = [("shear", 0), ("ext", 1)]


def make_oracle(g, **over):
    d = json.loads(str(g["system"]))
    d.update(over)
    flow = d.pop("flow")
    return O.Oracle(flow, **d), flow


@pytest.mark.parametrize("name,flow", FLOWS)
def test_lattice(golden, name, flow):
    g = golden(f"lattice_{name}")
    o, _ = make_oracle(g)
    assert o.s.tp == int(g["tp"])
    bins = g["bins"]
    assert (o.s.nbx, o.s.nby, o.s.nbz, o.s.nhx, o.s.nhy, o.s.nhz, o.s.nbins) == tuple(bins)
    for t, lat in zip(g["t"], g["lattice"]):
        o.lattice(int(t))
        s = o.s
        mine = [s.L1[0], s.L1[1], s.L2[0], s.L2[1], s.L1xp, s.L1yp, s.L2xp, s.L2yp, s.detL, s.tp]
        assert np.array_equal(np.array(mine), lat), t


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900", "shear_bend"])
def test_forces_and_verlet(golden, case):
    g = golden(f"forces_{case}")
    o, flow = make_oracle(g, kappab=float(g["kappab"]))
    t = int(g["t"])
    x, y, z = (g[k].copy() for k in ("x0", "y0", "z0"))
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    assert np.array_equal(x, g["px"]) and np.array_equal(y, g["py"]) and np.array_equal(z, g["pz"])
    cnt, rows = o.verlet(x, y, z, 64)
    assert np.array_equal(cnt, g["nb_count"])
    for i in range(len(cnt)):
        assert np.array_equal(rows[i, :cnt[i]], g["nb_rows"][i, :cnt[i]])
    f, st = np.zeros((3, o.N)), np.zeros(3)
    assert o.bond(x, y, z, f, st) == 0
    assert rel_err(f, g["f_bond"]) < 1e-12 and rel_err(st, g["s_bond"]) < 1e-12
    f, st = np.zeros((3, o.N)), np.zeros(3)
    o.ev(x, y, z, cnt, rows, f, st)
    assert rel_err(f, g["f_ev"]) < 1e-12 and rel_err(st, g["s_ev"]) < 1e-12
    q = np.zeros(o.N)
    q[g["charges"]] = 1.0
    f = np.zeros((3, o.N))
    o.coulomb(x, y, z, q, f)
    assert rel_err(f, g["f_coul"]) < 1e-12


def upper_and_diag(M, N):
    """The entries calcHI defines: upper 3x3 blocks and diagonal-block diagonals."""
    B = M.reshape(N, N, 3, 3)  # block (i, j) at 9 N i + 9 j, row-major 3x3
    iu = np.triu_indices(N, 1)
    d = np.array([[B[i, i, a, a] for a in range(3)] for i in range(N)])
    return B[iu], d


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900"])
def test_calc_hi_update_hi(golden, case):
    import make_golden as MG
    g = golden(f"hi_{case}")
    o, flow = make_oracle(g)
    t, N = int(g["t"]), o.N
    x, y, z = (g[k].copy() for k in ("x0", "y0", "z0"))
    o.lattice(t)
    if flow == 1:
        o.rotate(x, y, 0)
    o.apply_pbc(x, y, z)
    grid = MG.grid_table(o.s.nt_avg, o.s.nbins, int(g["grid_seed"]))
    M = o.calc_hi(x, y, z, grid)
    ub, db = upper_and_diag(M, N)
    ur, dr = upper_and_diag(g["M"], N)
    assert rel_err(ub, ur) < 1e-12 and rel_err(db, dr) < 1e-13
    beta, C = MG.tea_table(o.s.Nb, 20, int(g["grid_seed"]) + 1)
    sb = min(int(np.floor(float(g["strain"]) / 0.5)), 20)
    Ct = np.ascontiguousarray(np.tile(C[sb], o.s.Nc))
    dv = np.zeros((3, N))
    o.update_hi(x, y, z, dv, np.ascontiguousarray(g["F"]), g["R"], M, float(beta[sb]), Ct)
    for a, k in zip((x, y, z), ("ux", "uy", "uz")):
        assert rel_err(a, g[k]) < 1e-13
    assert rel_err(dv, g["dv"]) < 1e-12


@pytest.mark.parametrize("case", ["shear_0", "shear_2900", "ext_0", "ext_2900"])
def test_update_fd(golden, case):
    g = golden(f"fd_{case}")
    o, flow = make_oracle(g)
    x, y, z = (g[k].copy() for k in ("x0", "y0", "z0"))
    o.lattice(int(g["t"]))
    dv = np.zeros((3, o.N))
    o.update_fd(x, y, z, dv, np.ascontiguousarray(g["F"]), g["R"])
    assert np.array_equal(x, g["ux"]) and np.array_equal(y, g["uy"]) and np.array_equal(z, g["uz"])


@pytest.mark.parametrize("name,flow", FLOWS)
def test_ran1_gasdev_streams(golden, name, flow):
    g = golden(f"noise_{name}")
    rng = O.fresh_rng(int(g["seed"]))
    u = np.array([O.lib().bdo_ran1(rng) for _ in range(100)], np.float32)
    assert np.array_equal(u, g["u100"])
    R = np.zeros(len(g["R1"]))
    O.lib().bdo_noise(rng, R, len(R))
    assert np.array_equal(R, g["R1"])
    O.lib().bdo_noise(rng, R, len(R))
    assert np.array_equal(R, g["R2"])
    tail = np.array([O.lib().bdo_ran1(rng) for _ in range(5)], np.float32)
    assert np.array_equal(tail, g["tail"])


@pytest.mark.parametrize("name,flow", FLOWS)
def test_charge_hop_sequence(golden, name, flow):
    g = golden(f"hop_{name}")
    o, _ = make_oracle(g, barrier=float(g["barrier"]), barrier2=float(g["barrier2"]),
                       MStep=int(g["MStep"]))
    x, y, z = (g[k].copy() for k in ("px", "py", "pz"))
    track = g["charges"].astype(np.int32).copy()
    old = track.copy()
    rng = O.fresh_rng(int(g["seed"]))
    total = 0
    for s in range(len(g["tracks"])):
        o.lattice(s * 100)
        nacc, _ = o.charge_hop(x, y, z, track, old, rng)
        total += nacc
        assert np.array_equal(track, g["tracks"][s]), s
        assert np.array_equal(old, g["olds"][s]), s
    c = g["counters"][-1]
    assert total == c[0] + c[1] + c[3] + c[4]
    tail = np.array([O.lib().bdo_ran1(rng) for _ in range(3)], np.float32)
    assert np.array_equal(tail, g["tail"])


@pytest.mark.parametrize("name,flow", FLOWS)
def test_full_reference_steps(golden, name, flow):
    import make_golden as MG
    g = golden(f"step_{name}")
    o, _ = make_oracle(g, barrier=float(g["barrier"]), barrier2=float(g["barrier2"]),
                       MStep=int(g["MStep"]))
    grid = MG.grid_table(o.s.nt_avg, o.s.nbins, int(g["grid_seed"]))
    beta, C = MG.tea_table(o.s.Nb, 20, int(g["grid_seed"]) + 1)
    sim = O.OracleSim(o, g["x0"], g["y0"], g["z0"], g["charges"], MG.SEED0[flow], grid, beta, C,
                      MStep=int(g["MStep"]))
    sim.begin_iteration(0)
    for t in range(int(g["nsteps"])):
        sim.step_hi(t, True)
        assert rel_err(np.stack([sim.x, sim.y, sim.z]), g["pos"][t]) < 1e-12, t
        assert np.array_equal(sim.track, g["tracks"][t]), t


@pytest.mark.parametrize("name,flow", FLOWS)
def test_grid_table(golden, name, flow):
    """The restated gridHI against the reference's gridHI program."""
    g = golden(f"grid_{name}")
    geom = g["geom"]  # L box_volume bsx bsy bsz dt tp
    o = O.Oracle(flow, 8, 6, float(geom[0]), float(g["edot"]), 5e-4, nt_avg=int(g["nt_avg"]),
                 bin_size=float(g["bin_size"]))
    D, bins = o.grid(float(geom[5]), float(geom[1]))
    assert np.array_equal(bins, g["bins"])
    assert np.array_equal(D, g["D"])
