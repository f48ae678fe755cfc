"""Generate the golden fixtures in this directory from the reference itself.

Each scenario runs the unmodified reference routines (compiled from the
reference's own sources into oracle/_ref/ by oracle/Makefile) in a fresh
process, because ran1/gasdev keep function-local static state.  Inputs are
seeded synthetic chains; the far-field lookup table is a seeded synthetic
symmetric table (the reference copies its entries verbatim), so only its seed
is stored.

    python tests/golden/make_golden.py            # all scenarios
    python tests/golden/make_golden.py --list

Requires oracle/_ref/libref_{shear,ext}.so (``make -C oracle ref``).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "smdlt-ca-chrg-flow_b200"))

# small systems: 6 chains x 8 beads in an 18^3 box
SYSTEMS = {
    0: dict(flow=0, Nb=8, Nc=6, L=18.0, edot=0.5, dt=5e-4, spring="Hookean", kappas=200.0,
            qmax=2.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0, nt_avg=8, bin_size=2.0),
    1: dict(flow=1, Nb=8, Nc=6, L=18.0, edot=0.5, dt=5e-4, spring="FENE", kappas=30.0,
            qmax=3.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0, nt_avg=8, bin_size=2.0),
}
SEED0 = {0: 830062920, 1: 981272199}


def grid_table(nt_avg, nbins, seed):
    """Seeded symmetric 3x3 tensors, nt_avg frames of nbins, row-major."""
    g = np.random.default_rng(seed).normal(scale=0.05, size=(nt_avg, nbins, 3, 3))
    g = 0.5 * (g + np.swapaxes(g, -1, -2))
    return np.ascontiguousarray(g.reshape(nt_avg, nbins * 9))


def tea_table(Nb, sbins, seed):
    r = np.random.default_rng(seed)
    beta = r.uniform(0.2, 0.9, sbins + 1)
    C = r.uniform(0.6, 1.0, (sbins + 1, 3 * Nb))
    return beta, C


def chains(sysd, seed):
    from bd_b200 import lab_frame, random_chains
    x, y, z = random_chains(sysd["Nb"], sysd["Nc"], sysd["L"], seed, bond=2.0, min_sep=1.7)
    x, y = lab_frame(sysd["flow"], x, y)
    return x, y, z


def charges(sysd, seed, n):
    r = np.random.default_rng(seed)
    return np.sort(r.choice(sysd["Nb"] * sysd["Nc"], size=n, replace=False)).astype(np.int32)


def new_ref(flow, **over):
    import oracle as O
    d = dict(SYSTEMS[flow])
    d.update(over)
    kw = {k: v for k, v in d.items() if k != "flow"}
    return O.RefSim(flow, seed=SEED0[flow], **kw), d


def sc_lattice(flow):
    ref, d = new_ref(flow)
    tp = int(ref.tp())
    ts = [0, 1, tp // 4, tp // 2, tp // 2 + 1, tp - 1, tp, 2 * tp + 17]
    out = []
    for t in ts:
        ref.update_lattice(t)
        out.append(ref.lattice())
    return dict(t=np.array(ts, np.int64), lattice=np.array(out), tp=np.array(tp),
                bins=ref.bins())


def sc_forces(flow, t, kappab=0.0):
    ref, d = new_ref(flow, kappab=kappab)
    x, y, z = chains(d, 11 + t)
    q = charges(d, 5 + t, 16)
    ref.set_pos(x, y, z)
    ref.set_charges(q, len(q))
    ref.update_lattice(t)
    ref.set_t(t)
    if flow == 1:
        ref.transform()
    ref.apply_pbc()
    px, py, pz = ref.pos()
    ref.verlet()
    cnt, rows = ref.verlet_rows(64)
    ref.reset_force()
    ref.bondforce()
    fb, sb = ref.force(), ref.stress()
    ref.reset_force()
    ref.ljforce()
    fe, se = ref.force(), ref.stress()
    ref.reset_force()
    ref.coulomb()
    fc = ref.force()
    return dict(x0=x, y0=y, z0=z, t=np.array(t), charges=q, kappab=np.array(kappab),
                px=px, py=py, pz=pz, nb_count=cnt, nb_rows=rows, f_bond=fb, s_bond=sb,
                f_ev=fe, s_ev=se, f_coul=fc)


def sc_hi(flow, t):
    ref, d = new_ref(flow)
    N = d["Nb"] * d["Nc"]
    x, y, z = chains(d, 21 + t)
    bins = ref.bins()
    gseed = 1000 + flow * 10 + (t % 7)
    G = grid_table(d["nt_avg"], int(bins[6]), gseed)
    for nt in range(d["nt_avg"]):
        ref.set_grid(nt, np.ascontiguousarray(G[nt]))
    beta, C = tea_table(d["Nb"], 20, gseed + 1)
    for sb in range(21):
        ref.set_tea(sb, float(beta[sb]), np.ascontiguousarray(C[sb]))
    ref.set_pos(x, y, z)
    ref.update_lattice(t)
    ref.set_t(t)
    ref.set_tstart(t)
    strain = t * d["dt"] * d["edot"]
    ref.set_strain(strain)
    if flow == 1:
        ref.transform()
    ref.apply_pbc()
    px, py, pz = ref.pos()
    ref.calc_hi()
    M = ref.M()
    # updateHI with fixed forces and noise (it recomputes M since t == tstart)
    r = np.random.default_rng(gseed + 2)
    F = r.normal(scale=3.0, size=(3, N))
    R = r.normal(size=3 * N)
    ref.set_force(*F)
    ref.set_noise(R)
    ref.update_hi()
    ux, uy, uz = ref.pos()
    dv = ref.dv()
    return dict(x0=x, y0=y, z0=z, t=np.array(t), grid_seed=np.array(gseed), strain=np.array(strain),
                px=px, py=py, pz=pz, M=M, F=F, R=R, ux=ux, uy=uy, uz=uz, dv=dv)


def sc_fd(flow, t):
    ref, d = new_ref(flow)
    N = d["Nb"] * d["Nc"]
    x, y, z = chains(d, 31 + t)
    ref.set_pos(x, y, z)
    ref.update_lattice(t)
    ref.set_t(t)
    r = np.random.default_rng(77 + t)
    F = r.normal(scale=3.0, size=(3, N))
    R = r.normal(size=3 * N)
    ref.set_force(*F)
    ref.set_noise(R)
    ref.update_fd()
    ux, uy, uz = ref.pos()
    return dict(x0=x, y0=y, z0=z, t=np.array(t), F=F, R=R, ux=ux, uy=uy, uz=uz, dv=ref.dv())


def sc_noise(flow):
    ref, d = new_ref(flow)
    N = d["Nb"] * d["Nc"]
    u = np.array([ref.ran1() for _ in range(100)], np.float32)
    ref.gen_noise()
    R1 = np.zeros(3 * N)
    ref.lib.h_get_noise(R1)
    ref.gen_noise()
    R2 = np.zeros(3 * N)
    ref.lib.h_get_noise(R2)
    tail = np.array([ref.ran1() for _ in range(5)], np.float32)
    return dict(seed=np.array(SEED0[flow], np.int64), u100=u, R1=R1, R2=R2, tail=tail)


def sc_hop(flow, nsweep=3):
    ref, d = new_ref(flow, Ncharges=16, barrier=1.0, barrier2=1.5)
    x, y, z = chains(d, 41)
    q = charges(d, 43, 16)
    ref.set_pos(x, y, z)
    ref.set_charges(q, len(q))
    ref.update_lattice(0)
    ref.set_t(0)
    if flow == 1:
        ref.transform()
    ref.apply_pbc()
    px, py, pz = ref.pos()
    tracks, olds, cnts = [], [], []
    for s in range(nsweep):
        ref.set_t(s * 100)
        ref.charge_hop()
        tr, old, fl = ref.charges(len(q))
        tracks.append(tr)
        olds.append(old)
        c = np.zeros(6, np.int32)
        ref.lib.h_hop_counters(c)
        cnts.append(c)
    tail = np.array([ref.ran1() for _ in range(3)], np.float32)
    return dict(x0=x, y0=y, z0=z, charges=q, px=px, py=py, pz=pz, seed=np.array(SEED0[flow]),
                barrier=np.array(1.0), barrier2=np.array(1.5), tracks=np.array(tracks),
                olds=np.array(olds), counters=np.array(cnts), tail=tail, MStep=np.array(100))


def sc_step(flow, nsteps=4):
    ref, d = new_ref(flow, Ncharges=16, MStep=2, barrier=1.0, barrier2=1.5)
    N = d["Nb"] * d["Nc"]
    x, y, z = chains(d, 51)
    q = charges(d, 53, 16)
    bins = ref.bins()
    gseed = 2000 + flow
    G = grid_table(d["nt_avg"], int(bins[6]), gseed)
    for nt in range(d["nt_avg"]):
        ref.set_grid(nt, np.ascontiguousarray(G[nt]))
    beta, C = tea_table(d["Nb"], 20, gseed + 1)
    for sb in range(21):
        ref.set_tea(sb, float(beta[sb]), np.ascontiguousarray(C[sb]))
    ref.set_pos(x, y, z)
    ref.set_charges(q, len(q))
    ref.set_tstart(0)
    ref.begin_iteration()
    pos, tracks = [], []
    for t in range(nsteps):
        ref.step_hi(t, 1)
        pos.append(np.stack(ref.pos()))
        tracks.append(ref.charges(len(q))[0])
    return dict(x0=x, y0=y, z0=z, charges=q, grid_seed=np.array(gseed), MStep=np.array(2),
                barrier=np.array(1.0), barrier2=np.array(1.5), pos=np.array(pos),
                tracks=np.array(tracks), nsteps=np.array(nsteps))


def sc_grid(flow):
    """gridHI's table for a small box (2 lattice frames), from the reference's
    own gridHI main run in a scratch directory."""
    import tempfile
    import oracle as O
    c_norm, edot = 0.6, 0.5
    D, bins, geom = O.ref_grid(flow, 8, 6, c_norm, edot, 2, 2.0, tempfile.mkdtemp())
    return dict(D=D, bins=bins, geom=geom, c_norm=np.array(c_norm), edot=np.array(edot),
                nt_avg=np.array(2), bin_size=np.array(2.0))


SCENARIOS = {}
for f in (0, 1):
    fl = "shear" if f == 0 else "ext"
    SCENARIOS[f"lattice_{fl}"] = (sc_lattice, (f,))
    SCENARIOS[f"noise_{fl}"] = (sc_noise, (f,))
    SCENARIOS[f"hop_{fl}"] = (sc_hop, (f,))
    SCENARIOS[f"step_{fl}"] = (sc_step, (f,))
    SCENARIOS[f"grid_{fl}"] = (sc_grid, (f,))
    for t in (0, 2900):
        SCENARIOS[f"forces_{fl}_{t}"] = (sc_forces, (f, t))
        SCENARIOS[f"hi_{fl}_{t}"] = (sc_hi, (f, t))
        SCENARIOS[f"fd_{fl}_{t}"] = (sc_fd, (f, t))
SCENARIOS["forces_shear_bend"] = (sc_forces, (0, 100, 5.0))


def run_one(name):
    fn, args = SCENARIOS[name]
    out = fn(*args)
    flow = args[0]
    meta = dict(SYSTEMS[flow])
    out["system"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def main():
    if "--list" in sys.argv:
        print("\n".join(SCENARIOS))
        return
    if len(sys.argv) > 2 and sys.argv[1] == "--one":
        run_one(sys.argv[2])
        return
    names = [a for a in sys.argv[1:] if not a.startswith("-")] or list(SCENARIOS)
    for n in names:
        # one process per scenario: the reference's generator state is static
        subprocess.run([sys.executable, __file__, "--one", n], check=True,
                       stdout=subprocess.DEVNULL)
        print("wrote", n)


if __name__ == "__main__":
    main()
