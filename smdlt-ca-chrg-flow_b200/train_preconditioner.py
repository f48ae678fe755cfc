"""Train the learned Lanczos preconditioner on the GPU and save its parameters.

    python smdlt-ca-chrg-flow_b200/train_preconditioner.py --out mpnn_params.npy

Configurations are seeded synthetic bead-spring systems at the density of the
8000-bead extensional workload (chains of 100 beads, bond 2, no overlaps),
in shear and planar extension, some relaxed by a few hundred Brownian steps
so that they are consistent with the deforming lattice at later times.  The
mobility is the particle-mesh Ewald sum.  With --segment S > 1 (the
default, 10) the network learns bead blocks B applied on top of the segment
preconditioner L^-1 (G = B L^-1): each training step draws z ~ N(0, I),
forms A^-1/2 z for A = L^-1 M L^-T by Lanczos and takes one Adam step of the
library's own BF16 tensor-core kernels on (1/N) sum_i |B_i z_i - (A^-1/2 z)_i|^2;
with --segment 1 the targets are M^-1/2 z and B alone is the preconditioner.
The held-out Krylov iteration counts (plain, segment blocks, learned) are
printed as JSON.
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import bd_b200 as B  # noqa: E402


def configs(flow, Nb, Nc, L, seeds, relax_steps, edot, dt):
    """(x, y, z, t) in the frame the mobility build reads, PBC applied."""
    out = []
    for s in seeds:
        x, y, z = B.random_chains(Nb, Nc, L, s, bond=2.0, min_sep=2.0)
        x, y = B.lab_frame(flow, x, y)
        c = B.Context(B.make_params(flow, Nb, Nc, L, edot, dt, mobility="pme", precision="fp32",
                                    noise="philox", philox_seed=s, shear_kappas_override=1,
                                    srpy=25))
        c.set_positions(x, y, z)
        c.set_time(0, 0)
        c.update_lattice(0)
        c.transform_coords()
        c.apply_pbc()
        c.build_neighbors()
        c.inverse_coords()
        t = 0
        if relax_steps:
            c.step_lanczos(0, relax_steps, False)
            t = relax_steps
            c.set_time(t, t)
            c.update_lattice(t)
            c.transform_coords()
            c.apply_pbc()
        else:
            c.transform_coords()
        out.append(tuple(np.array(a) for a in c.positions()) + (t,))
        c.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "mpnn_params.npy"))
    ap.add_argument("--configs", type=int, default=24)
    ap.add_argument("--steps-per-config", type=int, default=30)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--segment", type=int, default=10)
    a = ap.parse_args()
    Nb, Nc, L, dt = 100, 20, 60.0 * 0.25 ** (1 / 3), 5e-4
    edot = 2.0 / (175.0 * 2 ** (3 * 0.588))
    train = []
    for k in range(a.configs):
        flow = k % 2
        train += configs(flow, Nb, Nc, L, [a.seed + k], 200 if k % 3 == 2 else 0, edot, dt)
    ctxs = {f: B.Context(B.make_params(f, Nb, Nc, L, edot, dt, mobility="pme", precision="fp64",
                                       noise="philox")) for f in (0, 1)}
    if a.segment > 1:
        for c in ctxs.values():
            c.set_preconditioner("segment", a.segment)
    # one context per flow (each keeps its own Adam moments and step count);
    # the parameters pass between them after every configuration
    w = B.mpnn_init(a.seed)
    losses, steps = [], {0: 0, 1: 0}
    for k, cfg in enumerate(train):
        f = k % 2
        c = ctxs[f]
        c.mpnn_set_params(w)
        ls = B.train_preconditioner(c, [cfg], a.steps_per_config, a.lr, a.seed + 1000 + k,
                                    steps[f])
        steps[f] += a.steps_per_config
        w = c.mpnn_params()
        losses.append(float(np.mean(ls)))
    step = steps[0] + steps[1]
    np.save(a.out, w)
    # held out: Krylov iterations of sqrt(M) z with and without the network
    res = []
    for flow in (0, 1):
        c = ctxs[flow]
        c.mpnn_set_params(w)
        for (x, y, z, t) in configs(flow, Nb, Nc, L, [a.seed + 500 + flow], 0, edot, dt):
            c.set_positions(x, y, z)
            c.set_time(t, t)
            c.update_lattice(t)
            c.build_neighbors()
            c.set_preconditioner("none")
            c.calc_hi()
            zz = np.random.default_rng(7).normal(size=3 * c.N)
            _, plain = c.lanczos_sqrt(zz)
            c.set_preconditioner("segment", max(a.segment, 1))
            _, seg = c.lanczos_sqrt(zz)
            c.set_preconditioner("learned", a.segment)
            _, learned = c.lanczos_sqrt(zz)
            res.append(dict(flow=flow, plain=plain, segment=seg, learned=learned))
            c.set_preconditioner("none")
    print(json.dumps({"loss_per_config": losses, "held_out_iterations": res,
                      "params": a.out, "steps": step}))


if __name__ == "__main__":
    main()
