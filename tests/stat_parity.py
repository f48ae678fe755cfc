"""Long-run statistics of the Brownian-dynamics step, compared between two
runs that share the initial configuration and differ in the method (or the
implementation) and in the noise stream.

The statistics (the reference's own observables: chain extension as printed
by printExt, polymer stress from the virial accumulators of bondforce and
LJforce that printVisc reports, bead mean-squared displacement as calcMSD
computes it; shear/src/main26.c:925-974, 1866-1880, 2494-2637):

* end-to-end distance of every chain (unwrapped along the chain), averaged
  over the second half of the run: one value per chain, compared as
  distributions by the two-sample Kolmogorov-Smirnov test;
* the virial stress per step (tauxx, tauyy, tauxy), averaged over blocks of
  the second half: means compared in units of their combined standard error
  (blocks longer than the stress correlation time);
* the mean-squared displacement of the beads along z (the neutral direction
  of both flows, unaffected by the flow and the lattice deformation), from
  positions unwrapped with period L every sample: compared in units of its
  standard error over chains.

Pairs compared:

* north: the headline path (FP32 particle-mesh products, learned
  preconditioner, noise blocks) against the plain FP64 method (pme64), both on
  the GPU with the configs' physics;
* reference: the GPU's reference-mode step (bd_step_reference: hybrid dense
  mobility, CA-TEA noise, Debye-Hueckel, sequential hop, ran1) against the
  reference's own routines on the host (oracle/_ref), different ran1 seeds.

tests/test_gpu_stat_parity.py runs short versions; the long runs:

    python tests/stat_parity.py --pair north --workload c4 --steps 2000
    python tests/stat_parity.py --pair reference --workload c0 --steps 5000 --replicas 8
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "smdlt-ca-chrg-flow_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)


class Stats:
    """Accumulates the three statistics from samples taken every `every`
    steps (positions, unwrapped chain coordinates, stress accumulators)."""

    def __init__(self, N, Nb, Nc, L, every):
        self.N, self.Nb, self.Nc, self.L, self.every = N, Nb, Nc, L, every
        self.z0 = self.zu = self.zp = None
        self.ree = []
        self.tau = []

    def sample(self, z, unwrapped, tau_per_step):
        z = np.asarray(z, float)
        if self.zu is None:
            self.z0, self.zu = z.copy(), z.copy()
        else:
            dz = z - self.zp
            self.zu += dz - self.L * np.rint(dz / self.L)
        self.zp = z.copy()
        p = np.asarray(unwrapped).reshape(3, self.Nc, self.Nb)
        self.ree.append(np.linalg.norm(p[:, :, -1] - p[:, :, 0], axis=0))
        self.tau.append(np.asarray(tau_per_step, float))

    def result(self):
        h = len(self.ree) // 2
        ree = np.mean(self.ree[h:], axis=0)
        tau = np.array(self.tau[h:])
        msd_chain = ((self.zu - self.z0) ** 2).reshape(self.Nc, self.Nb).mean(1)
        return {"ree_per_chain": ree.tolist(), "tau_blocks": tau.tolist(),
                "msd_z_per_chain": msd_chain.tolist(), "samples": len(self.ree),
                "steps": len(self.ree) * self.every}


def compare(a, b):
    """KS p-value of the per-chain extension; z-scores of the mean stress
    components and of the mean z-MSD."""
    from scipy.stats import ks_2samp
    out = {"ree_mean": [float(np.mean(a["ree_per_chain"])), float(np.mean(b["ree_per_chain"]))],
           "ree_ks_p": float(ks_2samp(a["ree_per_chain"], b["ree_per_chain"]).pvalue)}
    ta, tb = np.array(a["tau_blocks"]), np.array(b["tau_blocks"])
    zt = []
    for k in range(3):
        ma, mb = ta[:, k].mean(), tb[:, k].mean()
        se = math.sqrt(ta[:, k].var(ddof=1) / len(ta) + tb[:, k].var(ddof=1) / len(tb))
        zt.append(float((ma - mb) / se) if se > 0 else 0.0)
    out["tau_mean"] = [ta.mean(0).tolist(), tb.mean(0).tolist()]
    out["tau_z"] = zt
    ma, mb = np.array(a["msd_z_per_chain"]), np.array(b["msd_z_per_chain"])
    se = math.sqrt(ma.var(ddof=1) / len(ma) + mb.var(ddof=1) / len(mb))
    out["msd_z"] = [float(ma.mean()), float(mb.mean())]
    out["msd_z_z"] = float((ma.mean() - mb.mean()) / se) if se > 0 else 0.0
    return out


def run_gpu(workload, path, steps, every, noise_seed, config_seed=1000, noise_block=10,
            reference_step=False):
    """One GPU run of `path` (bench.PATHS) from the seeded configuration."""
    import bench
    w = bench.WORKLOADS[workload]
    N = w["Nb"] * w["Nc"]
    pp = bench.PATHS[path]
    extra = {}
    if pp["mobility"] == "pme":
        extra = dict(noise_block=noise_block if path != "pme64" else 1,
                     pme_rc=w.get("pme_rc", 12.1))
    if reference_step:
        c = bench.build_context(w, config_seed, path, device_noise="ran1",
                                noise_seed=noise_seed, **extra)
    else:
        c = bench.build_context(w, config_seed, path, noise_seed=noise_seed, **extra)
    step = c.step_reference if pp["step"] == "reference" else c.step_lanczos
    st = Stats(N, w["Nb"], w["Nc"], w["L"], every)
    st.sample(c.positions()[2], c.chain_props()[0], np.zeros(3))
    t0 = time.time()
    for tb in range(0, steps, every):
        acc = np.zeros(3)
        for t in range(tb, tb + every):
            step(t, 1, True)
            acc += c.stress()  # the virial of this step (reset at each step's start)
        st.sample(c.positions()[2], c.chain_props()[0], acc / every)
    r = st.result()
    r["wall_s"] = time.time() - t0
    r["lanczos"] = c.lanczos_stats()
    c.close()
    return r


def _ref_worker(args):
    workload, steps, every, seed, config_seed, threads = args
    import bench
    import oracle as O
    w = bench.WORKLOADS[workload]
    N = w["Nb"] * w["Nc"]
    x, y, z, q, beta, C = bench.synth_inputs(w, config_seed)
    kw = bench.force_params(w)
    kw.pop("srpy")
    ref = O.RefSim(w["flow"], w["Nb"], w["Nc"], w["L"], bench.edot_of(w), w["dt"],
                   Ncharges=len(q), threads=threads, seed=seed, **kw)
    G = bench.grid_table_host(w)
    for nt in range(bench.COMMON["nt_avg"]):
        ref.set_grid(nt, np.ascontiguousarray(G[nt]))
    for sb in range(21):
        ref.set_tea(sb, float(beta[sb]), np.ascontiguousarray(C[sb]))
    ref.set_pos(x, y, z)
    ref.set_charges(q, len(q))
    ref.set_tstart(0)
    ref.begin_iteration()

    def unwrapped():
        u = [np.zeros(N) for _ in range(3)]
        ref.lib.h_get_unwrapped(*u)
        return np.stack(u)

    def stress():
        s = np.zeros(3)
        ref.lib.h_get_stress(s)
        return s

    st = Stats(N, w["Nb"], w["Nc"], w["L"], every)
    st.sample(ref.pos()[2], unwrapped(), np.zeros(3))
    t0 = time.time()
    for tb in range(0, steps, every):
        acc = np.zeros(3)
        for t in range(tb, tb + every):
            s0 = stress()
            ref.step_hi(t, 1)
            acc += stress() - s0  # the reference accumulates until printVisc
        st.sample(ref.pos()[2], unwrapped(), acc / every)
    r = st.result()
    r["wall_s"] = time.time() - t0
    return r


def run_reference_host(workload, steps, every, seed, config_seed=1000, threads=None):
    """The reference's own routines (oracle/_ref) on the host, in a fresh
    process (its generator and state are process-global)."""
    import subprocess
    threads = threads or len(os.sched_getaffinity(0))
    args = json.dumps([workload, steps, every, seed, config_seed, threads])
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-worker", args],
                       capture_output=True, text=True, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def merge(runs):
    """Independent runs (different noise streams) as one sample: their
    chains and stress blocks side by side."""
    out = dict(runs[0])
    for key in ("ree_per_chain", "tau_blocks", "msd_z_per_chain"):
        out[key] = [x for r in runs for x in r[key]]
    out["wall_s"] = sum(r["wall_s"] for r in runs)
    out["runs"] = len(runs)
    return out


def run_pair(pair, workload, steps, every, replicas=1):
    """Both sides of a pair, each as `replicas` independent runs from the same
    configuration with different noise streams."""
    A, B = [], []
    for k in range(replicas):
        if pair == "north":
            A.append(run_gpu(workload, "pme32-learned", steps, every, noise_seed=11 + 100 * k))
            B.append(run_gpu(workload, "pme64", steps, every, noise_seed=22 + 100 * k))
        else:
            A.append(run_gpu(workload, "tea", steps, every, noise_seed=830062920 + 7919 * k,
                             reference_step=True))
            B.append(run_reference_host(workload, steps, every, seed=123456789 + 104729 * k))
    a, b = (A[0], B[0]) if replicas == 1 else (merge(A), merge(B))
    return a, b, compare(a, b)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pair", choices=["north", "reference"], default="north")
    ap.add_argument("--workload", default="c4")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--replicas", type=int, default=1,
                    help="independent noise streams per side, pooled")
    ap.add_argument("--out", default="")
    ap.add_argument("--ref-worker", default="")
    args = ap.parse_args()
    if args.ref_worker:
        # the host reference run of run_reference_host, in this fresh process;
        # the reference's own status lines go to stderr
        saved = os.dup(1)
        os.dup2(2, 1)
        r = _ref_worker(tuple(json.loads(args.ref_worker)))
        sys.stdout.flush()
        os.dup2(saved, 1)
        print(json.dumps(r))
        return
    a, b, cmp_ = run_pair(args.pair, args.workload, args.steps, args.every, args.replicas)
    res = {"pair": args.pair, "workload": args.workload, "steps": args.steps,
           "every": args.every, "replicas": args.replicas, "compare": cmp_,
           "wall_s": [a["wall_s"], b["wall_s"]],
           "lanczos": [a.get("lanczos"), b.get("lanczos")]}
    print(json.dumps(res))
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"summary": res, "a": a, "b": b}, f)


if __name__ == "__main__":
    main()
