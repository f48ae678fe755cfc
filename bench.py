#!/usr/bin/env python
"""Throughput benchmark of the Brownian-dynamics step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1|c1s|c2|c3|c0] [--path ...] [--noise-block B]
                    [--pme-rc RC] [--pme-grid K] [--segment S] [--compare 0|1]

A "step" is one pass of the hydrodynamic step loop over the whole system:
lattice update, periodic wrap, neighbour check (and rebuild when due),
spring + excluded-volume + Coulomb forces, Brownian noise, mobility rebuild
every srpy=100 steps, Brownian displacement, and a charge-hop sweep every
MStep=100 steps.  The metric is bead-steps/s, whole-job (sum over GPUs).

Default workload (c3): planar extension with Kraynik-Reinelt boundaries,
500 chains x 100 beads (50 000 beads), box 110a, Wi = 3, dt = 5e-4, FENE k=30
Q0=3, WCA, 50% charged, charge hop every 100 steps (c1: 80 x 100 beads in a
box of 60a at Wi = 2).  Inputs are seeded synthetic chains.  The default path
(pme32-learned) computes the Ewald-summed Rotne-Prager-Yamakawa mobility by
smooth particle-mesh Ewald (FP32 grids; the cutoff, and with it the grid by
the library's accuracy rule, picked by bd_b200.autotune_pme_cutoff as the
fastest product on this GPU, reported in config) and the Brownian
displacement sqrt(M) z by a preconditioned
Lanczos solve at tolerance 1e-6 (learned bead blocks on 10-bead segment
blocks), the displacements of 10 consecutive steps solved by one multi-vector
Krylov run (noise blocks of 10 steps, which tile the rebuild period).  --compare 1 also times the plain FP64 method
(pme64, no preconditioner) on the same grid, with one solve per step and with
the same noise blocks, and the unpreconditioned FP32 path (pme32, same noise
blocks); --errors 1 reports the per-result error of the path
against pme64 on the same configuration.  The rebuild (every 100 steps) and
the sweep (every 100 steps) are timed on the device once each and carried at
their frequency in every figure (breakdown.amortised).

--impl reference times the reference's own CPU code (compiled from its sources
into oracle/_ref/) on this host's cores; every part of its value is measured
(a workload too large for its dense mobility is timed at 8000 beads).

One process per GPU (torchrun for N > 1); the path does not shard, so each
rank advances its own independent replica ("replicas only"); timing is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "smdlt-ca-chrg-flow_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "bead-steps/s on 1 B200 at 1e-6 Lanczos tol: learned-precond FP32 vs plain FP64"

# Relaxation time for Wi = edot * tau: the reference's notebooks quote
# tau = 175 for 50-bead chains; Zimm scaling tau ~ Nb^(3 nu), nu = 0.588.
def tau_estimate(Nb):
    return 175.0 * (Nb / 50.0) ** (3 * 0.588)


WORKLOADS = {
    "c1": dict(name="ext KRBC 80x100 beads (8000), box 60, Wi 2, 50% charged, hop/100 steps",
               flow=1, Nb=100, Nc=80, L=60.0, Wi=2.0, dt=5e-4, frac=0.5),
    # half of c1 at the same density, for profiling captures
    "c1s": dict(name="ext KRBC 40x100 beads (4000), box 47.6, Wi 2, 50% charged, hop/100 steps",
                flow=1, Nb=100, Nc=40, L=60.0 * 0.5 ** (1 / 3), Wi=2.0, dt=5e-4, frac=0.5),
    # the shear tree forces kappas = 200 (shear/src/main26.c:544); its own
    # Input.txt pairs that with a Hookean spring of rest length 2 and eps = 0.1
    "c3": dict(name="ext KRBC 500x100 beads (50000), box 110, Wi 3, 50% charged, hop/100 steps",
               flow=1, Nb=100, Nc=500, L=110.0, Wi=3.0, dt=5e-4, frac=0.5),
    # 64 replicas of seeded uneven sizes (see c2_replicas), one batch
    "c2": dict(name="64 replicas, 2k-20k beads each (chains 20-200 x 25-100), half shear half "
                    "KRBC, Wi uniform in [0.5, 5], 50% charged, hop/100 steps",
               flow=1, Nb=100, Nc=20, L=37.8, Wi=2.0, dt=5e-4, frac=0.5, ensemble=True),
    # config 4: semidilute charged solution in shear, 256^3 grid (the cutoff
    # that the grid rule pairs with it, 12.9 L / 256 = 8.82), hop every 50 steps
    "c4": dict(name="shear LE 2000x100 beads (200000), box 175, Wi 10, 50% charged, hop/50 steps",
               flow=0, Nb=100, Nc=2000, L=175.0, Wi=10.0, dt=5e-4, frac=0.5, pme_rc=8.82,
               force=dict(MStep=50)),
    "c0": dict(name="shear LE 20x25 beads (500), box 30, Wi 1, 50% charged, hop/100 steps",
               flow=0, Nb=25, Nc=20, L=30.0, Wi=1.0, dt=5e-4, frac=0.5,
               force=dict(spring="Hookean", kappas=200.0, qmax=2.0, epsilon=0.1)),
}
COMMON = dict(spring="FENE", kappas=30.0, qmax=3.0, epsilon=1.0, lambda_b=2.0, lambda_d=5.0,
              barrier=3.0, barrier2=3.0, MStep=100, nt_avg=8, bin_size=2.0, srpy=100)


def force_params(w):
    kw = dict(COMMON)
    kw.update(w.get("force", {}))
    return kw


def edot_of(w):
    return w["Wi"] / tau_estimate(w["Nb"])


def synth_inputs(w, seed):
    """Seeded chains, charges, far-field table and TEA parameters."""
    import bd_b200 as B
    x, y, z = B.random_chains(w["Nb"], w["Nc"], w["L"], seed, bond=2.0, min_sep=1.8)
    x, y = B.lab_frame(w["flow"], x, y)
    q = B.random_charges(w["Nb"], w["Nc"], w["frac"], seed + 1)
    r = np.random.default_rng(seed + 2)
    beta = r.uniform(0.3, 0.6, 21)
    C = r.uniform(0.8, 1.0, (21, 3 * w["Nb"]))
    return x, y, z, q, beta, C


def grid_table_host(w):
    """The far-field lookup table for the reference arm, computed on the host
    by the oracle's restatement of gridHI (pinned bit-exact to the reference's
    gridHI program); the GPU arm builds the same table with bd_build_grid."""
    import oracle as O
    o = O.Oracle(w["flow"], w["Nb"], w["Nc"], w["L"], edot_of(w), w["dt"],
                 nt_avg=COMMON["nt_avg"], bin_size=COMMON["bin_size"])
    D, _ = o.grid(0.001, w["L"] ** 3)
    return D


# ---------------------------------------------------------------------------
# the reference on the host cores


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class _StdoutToStderr:
    """Sends what C code writes to file descriptor 1 (the reference routines
    print status lines) to stderr, so stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def time_reference(w, steps, warmup, threads):
    with _StdoutToStderr():
        return _time_reference(w, steps, warmup, threads)


REF_MAX_BEADS = 8000  # largest system whose dense mobility (9 N^2 doubles, 4.6 GB) is timed


def _ref_sweep_seconds(O, w, Nc, seed, edot, threads, kw):
    """Wall time of one reference charge-hop sweep on a system with w's
    density, chain length and charge fraction but Nc chains."""
    ws = dict(w, Nc=Nc, L=w["L"] * (Nc / w["Nc"]) ** (1 / 3))
    xs, ys, zs, qs, _, _ = synth_inputs(ws, seed)
    refs = O.RefSim(w["flow"], ws["Nb"], ws["Nc"], ws["L"], edot, w["dt"], Ncharges=len(qs),
                    threads=threads, **kw)
    refs.set_pos(xs, ys, zs)
    refs.set_charges(qs, len(qs))
    refs.update_lattice(0)
    refs.set_t(0)
    if w["flow"] == 1:
        refs.transform()
    refs.apply_pbc()
    t0 = refs.wtime()
    refs.charge_hop()
    return refs.wtime() - t0, ws["Nb"] * ws["Nc"]


def _time_reference(w, steps, warmup, threads):
    """Per-step wall time of the reference's own routines (oracle/_ref) on the
    workload, every part measured:

    * plain hydrodynamic steps (updateHI with the dense mobility, forces,
      neighbour check) at full size;
    * the dense mobility rebuild (calcHI) at full size, timed once and
      amortised over its period of srpy steps;
    * the charge-hop sweep, which is O(Ncharges N^2) (about 17 min at 8000
      beads): timed at three smaller sizes of the same density, chain length
      and charge fraction, and a power law fitted to them.  The extrapolated
      sweep at full size is reported beside the measured value, not inside
      it, so the measured value leaves the sweep out (in the reference's
      favour).

    Systems above REF_MAX_BEADS (the 50 000-bead workload: a dense mobility of
    180 GB) cannot run; they are timed at the 8000-bead size of the same
    density and chain length, whose per-bead cost is lower (the dense product
    is O(N^2)), so the number is an upper bound on the reference's
    throughput at the larger size."""
    import oracle as O
    if not O.ref_available(w["flow"]):
        return None
    N_full = w["Nb"] * w["Nc"]
    at = w
    if N_full > REF_MAX_BEADS:
        Nc = REF_MAX_BEADS // w["Nb"]
        at = dict(w, Nc=Nc, L=w["L"] * (Nc / w["Nc"]) ** (1 / 3))
    edot = edot_of(at)
    N = at["Nb"] * at["Nc"]
    x, y, z, q, beta, C = synth_inputs(at, 1234)
    kw = force_params(at)
    kw.pop("srpy")
    ref = O.RefSim(at["flow"], at["Nb"], at["Nc"], at["L"], edot, at["dt"], Ncharges=len(q),
                   threads=threads, **kw)
    G = grid_table_host(at)
    for nt in range(COMMON["nt_avg"]):
        ref.set_grid(nt, np.ascontiguousarray(G[nt]))
    for sb in range(21):
        ref.set_tea(sb, float(beta[sb]), np.ascontiguousarray(C[sb]))
    ref.set_pos(x, y, z)
    ref.set_charges(q, len(q))
    ref.set_tstart(0)
    ref.begin_iteration()
    ref.step_hi(0, 0)  # t == tstart: builds M
    for t in range(1, 1 + warmup):
        ref.step_hi(t, 1)
    t0 = ref.wtime()
    for t in range(1 + warmup, 1 + warmup + steps):
        ref.step_hi(t, 1)
    t_plain = (ref.wtime() - t0) / steps
    t0 = ref.wtime()
    ref.calc_hi()
    t_hi = ref.wtime() - t0
    del ref
    # sweeps at 1/16, 1/8 and 1/4 of the chains; log-log least squares
    sizes, times = [], []
    for f in (16, 8, 4):
        ts, ns = _ref_sweep_seconds(O, at, max(1, at["Nc"] // f), 99 + f, edot, threads, kw)
        sizes.append(ns)
        times.append(ts)
    pw, lc = np.polyfit(np.log(sizes), np.log(times), 1)
    t_sweep = float(np.exp(lc) * N ** pw)
    per_step = t_plain + t_hi / COMMON["srpy"]
    per_step_x = per_step + t_sweep / COMMON["MStep"]
    where = (f"{N} beads" if at is w else
             f"{N} beads (the {N_full}-bead system's dense mobility, 9 N^2 doubles = "
             f"{9 * 8 * N_full ** 2 / 1e9:.0f} GB, cannot be allocated; same density and chain "
             f"length, lower per-bead cost, so an upper bound on the reference's throughput "
             f"there)")
    sample = (f"reference routines on {threads} host threads at {where}: {steps} plain steps "
              f"({t_plain*1e3:.1f} ms each) + dense mobility rebuild ({t_hi:.2f} s, amortised "
              f"over {COMMON['srpy']} steps), all measured; the charge-hop sweep (not in the "
              f"value) timed at {sizes} beads ({', '.join('%.2f' % v for v in times)} s), "
              f"fitted t ~ N^{pw:.2f}, extrapolated to {t_sweep:.0f} s at {N} beads")
    return dict(per_step=per_step, value=N / per_step, sample=sample, threads=threads,
                beads=N, value_with_extrapolated_sweep=N / per_step_x,
                components={"plain_step_s": t_plain, "mobility_build_s": t_hi,
                            "hop_sweep_sizes": sizes, "hop_sweep_s": times,
                            "hop_sweep_exponent": float(pw),
                            "hop_sweep_s_extrapolated": t_sweep,
                            "measured_at_beads": N, "workload_beads": N_full})


# ---------------------------------------------------------------------------
# clocks


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out = ""

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in (self.out or "").splitlines():
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our path


PATHS = {
    # north-star Brownian step: exact Ewald RPY mobility, Lanczos sqrt(M) z at
    # tol 1e-6 with FP64 orthogonalisation; mobility tiles stored in FP32
    # (products accumulated in FP64) or FP64
    "lanczos32": dict(mobility="ewald", precision="fp32", step="lanczos", bytes_per_block=24),
    "lanczos64": dict(mobility="ewald", precision="fp64", step="lanczos", bytes_per_block=48),
    # The particle-mesh paths run the configs' own physics ("north"): chains
    # alternately polyanion / polycation (charges -1 / +1 on the seeded half of
    # each chain's beads), Coulomb by Ewald summation, and the parallel
    # independent-set charge-hop sweep on Philox draws, FENE k = 30 in both
    # flows (the shear tree's forced k = 200 is a reference quirk, kept by
    # the reference-physics paths).  The dense-tile paths
    # keep the reference's (Debye-Hueckel, unsigned charges, sequential sweep).
    # the same Ewald sum applied matrix-free by smooth particle-mesh Ewald
    # (B-spline order 8; grid and real-space cutoff from --pme-rc / --pme-grid)
    "pme64": dict(mobility="pme", precision="fp64", step="lanczos", bytes_per_block=None,
                  physics="north"),
    # the same in FP32 storage (grids, FFTs, influence, pair tensors) with FP64
    # accumulation of the interpolation and pair sums
    "pme32": dict(mobility="pme", precision="fp32", step="lanczos", bytes_per_block=None,
                  physics="north"),
    # FP32 particle-mesh products with a preconditioned Krylov solve: segment
    # blocks (Cholesky of the free-space RPY mobility of 10 consecutive
    # beads), or those with the learned per-bead blocks on top (parameters
    # from smdlt-ca-chrg-flow_b200/mpnn_params.npy, made by
    # train_preconditioner.py)
    "pme32-seg": dict(mobility="pme", precision="fp32", step="lanczos", bytes_per_block=None,
                      precond="segment", physics="north"),
    "pme32-learned": dict(mobility="pme", precision="fp32", step="lanczos", bytes_per_block=None,
                          precond="learned", physics="north"),
    # the reference's own algorithm: hybrid mobility + CA-TEA displacement
    "tea": dict(mobility="hybrid", precision="fp64", step="reference", bytes_per_block=48),
}


def c2_replicas(seed=20261203, n=64):
    """Seeded replica set of config 2: chain counts 20-200, chain lengths 25,
    50, 75 or 100, 2000-20000 beads, alternately shear and extension, Wi
    uniform in [0.5, 5], box from the density of the 8000-bead workload."""
    r = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        Nc, Nb = int(r.integers(20, 201)), int(r.choice([25, 50, 75, 100]))
        if not 2000 <= Nb * Nc <= 20000:
            continue
        L = (Nb * Nc / (8000 / 60.0 ** 3)) ** (1 / 3)
        out.append(dict(name="replica", flow=len(out) % 2, Nb=Nb, Nc=Nc, L=L,
                        Wi=float(r.uniform(0.5, 5.0)), dt=5e-4, frac=0.5))
    return out


SEGMENT = [10]  # beads per preconditioner segment (--segment)


def build_context(w, seed, path="lanczos32", device_noise="philox", noise_seed=None, **extra):
    """A context on w's seeded synthetic configuration (seed), stepping path;
    the noise stream is keyed by noise_seed (default: seed)."""
    import bd_b200 as B
    edot = edot_of(w)
    x, y, z, q, beta, C = synth_inputs(w, seed)
    pp = PATHS[path]
    north = pp.get("physics") == "north"
    if device_noise == "ran1" and noise_seed is not None:
        extra.setdefault("seed", noise_seed)
    if pp["mobility"] == "pme":
        extra.setdefault("lanczos_max", 400)  # the plain method needs ~200 at 200 000 beads
    p = B.make_params(w["flow"], w["Nb"], w["Nc"], w["L"], edot, w["dt"], Ncharges=len(q),
                      noise=device_noise,
                      philox_seed=seed if noise_seed is None else noise_seed,
                      mobility=pp["mobility"],
                      precision=pp["precision"], lanczos_tol=1e-6,
                      coulomb="ewald" if north else "dh",
                      hop="parallel" if north else "sequential",
                      shear_kappas_override=1 if north else 0, **extra, **force_params(w))
    c = B.Context(p)
    if pp["mobility"] == "hybrid":
        c.build_grid(0.001)
    for sb in range(21):
        c.set_tea(sb, beta[sb], C[sb])
    c.set_positions(x, y, z)
    c.set_charges(q)
    if north:
        c.set_charge_values(np.where((q // w["Nb"]) % 2 == 0, -1.0, 1.0))
    c.set_time(0, 0)
    c.update_lattice(0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.inverse_coords()
    if pp.get("precond") == "segment":
        c.set_preconditioner("segment", SEGMENT[0] if w["Nb"] % SEGMENT[0] == 0 else 5)
    elif pp.get("precond") == "learned":
        c.mpnn_set_params(np.load(os.path.join(PKG, "mpnn_params.npy")))
        c.set_preconditioner("learned", SEGMENT[0] if w["Nb"] % SEGMENT[0] == 0 else 5)
    return c


# DRAM bytes (read + write, cold cache) of one block product, summed over its
# kernels from ncu captures of the bench's own command
# (profiles/launches_pme32-learned_c3.md); keyed by (beads, grid, cutoff,
# right-hand sides per product)
PRODUCT_TRAFFIC = {(50000, 100, 14.5, 10): 2.1933e9, (50000, 108, 13.6, 10): 2.6445e9}


def ranks_max(values, dist):
    """Element-wise maximum over the ranks (the slowest rank's device
    times); the values themselves without a process group."""
    if not dist:
        return [float(v) for v in values]
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def rank0_choice(choice, dist):
    """Rank 0's list of picks (the autotuned cutoff) on every rank."""
    if dist:
        dist.broadcast_object_list(choice, src=0)
    return choice


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measure(w, path, K, W, rank, dist, e2e_steps, noise_block=1, pme_rc=10.0, pme_grid=0):
    """Times K steps of one path after W warm-up steps; returns a dict."""
    import torch
    N = w["Nb"] * w["Nc"]
    pp = PATHS[path]
    nb = noise_block if pp["mobility"] == "pme" else 1
    extra = (dict(noise_block=nb, pme_rc=pme_rc, pme_grid=pme_grid)
             if pp["mobility"] == "pme" else {})
    c = build_context(w, 1000 + rank, path, **extra)
    step = c.step_lanczos if pp["step"] == "lanczos" else c.step_reference
    step(0, W, True)
    # noise blocks solved during the warm-up are dropped, so the timed steps
    # pay for every block they use (and the e2e loop below likewise)
    c.noise_block_release()
    c.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    lan0 = c.lanczos_stats()
    pre0 = c.precond_stats()
    blk0 = c.noise_block_stats()
    # step-level events only: per-product events would put the noise blocks'
    # Krylov loop back on the host (the products are timed in a pass below)
    c.profile(2)
    n0 = c.launches()
    dev = int(os.environ.get("LOCAL_RANK", 0))
    with ClockSampler(dev) as clk:
        step(W, K, True)
        c.sync()
    launches = c.launches() - n0
    prof = {k: c.profile_read(getattr(c, "PROF_" + k)) for k in
            ("STEP", "MATVEC", "HI_BUILD", "HOP", "FORCES", "BLOCK")}
    c.profile(False)
    lan1 = c.lanczos_stats()
    pre1 = c.precond_stats()
    blk1 = c.noise_block_stats()
    step_ms = prof["STEP"][0]
    # end to end through the C ABI with pinned host buffers: upload the
    # positions, one step, download the positions, every step
    Ke = max(1, min(K, e2e_steps))
    hb = [torch.empty(N, dtype=torch.float64, pin_memory=True).numpy() for _ in range(3)]
    for a, b in zip(hb, c.positions()):
        a[:] = b
    c.noise_block_release()
    c.sync()
    t0 = time.perf_counter()
    for t in range(W + K, W + K + Ke):
        c.set_positions(*hb)
        step(t, 1, True)
        for a, b in zip(hb, c.positions()):
            a[:] = b
    e2e_s = time.perf_counter() - t0
    # the periodic parts: a mobility rebuild every srpy steps and a charge-hop
    # sweep every MStep steps.  A window shorter than their period holds none
    # (or one, over-weighted), so one of each is timed on the device here, at
    # the next step that has both, and every timed figure carries them at
    # their own frequency (amortise below)
    c.noise_block_release()
    tp = (W + K + Ke + 99) // 100 * 100
    c.set_time(tp, 0)
    c.update_lattice(tp)
    c.profile(True)
    ext = w["flow"] == 1
    if ext:
        c.transform_coords()
    c.apply_pbc()
    c.calc_hi()
    if c.p.Ncharges > 0:
        c.charge_hop()
    if ext:
        c.inverse_coords()
    c.sync()
    per = {k: c.profile_read(getattr(c, "PROF_" + k)) for k in ("HI_BUILD", "HOP")}
    c.profile(False)
    # the dominant kernel, timed: the products of one noise block, each between
    # CUDA events on the library's stream (this pass checks convergence on the
    # host; the product kernels are those of the timed steps)
    c.noise_block_release()
    c.profile(True)
    step(tp + 1, nb, False)
    c.sync()
    prof["BLOCK"] = c.profile_read(c.PROF_BLOCK)
    c.profile(False)
    t_build = per["HI_BUILD"][0] / max(per["HI_BUILD"][1], 1)
    t_sweep = per["HOP"][0] / max(per["HOP"][1], 1)
    srpy, mstep = COMMON["srpy"], force_params(w)["MStep"]

    def amortise(ms, t_first, n):
        # remove the rebuilds and sweeps that fell in steps [t_first, t_first + n)
        # and add n / period of each, at the times measured above
        nb = sum(1 for t in range(t_first, t_first + n) if t % srpy == 0)
        ns = sum(1 for t in range(t_first, t_first + n) if t % mstep == 0)
        return ms - nb * t_build - ns * t_sweep + n * (t_build / srpy + t_sweep / mstep)

    step_ms_raw = step_ms
    step_ms = amortise(step_ms, W, K)
    e2e_s = amortise(e2e_s * 1e3, W + K, Ke) / 1e3
    t_max, e2e_s = ranks_max([step_ms, e2e_s], dist)
    mv_ms, mv_n = prof["MATVEC"]
    if pp["mobility"] == "pme":
        # compulsory bytes of one particle-mesh product, s bytes per value:
        # bead vectors and weights 48 N (s/4) plus 8 passes over 3 grids
        # 96 K^3 (s/4)
        import bd_b200 as B
        Kg = pme_grid or B.pme_default_grid(w["L"], pme_rc)
        sb = 8 if pp["precision"] == "fp64" else 4
        alg_bytes = (48 * N + 96 * Kg ** 3) * sb / 4
    else:
        alg_bytes = pp["bytes_per_block"] * N * (N - 1) / 2 + 4 * 3 * N * 8
    avg_ms = mv_ms / max(mv_n, 1)
    iters = lan1["iterations"] - lan0["iterations"]
    calls = lan1["calls"] - lan0["calls"]
    # noise blocks: the dominant kernel is the product of a whole block (its
    # right-hand sides share the launches); its algorithmic bytes are those of
    # one product times the mean right-hand sides per block iteration
    bk = {k: blk1[k] - blk0[k] for k in blk1}
    bl_ms, bl_n = prof["BLOCK"]
    block = None
    if bk["iterations"] > 0 and bl_n > 0:
        rhs = bk["rhs_iterations"] / bk["iterations"]
        b_avg = bl_ms / bl_n
        block = dict(noise_block=nb, blocks=bk["blocks"], block_iterations=bk["iterations"],
                     rhs_per_iteration=rhs, block_iterations_per_step=bk["iterations"] / K,
                     product_ms=bl_ms, products=bl_n, avg_product_ms=b_avg,
                     alg_bytes=alg_bytes * rhs,
                     achieved_gbs=alg_bytes * rhs / (b_avg / 1e3) / 1e9)
    out = dict(path=path, t_max_ms=t_max, launches=launches, clocks=clk.summary(),
               e2e_s=e2e_s, e2e_steps=Ke, matvec_ms=mv_ms, matvec_launches=mv_n,
               matvec_avg_ms=avg_ms, alg_bytes=alg_bytes,
               achieved_gbs=alg_bytes / (avg_ms / 1e3) / 1e9 if mv_n else None,
               lanczos_iters_per_step=(iters / calls) if calls else None, block=block,
               lanczos_maxed=lan1["maxed"] - lan0["maxed"],
               precond_fallbacks=pre1["fallbacks"] - pre0["fallbacks"],
               precond_calls=pre1["calls"] - pre0["calls"],
               breakdown={"window_ms": step_ms_raw,
                          "window_mobility_builds": prof["HI_BUILD"][1],
                          "window_hop_sweeps": prof["HOP"][1],
                          "mobility_build_ms_each": t_build, "hop_sweep_ms_each": t_sweep,
                          "amortised": "window - its rebuilds and sweeps + K/%d rebuilds + "
                                       "K/%d sweeps at the times measured" % (srpy, mstep),
                          "steps_ms_amortised": step_ms,
                          "forces_ms": prof["FORCES"][0], "matvec_ms": mv_ms})
    c.close()
    return out


def measure_batch(path, K, W, e2e_steps, noise_block=1):
    """Times K steps of the c2 ensemble advanced as one batch (bd_batch_*)
    after W warm-up steps: device time bracketed by full synchronisation and
    CUDA events.  The particle-mesh cutoff is autotuned once, on the largest
    replica (the replicas share the bead density, which sets the balance of
    real-space pairs and transforms); each replica takes it, bounded by its
    box, with the grid from the accuracy rule."""
    import bd_b200 as B
    import torch
    reps = c2_replicas()
    pp = PATHS[path]
    ctxs, grids, tuned, rc = [], [], None, None
    if pp["mobility"] == "pme":
        big = max(reps, key=lambda w: w["Nb"] * w["Nc"])
        nr = max(noise_block, 2)

        def make(rcut):
            c = build_context(big, 5000, path, noise_block=nr, pme_rc=rcut)
            c.calc_hi()
            return c
        rc, times = B.autotune_pme_cutoff(make, big["L"], nr)
        tuned = {str(k): round(v, 4) for k, v in times.items()}
    for k, w in enumerate(reps):
        extra = {}
        if pp["mobility"] == "pme":
            extra["pme_rc"] = min(rc, 0.43 * w["L"])
            extra["pme_grid"] = B.pme_default_grid(w["L"], extra["pme_rc"])
            extra["noise_block"] = noise_block
        grids.append(extra.get("pme_grid", B.pme_default_grid(w["L"])))
        ctxs.append(build_context(w, 5000 + k, path, **extra))
    batch = B.Batch(ctxs)
    batch.step_lanczos(0, W, True)
    for c in ctxs:
        c.noise_block_release()
    torch.cuda.synchronize()
    lan0 = [c.lanczos_stats() for c in ctxs]
    for c in ctxs:
        c.profile(True)
    n0 = sum(c.launches() for c in ctxs)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", 0))) as clk:
        torch.cuda.synchronize()
        e0.record()
        batch.step_lanczos(W, K, True)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
    t_ms = e0.elapsed_time(e1)
    launches = sum(c.launches() for c in ctxs) - n0
    mv = [c.profile_read(c.PROF_MATVEC) for c in ctxs]
    lan1 = [c.lanczos_stats() for c in ctxs]
    for c in ctxs:
        c.profile(False)
    iters = sum(b["iterations"] - a["iterations"] for a, b in zip(lan0, lan1))
    calls = sum(b["calls"] - a["calls"] for a, b in zip(lan0, lan1))
    maxed = sum(b["maxed"] - a["maxed"] for a, b in zip(lan0, lan1))
    sb = 8 if pp["precision"] == "fp64" else 4
    alg = sum((48 * w["Nb"] * w["Nc"] + 96 * Kg ** 3) * sb / 4 * m[1]
              for w, Kg, m in zip(reps, grids, mv))
    mv_ms = sum(m[0] for m in mv)
    nbeads = sum(w["Nb"] * w["Nc"] for w in reps)
    # end to end: every step uploads each replica's positions from pinned host
    # buffers, advances the batch one step and reads every replica back
    hb = [[torch.empty(w["Nb"] * w["Nc"], dtype=torch.float64, pin_memory=True).numpy()
           for _ in range(3)] for w in reps]
    for h, c in zip(hb, ctxs):
        for a, b in zip(h, c.positions()):
            a[:] = b
        c.noise_block_release()
    Ke = max(1, min(K, e2e_steps))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for t in range(W + K, W + K + Ke):
        for h, c in zip(hb, ctxs):
            c.set_positions(*h)
        batch.step_lanczos(t, 1, True)
        for h, c in zip(hb, ctxs):
            for a, b in zip(h, c.positions()):
                a[:] = b
    e2e_s = time.perf_counter() - t0
    batch.close()
    # the dominant kernel alone: the block products of one noise block of the
    # largest replica, each between CUDA events on its stream, nothing else
    # running (in the batch 64 streams overlap, so launch durations do not
    # measure a kernel)
    big = max(range(len(reps)), key=lambda q: reps[q]["Nb"] * reps[q]["Nc"])
    cb, wb = ctxs[big], reps[big]
    cb.noise_block_release()
    blk0 = cb.noise_block_stats()
    cb.profile(True)
    cb.step_lanczos(W + K + Ke, noise_block, False)
    cb.sync()
    bl_ms, bl_n = cb.profile_read(cb.PROF_BLOCK)
    cb.profile(False)
    blk1 = cb.noise_block_stats()
    sb = 8 if pp["precision"] == "fp64" else 4
    rhs = (blk1["rhs_iterations"] - blk0["rhs_iterations"]) / max(blk1["iterations"] - blk0["iterations"], 1)
    big_alg = (48 * wb["Nb"] * wb["Nc"] + 96 * grids[big] ** 3) * sb / 4 * rhs
    big_prod = dict(replica=big, beads=wb["Nb"] * wb["Nc"], grid=grids[big], rhs=rhs,
                    avg_product_ms=bl_ms / max(bl_n, 1), products=bl_n, alg_bytes=big_alg,
                    achieved_gbs=big_alg / (bl_ms / max(bl_n, 1) / 1e3) / 1e9 if bl_n else None)
    for c in ctxs:
        c.close()
    return dict(t_ms=t_ms, nbeads=nbeads, launches=launches, clocks=clk.summary(),
                iters_per_step=iters / max(calls, 1), maxed=maxed,
                achieved=alg / (mv_ms / 1e3) / 1e9 if mv_ms else None, alg=alg,
                mv_launches=sum(m[1] for m in mv), e2e=nbeads * Ke / e2e_s, e2e_steps=Ke,
                grids=sorted(set(grids)), big=big_prod, rc=rc, tuned=tuned)


def run_batch(args, world):
    K, W = args.steps, args.warmup
    m = measure_batch(args.path, K, W, args.e2e_steps, args.noise_block)
    peak, kind = peaks()
    value = world * m["nbeads"] * K / (m["t_ms"] / 1e3)
    line = {"metric": METRIC, "value": value, "unit": "bead-steps/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": m["t_ms"] / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if PATHS[args.path]["precision"] == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOADS["c2"]["name"], "replicas": 64,
                       "beads_total": m["nbeads"], "path": args.path,
                       "execution": "one batch: a worker thread and a CUDA stream per replica",
                       "pme_cutoff": m["rc"],
                       "pme_cutoff_autotune_ms": m["tuned"],
                       "pme_grids": "by the accuracy rule per replica box: %s" % m["grids"],
                       "lanczos_iters_per_step": m["iters_per_step"],
                       "lanczos_fallbacks": m["maxed"],
                       "l2": "per-replica grids L2-resident; inputs of all replicas together "
                             "exceed L2", "parallelism": "replicas in one process"},
            "roofline": {"kernel": "particle-mesh product of a noise block of the largest "
                                   "replica (%d beads, %d^3), timed alone"
                                   % (m["big"]["beads"], m["big"]["grid"]), "bound": "hbm",
                         "achieved": m["big"]["achieved_gbs"], "peak": peak, "peak_kind": kind,
                         "unit": "GB/s", "frac": (m["big"]["achieved_gbs"] or 0) / peak,
                         "traffic": None, "alg_bytes_per_launch": m["big"]["alg_bytes"],
                         "avg_launch_ms": m["big"]["avg_product_ms"],
                         "launches": m["big"]["products"],
                         "in_batch": {"achieved": m["achieved"], "launches": m["mv_launches"],
                                      "note": "single products of all replicas, overlapping "
                                              "on 64 streams"}},
            "e2e": {"value": world * m["e2e"], "unit": "bead-steps/s",
                    "h2d_bytes_per_step": 24 * m["nbeads"],
                    "d2h_bytes_per_step": 24 * m["nbeads"], "steps": m["e2e_steps"]},
            "clocks": m["clocks"], "gpu_launches": m["launches"]}
    return line


def accuracy_vs_fp64(w, path, noise_block, pme_rc, pme_grid, seed=1000):
    """Per-result relative error (2-norm over all beads) of the measured path
    against FP64 on the same configuration at the bench's discretisation:
    the forces and the mobility product M F against pme64; the Brownian
    displacement for one seeded z (each solve at tolerance 1e-6) against
    pme64 computing the same square-root factor, i.e. with the path's own
    preconditioner G (a preconditioned solve returns G^-1 sqrt(G M G^T) z,
    another valid factor than sqrt(M) z), and the plain FP32 sqrt(M) z
    (pme32) against plain pme64.  The FP64 path is itself checked against the
    CPU oracle's dense Ewald sum at sizes the oracle can hold (the
    particle-mesh tests)."""
    N = w["Nb"] * w["Nc"]
    z = np.random.default_rng(seed).normal(size=3 * N)
    pre = PATHS[path].get("precond")

    def run(name, precond_from=None):
        c = build_context(w, seed, name, noise_block=noise_block if name == path else 1,
                          pme_rc=pme_rc, pme_grid=pme_grid)
        if precond_from is not None:
            if precond_from == "learned":
                c.mpnn_set_params(np.load(os.path.join(PKG, "mpnn_params.npy")))
            c.set_preconditioner(precond_from, SEGMENT[0] if w["Nb"] % SEGMENT[0] == 0 else 5)
        ext = w["flow"] == 1
        # the step's order: forces and the mobility build in the flow frame,
        # the products after rotating back
        c.reset_force()
        if ext:
            c.transform_coords()
        c.apply_pbc()
        c.build_neighbors()
        c.bond_force()
        c.ev_force()
        c.coulomb_force()
        F = c.forces()
        c.calc_hi()
        if ext:
            c.inverse_coords()
        f = np.ascontiguousarray(F.T).reshape(-1)
        mf = c.mobility_apply(f)
        y, it = c.lanczos_sqrt(z)
        c.close()
        return F, mf, y, it

    rel = lambda u, v: float(np.linalg.norm(u - v) / np.linalg.norm(v))
    a = run(path)
    b = run("pme64", pre)
    out = {"against": "pme64 on the same configuration (FP64 storage)",
           "forces": rel(a[0], b[0]), "mobility_product": rel(a[1], b[1]),
           "displacement": rel(a[2], b[2]),
           "displacement_against": "pme64 with the same preconditioner (the same factor)",
           "krylov_iterations": {path: a[3], "pme64+" + str(pre): b[3]}, "gate": 1e-5,
           "note": "forces are FP64 in every path (springs, excluded volume, Ewald Coulomb); "
                   "a displacement error holds both solves' tolerance and the FP32 storage "
                   "error"}
    if pre is not None:
        p32 = run("pme32")
        p64 = run("pme64")
        out["displacement_plain"] = rel(p32[2], p64[2])
        out["krylov_iterations"].update({"pme32": p32[3], "pme64": p64[3]})
    if pre == "learned" and "pme32-seg" in PATHS:
        # the learned blocks' own share: the same solve on segment blocks alone
        out["krylov_iterations"]["pme32-seg"] = run("pme32-seg")[3]
    return out


def tune_cutoff(w, path, noise_block, rank, dist):
    """The particle-mesh cutoff (grid by the library's rule) whose product of
    the noise block's right-hand sides is fastest on this GPU for the
    workload's seeded configuration (bd_b200.autotune_pme_cutoff); rank 0
    decides and the other ranks take its choice."""
    import bd_b200 as B
    choice = [None, None]
    if rank == 0:
        def make(rc):
            c = build_context(w, 1000, path, noise_block=max(noise_block, 2), pme_rc=rc)
            c.calc_hi()
            return c
        best, times = B.autotune_pme_cutoff(make, w["L"], max(noise_block, 2))
        choice = [best, {str(k): round(v, 4) for k, v in times.items()}]
    choice = rank0_choice(choice, dist)
    return choice[0], choice[1]


def run_ours(args, rank, world, dist):
    w = WORKLOADS[args.workload]
    N = w["Nb"] * w["Nc"]
    K, W = args.steps, args.warmup
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    tuned = None
    if args.pme_rc == "auto":
        if PATHS[args.path]["mobility"] == "pme":
            args.pme_rc, tuned = tune_cutoff(w, args.path, args.noise_block, rank, dist)
        else:
            args.pme_rc = 12.1
    main = measure(w, args.path, K, W, rank, dist, args.e2e_steps, args.noise_block, args.pme_rc,
                   args.pme_grid)
    value = world * N * K / (main["t_max_ms"] / 1e3)
    peak, kind = peaks()
    pme = PATHS[args.path]["mobility"] == "pme"
    roof = {"kernel": ("particle-mesh product (spread, R2C, influence, C2R, gather)" if pme else
                       "k_sym_matvec<%s>" % ("float" if PATHS[args.path]["precision"] == "fp32"
                                             else "double")),
            "bound": "hbm", "achieved": main["achieved_gbs"], "peak": peak, "peak_kind": kind,
            "unit": "GB/s", "frac": (main["achieved_gbs"] or 0) / peak, "traffic": None,
            "alg_bytes_per_launch": main["alg_bytes"], "avg_launch_ms": main["matvec_avg_ms"],
            "launches": main["matvec_launches"]}
    if main["block"]:
        b = main["block"]
        roof.update({"kernel": "particle-mesh product of a noise block (%.1f right-hand sides "
                               "per launch: spread, R2C, influence, C2R, gather)"
                               % b["rhs_per_iteration"],
                     "achieved": b["achieved_gbs"], "frac": b["achieved_gbs"] / peak,
                     "traffic": PRODUCT_TRAFFIC.get(
                         (N, args.pme_grid or __import__("bd_b200").pme_default_grid(
                             w["L"], args.pme_rc), round(float(args.pme_rc), 2),
                          int(round(b["rhs_per_iteration"])))),
                     "alg_bytes_per_launch": b["alg_bytes"], "avg_launch_ms": b["avg_product_ms"],
                     "launches": b["products"],
                     "single_product": {"achieved": main["achieved_gbs"],
                                        "avg_launch_ms": main["matvec_avg_ms"],
                                        "launches": main["matvec_launches"]}})
    e2e = {"value": world * N * main["e2e_steps"] / main["e2e_s"], "unit": "bead-steps/s",
           "h2d_bytes_per_step": 3 * 8 * N, "d2h_bytes_per_step": 3 * 8 * N,
           "steps": main["e2e_steps"]}
    line = {"metric": METRIC, "value": value, "unit": "bead-steps/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": main["t_max_ms"] / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if PATHS[args.path]["precision"] == "fp32" else "f64",
            "data": "synthetic",
            "config": {"workload": w["name"], "beads": N, "path": args.path,
                       "mobility": ("Ewald-summed RPY by smooth PME, grid %d^3, order 8, cutoff %g"
                                    % (args.pme_grid or
                                       __import__("bd_b200").pme_default_grid(w["L"], args.pme_rc),
                                       args.pme_rc) if pme else
                                    "Ewald-summed RPY, every pair (dense packed tiles)"),
                       "pme_cutoff_autotune_ms": tuned,
                       "noise": "Lanczos sqrt(M) z, tol 1e-6, FP64 recurrence and basis" +
                                (", noise blocks of %d steps" % main["block"]["noise_block"]
                                 if main["block"] else "") +
                                (" (Gram-Schmidt pass on an FP32 copy of the basis)"
                                 if main["block"] and PATHS[args.path]["precision"] == "fp32"
                                 else ""),
                       "noise_block": main["block"],
                       "electrostatics": ("Ewald Coulomb, chains alternately -1 / +1 on half "
                                          "their beads" if PATHS[args.path].get("physics") ==
                                          "north" else "Debye-Hueckel, unsigned charges "
                                          "(reference)"),
                       "charge_hop": ("parallel independent sets, Philox draws, "
                                      "Debye-Hueckel energies" if PATHS[args.path].get("physics")
                                      == "north" else "reference sequential sweep"),
                       "preconditioner": {None: "none", "segment": "segment blocks of 10 beads",
                                          "learned": "learned bead blocks on segment blocks "
                                                     "of 10 beads"}[
                                              PATHS[args.path].get("precond")],
                       "precond_fallbacks": main["precond_fallbacks"],
                       "lanczos_iters_per_step": main["lanczos_iters_per_step"],
                       "lanczos_fallbacks": main["lanczos_maxed"],
                       "edot": edot_of(w), "tau_estimate": tau_estimate(w["Nb"]),
                       "l2": ("PME grids of 3 x K^3 FP64 values; working set per product "
                              "near or above L2" if pme else
                              "inputs larger than L2 (packed mobility tiles >> 126 MB)"),
                       "parallelism": "replicas only" if world > 1 else "single GPU"},
            "roofline": roof, "e2e": e2e, "clocks": main["clocks"],
            "gpu_launches": main["launches"], "breakdown": main["breakdown"]}
    plain = "pme64" if pme else "lanczos64"
    if args.compare and args.path != plain:
        # the plain method: the same mobility in FP64 storage, no
        # preconditioner, one Krylov solve per step
        ref64 = measure(w, plain, K, W, rank, dist, 1, 1, args.pme_rc, args.pme_grid)
        line["plain_fp64"] = {"path": plain, "noise_block": 1,
                              "value": world * N * K / (ref64["t_max_ms"] / 1e3),
                              "ms_per_step": ref64["t_max_ms"] / K,
                              "lanczos_iters_per_step": ref64["lanczos_iters_per_step"],
                              "matvec_gbs": ref64["achieved_gbs"]}
        line["speedup_vs_plain_fp64"] = line["value"] / line["plain_fp64"]["value"]
        if pme and args.noise_block > 1:
            # the plain method with the same noise blocks: isolates what FP32
            # storage and the preconditioner gain
            refb = measure(w, plain, K, W, rank, dist, 1, args.noise_block, args.pme_rc,
                           args.pme_grid)
            line["plain_fp64_noise_blocks"] = {
                "path": plain, "noise_block": args.noise_block,
                "value": world * N * K / (refb["t_max_ms"] / 1e3),
                "ms_per_step": refb["t_max_ms"] / K,
                "block_iterations_per_step": (refb["block"] or {}).get(
                    "block_iterations_per_step"),
                "lanczos_iters_per_step": refb["lanczos_iters_per_step"]}
            line["speedup_vs_plain_fp64_noise_blocks"] = (
                line["value"] / line["plain_fp64_noise_blocks"]["value"])
            if PATHS[args.path].get("precond") and "pme32" in PATHS:
                # unpreconditioned Lanczos with everything else the same (FP32
                # storage, noise blocks): what the preconditioner gains
                refu = measure(w, "pme32", K, W, rank, dist, 1, args.noise_block, args.pme_rc,
                               args.pme_grid)
                line["unpreconditioned_fp32"] = {
                    "path": "pme32", "noise_block": args.noise_block,
                    "value": world * N * K / (refu["t_max_ms"] / 1e3),
                    "ms_per_step": refu["t_max_ms"] / K,
                    "lanczos_iters_per_step": refu["lanczos_iters_per_step"]}
                line["speedup_vs_unpreconditioned_fp32"] = (
                    line["value"] / line["unpreconditioned_fp32"]["value"])
    if pme and args.errors and args.path != "pme64":
        line["errors"] = accuracy_vs_fp64(w, args.path, args.noise_block, args.pme_rc,
                                          args.pme_grid)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="c3")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--path", choices=sorted(PATHS), default="pme32-learned")
    # 10 divides the rebuild period of 100 steps (a block never spans a
    # rebuild), so every block is full; 8 would leave one of 4 per period
    ap.add_argument("--noise-block", type=int, default=10,
                    help="steps whose Brownian displacements one multi-vector Lanczos run "
                         "solves (particle-mesh paths; 1 = one solve per step)")
    ap.add_argument("--pme-rc", default=None,
                    help="particle-mesh real-space cutoff, or 'auto' (the default where the "
                         "workload fixes none): the fastest of bd_b200.PME_CUTOFFS for the "
                         "product on this GPU; the grid follows it (12.9 L / rc points, "
                         "constant interpolation accuracy)")
    ap.add_argument("--pme-grid", type=int, default=0,
                    help="particle-mesh grid points per cell edge (0: the library's rule "
                         "for the cutoff)")
    ap.add_argument("--segment", type=int, default=10,
                    help="beads per segment block of the preconditioned paths")
    ap.add_argument("--compare", type=int, default=1,
                    help="also time the plain FP64 Krylov path, one solve per step "
                         "(plain_fp64) and with the same noise blocks "
                         "(plain_fp64_noise_blocks)")
    ap.add_argument("--errors", type=int, default=1,
                    help="per-result error of the path against pme64 at the bench config")
    args = ap.parse_args()
    if args.pme_rc is None:
        args.pme_rc = WORKLOADS[args.workload].get("pme_rc", "auto")
    if args.pme_rc != "auto":
        args.pme_rc = float(args.pme_rc)
    SEGMENT[0] = args.segment
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    w = WORKLOADS[args.workload]
    N = w["Nb"] * w["Nc"]

    if args.impl == "reference":
        if rank != 0:
            return
        th = host_threads()
        r = time_reference(w, steps=min(args.steps, 10), warmup=min(args.warmup, 1), threads=th)
        if r is None:
            print(json.dumps({"impl": "reference",
                              "unavailable": "reference library oracle/_ref not built here"}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": r["value"],
                "unit": "bead-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["per_step"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": w["name"], "beads": N,
                           "measured_at_beads": r["beads"]},
                "cpu_baseline": {"value": r["value"], "unit": "bead-steps/s", "cores": th,
                                 "kind": "reference", "sample": r["sample"]},
                "value_with_extrapolated_sweep": r["value_with_extrapolated_sweep"],
                "components": r["components"],
                "e2e": {"value": r["value"], "unit": "bead-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if WORKLOADS[args.workload].get("ensemble"):
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            line = run_batch(args, world)
        else:
            line = run_ours(args, rank, world, dist)
        if rank == 0 and not args.no_cpu_baseline and not WORKLOADS[args.workload].get("ensemble"):
            r = time_reference(w, steps=5, warmup=1, threads=host_threads())
            if r is not None:
                line["cpu_baseline"] = {"value": r["value"], "unit": "bead-steps/s",
                                        "cores": r["threads"], "kind": "reference",
                                        "sample": r["sample"], "beads": r["beads"],
                                        "value_with_extrapolated_sweep":
                                            r["value_with_extrapolated_sweep"]}
        if rank == 0:
            print(json.dumps(line))
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
