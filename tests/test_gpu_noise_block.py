"""Noise blocks of the Krylov Brownian step on the GPU.

No reference counterpart (the reference draws and solves one step at a
time).  With noise_block B, bd_step_lanczos solves the displacements
sqrt(M) z_t of up to B consecutive steps by one multi-vector Lanczos run.
The mobility is frozen between rebuilds and z_t does not depend on the state,
so a run with blocks must reproduce the per-step run:

* the draws are the same and in the same order: the context's noise vector
  after the call is bit-identical (Philox, and the reference's ran1 with the
  sequential charge hop, whose sweeps cut the blocks);
* positions after the call agree with the per-step run to 1e-8 of the total
  displacement at Lanczos tolerance 1e-10 (FP64 particle-mesh products whose
  atomic spreading is the only difference in rounding), plain and
  segment-preconditioned, shear and planar extension;
* blocks stop at mobility rebuilds and at the end of the call (the number of
  block solves is the count of those cut points);
* at the default tolerance 1e-6 and FP32 grids, the per-right-hand-side
  Krylov dimensions stay those of the per-step solves (within the check
  interval) and the displacements within the tolerance;
* the block solve with its convergence checks and loop on the device (one
  graph with a conditional while node) takes the Krylov dimensions of the
  host-checked loop and the same displacements to 1e-10.
"""
import numpy as np
import pytest

import bd_b200 as B

pytestmark = pytest.mark.gpu


def _run(nb, *, flow=1, steps=12, srpy=5, precond="none", noise="philox", hop="parallel",
         with_hop=False, tol=1e-10, precision="fp64", charges=False, MStep=4, t0=0,
         device=True):
    Nb, Nc, L = 25, 20, 30.0
    x, y, z = B.random_chains(Nb, Nc, L, 3, bond=2.0, min_sep=2.0)
    x, y = B.lab_frame(flow, x, y)
    kw = {}
    track = None
    if charges:
        track = B.random_charges(Nb, Nc, 0.5, 4)
        kw = dict(Ncharges=len(track), barrier=0.5, barrier2=1.0)
    c = B.Context(B.make_params(flow, Nb, Nc, L, 0.05, 5e-4, mobility="pme", noise=noise,
                                precision=precision, shear_kappas_override=1, srpy=srpy,
                                MStep=MStep, hop=hop, lanczos_tol=tol, noise_block=nb, **kw))
    c.set_device_krylov(device)
    c.set_positions(x, y, z)
    if track is not None:
        c.set_charges(track)
    c.set_time(t0, t0)
    c.update_lattice(t0)
    c.transform_coords()
    c.apply_pbc()
    c.build_neighbors()
    c.inverse_coords()
    if precond != "none":
        c.set_preconditioner(precond, 5)
    x0 = np.stack(c.positions())
    c.step_lanczos(t0, steps, with_hop)
    return c, x0, np.stack(c.positions())


def _compare(a, b, tol):
    (ca, x0, xa), (cb, _, xb) = a, b
    assert np.all(np.isfinite(xa)) and np.all(np.isfinite(xb))
    assert np.array_equal(ca.noise(), cb.noise())
    d = np.linalg.norm(xa - x0)
    assert np.linalg.norm(xa - xb) <= tol * d, (np.linalg.norm(xa - xb) / d)


@pytest.mark.parametrize("flow", [0, 1])
@pytest.mark.parametrize("precond", ["none", "segment"])
def test_block_matches_per_step(flow, precond):
    ref = _run(1, flow=flow, precond=precond)
    blk = _run(8, flow=flow, precond=precond)
    _compare(ref, blk, 1e-8)
    # rebuilds at t = 0, 5, 10 and the end of the call at 12 cut the blocks:
    # [0, 5), [5, 10), [10, 12)
    st = blk[0].noise_block_stats()
    assert st["blocks"] == 3, st
    ls0, ls1 = ref[0].lanczos_stats(), blk[0].lanczos_stats()
    # the last block also solved steps 12-14 ahead of the next call
    assert ls0["calls"] == 12 and ls1["calls"] == 15
    assert ls1["maxed"] == 0
    if precond != "none":
        assert blk[0].precond_stats()["fallbacks"] == 0


@pytest.mark.parametrize("precond,precision,tol,agree", [("none", "fp64", 1e-10, 1e-10),
                                                          ("segment", "fp64", 1e-6, 1e-10),
                                                          ("segment", "fp32", 1e-6, 1e-7)])
def test_device_checked_loop_matches_host_checks(precond, precision, tol, agree):
    """The whole block solve as one graph with the convergence checks on the
    device (quadrature square root of the tridiagonal) against the host's
    checks (implicit QR), one iteration behind: the same Krylov dimensions
    and displacements to 1e-10 of the total (1e-7 with FP32 grids, whose
    atomic spreading differs in rounding between any two runs).  The host
    loop runs one more block iteration per block (the one it launches ahead
    while checking), the device loop none."""
    dev = _run(8, precond=precond, precision=precision, tol=tol, device=True)
    host = _run(8, precond=precond, precision=precision, tol=tol, device=False)
    _compare(host, dev, agree)
    sd, sh = dev[0].lanczos_stats(), host[0].lanczos_stats()
    assert sd["iterations"] == sh["iterations"] and sd["calls"] == sh["calls"], (sd, sh)
    bd, bh = dev[0].noise_block_stats(), host[0].noise_block_stats()
    assert bd["blocks"] == bh["blocks"]
    assert bh["iterations"] - bh["blocks"] <= bd["iterations"] <= bh["iterations"], (bd, bh)
    kd, kh = dev[0].krylov_check_stats(), host[0].krylov_check_stats()
    assert kd["device_solves"] == dev[0].noise_block_stats()["blocks"] and kd["host_fallbacks"] == 0
    assert kh["device_solves"] == 0


def test_block_capacity_and_start_time():
    # block capacity 3 inside rebuild windows of 5, starting mid-window at t0 = 7:
    # [7, 10), [10, 13), [13, 15), [15, 18), [18, 20)
    ref = _run(1, steps=12, t0=7)
    blk = _run(3, steps=12, t0=7)
    _compare(ref, blk, 1e-8)
    assert blk[0].noise_block_stats()["blocks"] == 5


def _setup(nb, noise="philox"):
    c, x0, _ = _run(nb, steps=0, noise=noise, srpy=100)
    return c, x0


@pytest.mark.parametrize("noise", ["philox", "ran1"])
def test_blocks_across_calls(noise):
    """One step per call with host round trips of the positions (the caller
    pattern of an end-to-end loop): the block made by the first call serves
    the next calls; then a generator use outside the step (bd_get_noise)
    winds the generator back, so the draw equals the per-step run's next."""
    out = []
    for nb in (1, 6):
        c, _ = _setup(nb, noise)
        for t in range(8):
            x = c.positions()
            c.set_positions(*x)
            c.step_lanczos(t, 1, False)
        xs = np.stack(c.positions())
        r8 = c.noise()
        c.get_noise()
        out.append((c, xs, r8, c.noise()))
    (c1, x1, a1, b1), (c6, x6, a6, b6) = out
    assert np.array_equal(a1, a6) and np.array_equal(b1, b6)
    assert np.linalg.norm(x1 - x6) <= 1e-8 * np.linalg.norm(x1)
    # [0, 6) and [6, 12): two blocks; the second left after two of its steps
    assert c6.noise_block_stats()["blocks"] == 2
    if noise == "ran1":
        assert np.array_equal(c1.rng().state_words(), c6.rng().state_words())


def test_rebuild_between_calls_voids_block():
    """A mobility rebuild requested between calls voids the block; the steps
    after it use the new mobility and the rewound draws."""
    out = []
    for nb in (1, 6):
        c, _ = _setup(nb)
        c.step_lanczos(0, 3, False)
        c.calc_hi()
        c.step_lanczos(3, 4, False)
        out.append((c, np.stack(c.positions()), c.noise()))
    (c1, x1, r1), (c6, x6, r6) = out
    assert np.array_equal(r1, r6)
    assert np.linalg.norm(x1 - x6) <= 1e-8 * np.linalg.norm(x1)
    assert c6.noise_block_stats()["blocks"] == 2


def test_ran1_blocks_stop_at_sequential_hop():
    # one generator for the noise and the sequential sweep (every 4 steps):
    # blocks end at each sweep step, so the draws keep their order
    ref = _run(1, noise="ran1", hop="sequential", with_hop=True, charges=True, srpy=100)
    blk = _run(8, noise="ran1", hop="sequential", with_hop=True, charges=True, srpy=100)
    _compare(ref, blk, 1e-8)
    assert np.array_equal(ref[0].charges()[0], blk[0].charges()[0])
    assert np.array_equal(ref[0].rng().state_words(), blk[0].rng().state_words())
    # sweeps at t = 0, 4, 8: blocks [0, 1), [1, 5), [5, 9), [9, 12)
    assert blk[0].noise_block_stats()["blocks"] == 4


def test_default_tolerance_fp32():
    ref = _run(1, tol=1e-6, precision="fp32", steps=10, srpy=100, precond="segment")
    blk = _run(10, tol=1e-6, precision="fp32", steps=10, srpy=100, precond="segment")
    (ca, x0, xa), (cb, _, xb) = ref, blk
    assert np.array_equal(ca.noise(), cb.noise())
    # each run within the tolerance (1e-6) of its own operator's root; the
    # block product (complex-packed pairs) and the single product (real
    # transforms) differ by up to 2e-6 in FP32 storage, so 3e-6 of the
    # displacement over the ten steps
    assert np.linalg.norm(xa - xb) <= 3e-6 * np.linalg.norm(xa - x0), (
        np.linalg.norm(xa - xb) / np.linalg.norm(xa - x0))
    ia = ca.lanczos_stats()["iterations"] / 10
    ib = cb.lanczos_stats()["iterations"] / 10
    assert abs(ia - ib) <= 2.0, (ia, ib)
    st = cb.noise_block_stats()
    assert st["blocks"] == 1 and st["iterations"] <= ib + 6
