"""CPU model of the learned preconditioner network (test infrastructure only).

No counterpart in the reference.  A numpy restatement of the forward and
backward passes of smdlt-ca-chrg-flow_b200/csrc/bd_mpnn.cu: the same neighbour
features (the 12 nearest beads within 6, minimum image, ties by index; unit
vectors; 16 Gaussian radial features centred on 2..6 with width 0.35), the
same three layers of width 64 with SiLU, the same heads
G_i = a_i (I + sum_j c_ij n_ij n_ij^T), a_i = exp(clamp(wa.u_i + ca, -4, 4)),
c_ij = tanh(wb.(u_i * e_ij) + cb) / 24, and the loss
(1/N) sum_i |G_i z_i - t_i|^2.  With bf16=True the operands of every dense
product are rounded to BF16 (round to nearest even) as the tensor-core
kernels do, so the model and the CUDA gradients agree to FP32 accumulation
order; with bf16=False it is the exact function, whose analytic gradient the
tests check against finite differences.  Only tests/ may import this module.
"""
from __future__ import annotations

import numpy as np

KN, WD, NR, CUT = 12, 64, 16, 6.0
LAYOUT = [("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
          ("W34", (64, 128)), ("b3", (64,)), ("wa", (64,)), ("ca", (1,)),
          ("wb", (64,)), ("cb", (1,))]


def unpack(w):
    out, o = {}, 0
    for name, shp in LAYOUT:
        n = int(np.prod(shp))
        out[name] = np.asarray(w[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[n], np.float64).reshape(-1) for n, _ in LAYOUT])


def to_bf16(x):
    """Round to BF16 (nearest even) through FP32, returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def features(nid, candidates, N):
    """nid(i, j) -> lab-frame r_i - r_j (the oracle's getNID); candidates[i]
    the beads to consider (the Verlet row).  Returns nbr (N, 12) with -1 for
    empty slots, unit vectors (N, 12, 3) and radial features (N, 12, 16)."""
    nbr = -np.ones((N, KN), np.int64)
    nvec = np.zeros((N, KN, 3))
    rbf = np.zeros((N, KN, NR))
    mu = (np.float32(2.0) + np.float32(4.0) * np.arange(NR, dtype=np.float32) / np.float32(NR - 1))
    for i in range(N):
        cand = []
        for j in candidates[i]:
            d = np.asarray(nid(i, j))
            r = float(np.float32(np.sqrt(d @ d)))
            if r < CUT:
                cand.append((r, int(j), d))
        cand.sort(key=lambda q: (q[0], q[1]))
        for k, (r, j, d) in enumerate(cand[:KN]):
            nbr[i, k] = j
            nvec[i, k] = (d / np.sqrt(d @ d)).astype(np.float32)
            x = (np.float32(r) - mu) / np.float32(0.35)
            rbf[i, k] = np.exp(np.float32(-0.5) * x * x).astype(np.float32)
    return nbr, nvec, rbf


def _silu(x):
    return x / (1 + np.exp(-x))


def _silu_grad(x):
    s = 1 / (1 + np.exp(-x))
    return s * (1 + x * (1 - s))


def forward(w, nbr, nvec, rbf, bf16=True):
    P = unpack(w)
    r = to_bf16 if bf16 else (lambda x: np.asarray(x, np.float64))
    N = nbr.shape[0]
    mask = (nbr >= 0).astype(np.float64)
    c = {}
    c["g1"] = r(rbf.reshape(-1, NR)) @ r(P["W1"]).T + P["b1"]
    c["e"] = _silu(c["g1"]).reshape(N, KN, WD)
    c["mv"] = np.einsum("ik,iko->io", mask, c["e"]) / KN
    c["o2"] = r(c["mv"]) @ r(P["W2"]).T + P["b2"]
    c["h"] = _silu(c["o2"])
    hn = np.where(nbr[..., None] >= 0, c["h"][np.maximum(nbr, 0)], 0.0)
    c["X3"] = np.concatenate([hn.sum(1) / KN, c["h"]], axis=1)
    c["p3"] = r(c["X3"]) @ r(P["W34"]).T + P["b3"]
    c["u"] = _silu(c["p3"])
    c["s"] = c["u"] @ P["wa"] + P["ca"][0]
    c["a"] = np.exp(np.clip(c["s"], -4, 4))
    c["t"] = np.einsum("io,iko->ik", c["u"] * P["wb"], c["e"]) + P["cb"][0]
    c["c"] = np.tanh(c["t"]) * (0.5 / KN) * mask
    G = np.eye(3)[None] + np.einsum("ik,ikp,ikq->ipq", c["c"], nvec, nvec)
    c["G"] = c["a"][:, None, None] * G
    c["mask"], c["nbr"], c["nvec"], c["rbf"], c["P"] = mask, nbr, nvec, rbf, P
    return c


def loss_grad(w, nbr, nvec, rbf, z, t, bf16=True):
    """Loss and gradient (flat, in the parameter layout) for z, t of shape (N, 3)."""
    c = forward(w, nbr, nvec, rbf, bf16)
    P = c["P"]
    rr = to_bf16 if bf16 else (lambda x: np.asarray(x, np.float64))
    N = nbr.shape[0]
    z = np.asarray(z, np.float64).reshape(N, 3)
    t = np.asarray(t, np.float64).reshape(N, 3)
    res = np.einsum("ipq,iq->ip", c["G"], z) - t
    loss = float((res * res).sum() / N)
    dG = 2.0 / N * np.einsum("ip,iq->ipq", res, z)
    mask, nvec = c["mask"], c["nvec"]
    ndn = np.einsum("ikp,ipq,ikq->ik", nvec, dG, nvec) * mask
    da = np.einsum("ipp->i", dG) + (c["c"] * ndn).sum(1)
    dc = c["a"][:, None] * ndn
    dt = dc * (0.5 / KN) * (1 - np.tanh(c["t"]) ** 2) * mask
    ds = np.where((c["s"] > -4) & (c["s"] < 4), da * c["a"], 0.0)
    g = {}
    g["wa"] = ds @ c["u"]
    g["ca"] = np.array([ds.sum()])
    g["wb"] = np.einsum("ik,io,iko->o", dt, c["u"], c["e"])
    g["cb"] = np.array([dt.sum()])
    du = ds[:, None] * P["wa"] + np.einsum("ik,iko->io", dt, c["e"]) * P["wb"]
    de = dt[:, :, None] * (P["wb"] * c["u"])[:, None, :]
    dp3 = du * _silu_grad(c["p3"])
    g["W34"] = rr(dp3).T @ rr(c["X3"])
    g["b3"] = dp3.sum(0)
    dX3 = rr(dp3) @ rr(P["W34"])
    dh = dX3[:, WD:].copy()
    nbr = c["nbr"]
    for k in range(KN):
        sel = nbr[:, k] >= 0
        np.add.at(dh, nbr[sel, k], dX3[sel, :WD] / KN)
    do2 = dh * _silu_grad(c["o2"])
    g["W2"] = rr(do2).T @ rr(c["mv"])
    g["b2"] = do2.sum(0)
    dm = rr(do2) @ rr(P["W2"])
    de = de + mask[:, :, None] * dm[:, None, :] / KN
    dg1 = de.reshape(-1, WD) * _silu_grad(c["g1"])
    g["W1"] = rr(dg1).T @ rr(c["rbf"].reshape(-1, NR))
    g["b1"] = dg1.sum(0)
    return loss, pack(g), c
