"""CPU model of the Ewald-summed Coulomb interaction (test infrastructure only).

No counterpart in the reference, whose electrostatics is the Debye-Hueckel
pair force of coulombForce (shear/src/main26.c:1891-1925).  This is the
textbook Ewald sum of U = lambda_B sum_{i<j} q_i q_j / r over the periodic
cell H (real-space images within a converged cutoff, explicit k-space sum,
self term, neutralising background for a net charge), converged to about
exp(-tol_exp), giving forces (kT per unit length) and the total energy (kT).
Only tests/ may import this module.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc


def ewald_coulomb(H, pos, q, lambda_b, alpha=None, tol_exp=30.0):
    H = np.asarray(H, float)
    pos = np.asarray(pos, float)
    q = np.asarray(q, float)
    N = len(pos)
    V = abs(np.linalg.det(H))
    Hi = np.linalg.inv(H)
    a = H.T
    w = np.array([V / np.linalg.norm(np.cross(a[(j + 1) % 3], a[(j + 2) % 3])) for j in range(3)])
    if alpha is None:
        alpha = 5.0 / w.min()
    rcut = math.sqrt(tol_exp) / alpha
    kcut = 2 * alpha * math.sqrt(tol_exp)
    nimg = [int(math.ceil(rcut / w[d])) + 1 for d in range(3)]
    shifts = np.array([[i, j, k] for i in range(-nimg[0], nimg[0] + 1)
                       for j in range(-nimg[1], nimg[1] + 1)
                       for k in range(-nimg[2], nimg[2] + 1)], float) @ H.T
    F = np.zeros((N, 3))
    E = 0.0
    for i in range(N):
        d = pos[i][None, None, :] - pos[None, :, :] + shifts[:, None, :]  # r_i - r_j - n
        rr = np.einsum("snk,snk->sn", d, d)
        m = (rr < rcut * rcut) & (rr > 0)
        rrm = np.where(m, rr, 1.0)
        r = np.sqrt(rrm)
        qq = lambda_b * q[i] * q[None, :]
        ec = np.where(m, erfc(alpha * r) / r, 0.0)
        fr = np.where(m, (ec + 2 * alpha / math.sqrt(math.pi) * np.exp(-alpha ** 2 * rrm)) / rrm, 0.0)
        F[i] += np.einsum("sn,n,snk->k", fr, qq[0], d)
        E += 0.5 * float((qq[0][None, :] * ec).sum())
    B = 2 * math.pi * Hi.T
    mmax = [int(math.ceil(kcut / (2 * math.pi) * np.linalg.norm(H[:, d]))) + 1 for d in range(3)]
    g = np.mgrid[-mmax[0]:mmax[0] + 1, -mmax[1]:mmax[1] + 1, -mmax[2]:mmax[2] + 1].reshape(3, -1).T
    k = g @ B.T
    kk = np.einsum("ij,ij->i", k, k)
    keep = (kk > 0) & (kk < kcut * kcut)
    k, kk = k[keep], kk[keep]
    G = 4 * math.pi * lambda_b / (V * kk) * np.exp(-kk / (4 * alpha ** 2))
    for s in range(0, len(k), 4096):
        ks, Gs = k[s:s + 4096], G[s:s + 4096]
        ph = pos @ ks.T
        c, sn = np.cos(ph), np.sin(ph)
        Sc, Ss = q @ c, q @ sn
        E += 0.5 * float((Gs * (Sc * Sc + Ss * Ss)).sum())
        # F_i = q_i sum_k G k (sin(k r_i) Sc - cos(k r_i) Ss)
        F += q[:, None] * ((sn * Sc - c * Ss) * Gs) @ ks
    E -= lambda_b * alpha / math.sqrt(math.pi) * float((q * q).sum())
    Q = float(q.sum())
    E -= math.pi * lambda_b * Q * Q / (2 * V * alpha ** 2)
    return F, E
