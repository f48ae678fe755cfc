"""CPU model of the parallel charge-hop sweep (test infrastructure only).

No counterpart in the reference (whose sweep is sequential: chargeHop,
shear/src/main26.c:1926-2390).  Restates csrc/bd_mc.cu's independent-set
sweep: cells of the Gauss-reduced cell at least R wide (an even number per
direction), eight parity colours run in turn, each cell's charges visited in
index order; the reference's proposal rules (first bead by index within
|NID|^2 < 4.41 excluding the own bead and its index neighbours, the 0.33 /
0.66 / 0.5 thresholds, chain ends, occupancy); acceptance
min(1, exp(-barrier - dE/2)) with dE the Debye-Hueckel energy change against
every other charge, or the Ewald one (EwaldTerms), other cells' charges at
their sites at the start of the colour; Philox4x32-10 draws (Salmon et al., SC'11) keyed by philox_seed with
counters (charge, sweep, purpose).  Distances come from the oracle's getNID,
which is bit-exact to the reference's.  Only tests/ may import this module.
"""
from __future__ import annotations

import math

import numpy as np

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    x0, x1, x2, x3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0 = M0 * x0
        p1 = M1 * x2
        hi0, lo0 = p0 >> 32, p0 & MASK
        hi1, lo1 = p1 >> 32, p1 & MASK
        x0, x1, x2, x3 = (hi1 ^ x1 ^ k0) & MASK, lo1, (hi0 ^ x3 ^ k1) & MASK, lo0
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return x0, x1, x2, x3


def u01(k, sweep, tag, seed):
    x = philox4x32_10((k & MASK, sweep & MASK, (sweep >> 32) & MASK, 0x4D430000 | tag),
                      (seed & MASK, (seed >> 32) & MASK))
    return float(((x[0] >> 5) << 26) | (x[1] >> 6)) / 9007199254740992.0


class EwaldTerms:
    """Ewald energy differences of a trial in the parallel sweep (the GPU's
    BD_COULOMB_EWALD acceptance, csrc/bd_mc.cu k_hop_colour).  The reciprocal
    potential is the explicit k-space sum (converged to about exp(-tol_exp))
    where the GPU interpolates its mesh; the other terms are the same
    formulas.  Also keeps the structure factor of the current charge state, so
    that each trial's exact Ewald energy difference (every term from the
    k-space sum, the periodic pair term included) can be set beside the
    model's."""

    def __init__(self, H, beta, rc, lambda_b, tol_exp=30.0):
        self.H = np.asarray(H, float)
        self.Hi = np.linalg.inv(self.H)
        self.V = abs(np.linalg.det(self.H))
        self.beta, self.rc, self.lb = beta, rc, lambda_b
        kcut = 2 * beta * math.sqrt(tol_exp)
        B = 2 * math.pi * self.Hi.T
        mmax = [int(math.ceil(kcut / (2 * math.pi) * np.linalg.norm(self.H[:, d]))) + 1
                for d in range(3)]
        g = np.mgrid[-mmax[0]:mmax[0] + 1, -mmax[1]:mmax[1] + 1,
                     -mmax[2]:mmax[2] + 1].reshape(3, -1).T
        k = g @ B.T
        kk = np.einsum("ij,ij->i", k, k)
        keep = (kk > 0) & (kk < kcut * kcut)
        self.k, kk = k[keep], kk[keep]
        # E_rec = sum_k A_k |S(k)|^2 over all k != 0
        self.A = 2 * math.pi * lambda_b / self.V * np.exp(-kk / (4 * beta ** 2)) / kk
        # quadratic form of the reciprocal pair term's periodic remainder:
        # G(r) = lambda_B erf(beta r)/r + r^T Q r + const + O(r^4)
        self.Q = (-(self.A[:, None, None] * self.k[:, :, None] * self.k[:, None, :]).sum(0)
                  + lambda_b * 2 * beta ** 3 / (3 * math.sqrt(math.pi)) * np.eye(3))

    def minimg(self, d):
        s = self.Hi @ d
        s -= np.rint(s)
        return self.H @ s

    def real(self, d):
        rr = float(self.minimg(d) @ self.minimg(d))
        if rr >= self.rc ** 2:
            return 0.0
        r = math.sqrt(rr)
        return self.lb * math.erfc(self.beta * r) / r

    def G(self, d):
        v = self.minimg(d)
        r = math.sqrt(float(v @ v))
        if r <= 1e-12:
            return self.lb * 2 * self.beta / math.sqrt(math.pi)
        return self.lb * math.erf(self.beta * r) / r + float(v @ self.Q @ v)

    def phase(self, r):
        return np.exp(1j * (self.k @ r))

    def structure(self, pos, q):
        return (q[:, None] * np.exp(1j * (pos @ self.k.T))).sum(0)

    def phi(self, S, r):
        """Reciprocal potential at r of the charges with structure factor S
        (all of them, none excluded): 2 sum_k A_k Re(S conj(e^{ik.r}))."""
        return 2.0 * float((self.A * (S * np.conj(self.phase(r))).real).sum())


def parallel_sweep(o, x, y, z, track, qk, flags, H, cth, sth, R, lambda_b, kappa_d,
                   barrier, barrier2, seed, sweep, ewald=None):
    """One sweep; x, y, z in the stored frame, H the lab-frame reduced cell.
    Returns (track, old, log, flags) after the sweep.  With ewald (an
    EwaldTerms) the trial energies are the Ewald ones and the return value
    gains two arrays: the model energy difference of each trial (NaN where
    blocked) and the exact Ewald difference in the same state."""
    track = np.array(track, dtype=np.int64)
    flags = np.array(flags, dtype=np.int64)
    N, Nb, nch = o.N, o.s.Nb, len(track)
    old = np.zeros(nch, np.int64)
    log = np.zeros((nch, 3), np.int64)
    V = abs(np.linalg.det(H))
    Hi = np.linalg.inv(H)
    a = H.T
    n = []
    for j in range(3):
        w = V / np.linalg.norm(np.cross(a[(j + 1) % 3], a[(j + 2) % 3]))
        m = int(math.floor(w / R))
        n.append(m - (m & 1) if m >= 2 else 1)
    cell_of = np.zeros(nch, np.int64)
    for k in range(nch):
        b = track[k]
        xl, yl = x[b] * cth - y[b] * sth, x[b] * sth + y[b] * cth
        s = Hi @ np.array([xl, yl, z[b]])
        cd = []
        for d in range(3):
            sd = s[d] - math.floor(s[d])
            cd.append(min(int(sd * n[d]), n[d] - 1))
        cell_of[k] = (cd[0] * n[1] + cd[1]) * n[2] + cd[2]

    def dh(bi, bj):
        v = o.nid(x, y, z, bi, bj)
        r = math.sqrt(v @ v)
        return lambda_b / r * math.exp(-kappa_d * r)

    lab = np.stack([x * cth - y * sth, x * sth + y * cth, z], 1)
    de_model = np.full(nch, np.nan)
    de_exact = np.full(nch, np.nan)
    ew = ewald
    for colour in range(8):
        site0 = track.copy()
        if ew is not None:
            S0 = ew.structure(lab[site0], np.asarray(qk, float))
        for cell in range(n[0] * n[1] * n[2]):
            cz, cy, cx = cell % n[2], (cell // n[2]) % n[1], cell // (n[1] * n[2])
            col = ((cx & 1 if n[0] > 1 else 0) << 2) | ((cy & 1 if n[1] > 1 else 0) << 1) | \
                  (cz & 1 if n[2] > 1 else 0)
            if col != colour:
                continue
            moved = []  # (a_j, b_j, q_j) of this cell's accepted moves in the colour
            for k in np.nonzero(cell_of == cell)[0]:
                c = int(track[k])
                first = None
                for j in range(N):
                    if j in (c - 1, c, c + 1):
                        continue
                    v = o.nid(x, y, z, c, j)
                    if v @ v < 4.41:
                        first = j
                        break
                mm = u01(int(k), sweep, 0, seed)
                test = 0
                if first is not None:
                    if mm < .33:
                        c2, sblock, test = c + 1, (c == N - 1 or c % Nb == Nb - 1 or c == Nb - 1), 1
                    elif mm > 0.66:
                        c2, sblock, test = c - 1, (c - 1 < 0 or c == 0 or c % Nb == 0), 1
                    else:
                        c2, sblock, test = first, False, 2
                elif mm > .5:
                    c2, sblock = c + 1, (c == N - 1 or c % Nb == Nb - 1 or c == Nb - 1)
                else:
                    c2, sblock = c - 1, (c - 1 < 0 or c == 0 or c % Nb == 0)
                if not sblock and flags[c2]:
                    sblock = True
                if sblock:
                    log[k] = (0, c2, 0)
                    continue
                de = 0.0
                if ew is None:
                    for oo in range(nch):
                        if oo == k:
                            continue
                        b = track[oo] if cell_of[oo] == cell else site0[oo]
                        de += qk[k] * qk[oo] * (dh(c2, b) - dh(c, b))
                else:
                    qm = float(qk[k])
                    ra, rb = lab[c], lab[c2]
                    for oo in range(nch):
                        if oo == k:
                            continue
                        b = track[oo] if cell_of[oo] == cell else site0[oo]
                        de += qm * qk[oo] * (ew.real(rb - lab[b]) - ew.real(ra - lab[b]))
                    de_real = de
                    de += qm * (ew.phi(S0, rb) - ew.phi(S0, ra))
                    de -= qm * qm * (ew.G(rb - ra) - ew.G(np.zeros(3)))
                    St = S0.copy()
                    for aj, bj, qj in moved:
                        de += qm * qj * (ew.G(rb - lab[bj]) - ew.G(rb - lab[aj])
                                         - ew.G(ra - lab[bj]) + ew.G(ra - lab[aj]))
                        St += qj * (ew.phase(lab[bj]) - ew.phase(lab[aj]))
                    # exact: real space as above, reciprocal from the structure
                    # factor the trial sees (colour start + this cell's moves)
                    Sn = St + qm * (ew.phase(rb) - ew.phase(ra))
                    de_exact[k] = de_real + float((ew.A * (np.abs(Sn) ** 2 - np.abs(St) ** 2)).sum())
                    de_model[k] = de
                xx = math.exp(-(barrier2 if test == 2 else barrier) - 0.5 * de)
                acc = 1 if xx >= 1 else int(u01(int(k), sweep, 1, seed) <= xx)
                old[k] = c
                if acc:
                    flags[c], flags[c2] = 0, 1
                    track[k] = c2
                    moved.append((c, c2, float(qk[k])))
                log[k] = (1 if acc else 2, c2, test)
    if ew is not None:
        return track, old, log, flags, de_model, de_exact
    return track, old, log, flags
