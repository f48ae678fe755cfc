"""CPU model of the matrix-free RPY mobility (test infrastructure only).

The reference has no particle-mesh path: its mobility is the dense Ewald-
summed Rotne-Prager-Yamakawa matrix of calcHI (shear/src/main26.c:1530-1806,
extensional/src/main14.c:1548-1824).  This module gives the tests two numpy
models of M v on the same periodic cell:

* ewald_apply: the Ewald sum itself (Beenakker split, real-space images within
  a cutoff, explicit k-space sum, full 3x3 self block), converged to ~1e-9,
  evaluated as M v without forming M (O(N n_k) for the k-space part).  Its
  pair tensors are those of calcHI (real-space C1..C4 terms,
  shear/src/main26.c:1727-1741; k-space coefficient, shear/src/main26.c:
  1602-1622), so on every off-diagonal block it equals oracle/bd_oracle.c's
  bdo_calc_hi_ewald; on the diagonal blocks it also keeps the off-diagonal
  entries of the self block, which calcHI does not store;
* pme_apply: the smooth particle-mesh restatement (Essmann et al.,
  J. Chem. Phys. 103, 8577 (1995)) with the same grid, spline order, split
  and real-space cutoff as the CUDA path, to check that path to rounding.

parity: the Ewald model is pinned against bdo_calc_hi_ewald (itself pinned
against the reference's calcHI) in tests/test_oracle_pin.py; the PME model is
checked against the Ewald model within its discretisation error.
Only tests/ may import this module.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc


def cell(L1, L2, L):
    """Lab-frame cell matrix with the lattice vectors as columns."""
    return np.array([[L1[0], L2[0], 0.0], [L1[1], L2[1], 0.0], [0.0, 0.0, L]], dtype=float)


def reduced_cell(L1, L2, L):
    """Cell of the same lattice on the Gauss-reduced basis (b1, b2) of the
    lattice spanned by L1, L2: |b1| <= |b2| and |b1.b2| <= |b1|^2/2."""
    a = np.array(L1[:2], float)
    b = np.array(L2[:2], float)
    for _ in range(64):
        if a @ a > b @ b:
            a, b = b, a
        mu = np.rint((a @ b) / (a @ a))
        if mu == 0:
            break
        b = b - mu * a
    return cell(a, b, L)


def real_terms(alpha, rr):
    """t1, t2 of the real-space Beenakker tensor t1 I + t2 r r^T / r^2, with
    the overlap form for r <= 2 (shear/src/main26.c:1727-1741)."""
    rr = np.asarray(rr, dtype=float)
    r = np.sqrt(rr)
    a = alpha
    a3, a5, a7 = a ** 3, a ** 5, a ** 7
    far = r > 2.0
    C1 = np.where(far, 0.75 / r + 0.5 / (r * rr), 1.0 - 0.28125 * r)
    C2 = np.where(far, 4 * a7 * rr * rr + 3 * a3 * rr - 20 * a5 * rr - 4.5 * a + 14 * a3 + a / rr,
                  64 * a7 + 12 * a3 - 80 * a5 - 4.5 * a + 14 * a3 + 0.25 * a)
    C3 = np.where(far, 0.75 / r - 1.5 / (r * rr), 0.09375 * r)
    C4 = np.where(far, -4 * a7 * rr * rr - 3 * a3 * rr + 16 * a5 * rr + 1.5 * a - 2 * a3 - 3 * a / rr,
                  -64 * a7 - 12 * a3 + 64 * a5 + 1.5 * a - 2 * a3 - 0.75 * a)
    ec = erfc(a * r)
    ex = np.exp(-a * a * rr) / math.sqrt(math.pi)
    return C1 * ec + C2 * ex, C3 * ec + C4 * ex


def real_terms_far(alpha, rr):
    """t1, t2 of the real-space tensor in its r > 2 form at any r > 0."""
    rr = np.asarray(rr, dtype=float)
    r = np.sqrt(rr)
    a = alpha
    a3, a5, a7 = a ** 3, a ** 5, a ** 7
    C1 = 0.75 / r + 0.5 / (r * rr)
    C2 = 4 * a7 * rr * rr + 3 * a3 * rr - 20 * a5 * rr - 4.5 * a + 14 * a3 + a / rr
    C3 = 0.75 / r - 1.5 / (r * rr)
    C4 = -4 * a7 * rr * rr - 3 * a3 * rr + 16 * a5 * rr + 1.5 * a - 2 * a3 - 3 * a / rr
    ec = erfc(a * r)
    ex = np.exp(-a * a * rr) / math.sqrt(math.pi)
    return C1 * ec + C2 * ex, C3 * ec + C4 * ex


def ref_alpha(t, tp, L2yp, M_HI=4.0):
    """The split parameter calcHI uses at step t: M_HI / rce with rce = L2yp
    in the first half of the lattice period and 2 L2yp in the second
    (shear/src/main26.c:1536-1552)."""
    treal = int(t % tp)
    rce = L2yp if treal <= tp // 2 else 2.0 * L2yp
    return M_HI / rce


def phi_k(alpha, kk):
    """k-space coefficient (1 - k^2/3)(1 + k^2/4a^2 + k^4/8a^4) 6 pi/k^2
    exp(-k^2/4a^2) (shear/src/main26.c:1602-1622 without the factor 2 of the
    half-space sum)."""
    a2 = alpha * alpha
    return (1 - kk / 3) * (1 + kk / (4 * a2) + kk * kk / (8 * a2 * a2)) * 6 * math.pi / kk * np.exp(-kk / (4 * a2))


def self_const(alpha):
    return 1 - 6 / math.sqrt(math.pi) * alpha + 40 / (3 * math.sqrt(math.pi)) * alpha ** 3


def _widths(H):
    V = abs(np.linalg.det(H))
    a = H.T
    return np.array([V / np.linalg.norm(np.cross(a[(j + 1) % 3], a[(j + 2) % 3])) for j in range(3)])


def ewald_apply(H, pos, v, alpha=None, tol_exp=20.0):
    """M v by the Ewald sum.  pos: (N, 3) lab-frame positions, v: (N, 3).
    alpha defaults to 4 / (half the narrowest cell width); the real-space
    cutoff and k-space cutoff are set so the neglected terms are below
    exp(-tol_exp)."""
    pos = np.asarray(pos, float)
    v = np.asarray(v, float)
    N = len(pos)
    H = np.asarray(H, float)
    Hi = np.linalg.inv(H)
    V = abs(np.linalg.det(H))
    w = _widths(H)
    if alpha is None:
        alpha = 4.0 / (0.5 * w.min())
    rcut = math.sqrt(tol_exp) / alpha
    kcut = 2 * alpha * math.sqrt(tol_exp)
    out = self_const(alpha) * v.copy()
    # real space: all images within rcut (self images included, n != 0)
    nimg = [int(math.ceil(rcut / w[d])) + 1 for d in range(3)]
    shifts = np.array([[i, j, k] for i in range(-nimg[0], nimg[0] + 1)
                       for j in range(-nimg[1], nimg[1] + 1)
                       for k in range(-nimg[2], nimg[2] + 1)], dtype=float) @ H.T
    for i in range(N):
        d = pos[None, :, :] - pos[i][None, None, :] + shifts[:, None, :]  # (S, N, 3)
        rr = np.einsum("snk,snk->sn", d, d)
        mask = (rr < rcut * rcut) & (rr > 0)
        rrm = np.where(mask, rr, 1.0)
        t1, t2 = real_terms(alpha, rrm)
        t1 = np.where(mask, t1, 0.0)
        t2 = np.where(mask, t2 / rrm, 0.0)
        dv = np.einsum("snk,nk->sn", d, v)
        out[i] += np.einsum("sn,nk->k", t1, v) + np.einsum("sn,sn,snk->k", t2, dv, d)
    # k space: m = integer triples with |k| < kcut, k = 2 pi Hi^T m
    B = 2 * math.pi * Hi.T  # columns b_d: k = B m
    mmax = [int(math.ceil(kcut / (2 * math.pi) * np.linalg.norm(H[:, d]))) + 1 for d in range(3)]
    g = np.mgrid[-mmax[0]:mmax[0] + 1, -mmax[1]:mmax[1] + 1, -mmax[2]:mmax[2] + 1].reshape(3, -1).T
    k = g @ B.T
    kk = np.einsum("ij,ij->i", k, k)
    keep = (kk > 0) & (kk < kcut * kcut)
    k, kk = k[keep], kk[keep]
    f = phi_k(alpha, kk) / V
    for s in range(0, len(k), 2048):
        ks, kks, fs = k[s:s + 2048], kk[s:s + 2048], f[s:s + 2048]
        ph = pos @ ks.T  # (N, nk)
        c, sn = np.cos(ph), np.sin(ph)
        Sc = c.T @ v  # (nk, 3) sum_j cos(k r_j) v_j
        Ss = sn.T @ v
        # (I - k k^T/k^2) applied to the structure factors
        Pc = Sc - ks * (np.einsum("ij,ij->i", ks, Sc) / kks)[:, None]
        Ps = Ss - ks * (np.einsum("ij,ij->i", ks, Ss) / kks)[:, None]
        out += c @ (fs[:, None] * Pc) + sn @ (fs[:, None] * Ps)
    return out


def self_block(H, alpha=None, tol_exp=20.0):
    """The 3x3 diagonal block M_ii (the same for every bead): self constant,
    real-space self images and the k-space sum at r = 0."""
    H = np.asarray(H, float)
    e = np.zeros((1, 3))
    cols = []
    for a in range(3):
        v = np.zeros((1, 3))
        v[0, a] = 1.0
        cols.append(ewald_apply(H, e, v, alpha, tol_exp)[0])
    return np.array(cols).T


def self_offdiag(H, alpha=None, tol_exp=20.0):
    """Off-diagonal part of the self block (real-space self images and the
    k-space sum), the entries calcHI does not store."""
    S = self_block(H, alpha, tol_exp)
    np.fill_diagonal(S, 0.0)
    return S


def bspline_weights(f, p):
    """w[k] = M_p(f + k), k = 0..p-1 (cardinal B-spline of order p)."""
    a = np.array([f, 1.0 - f])
    for n in range(3, p + 1):
        b = np.zeros(n)
        for k in range(n):
            hi = a[k] if k < n - 1 else 0.0
            lo = a[k - 1] if k >= 1 else 0.0
            b[k] = ((f + k) * hi + (n - f - k) * lo) / (n - 1)
        a = b
    return a


def bspline_moduli(K, p):
    """|b(m)|^2 = 1 / |sum_{k=0}^{p-2} M_p(k + 1) exp(2 pi i m k / K)|^2."""
    Mk = bspline_weights(0.0, p)  # M_p(k), k = 0..p-1
    m = np.arange(K)
    s = sum(Mk[k + 1] * np.exp(2j * math.pi * m * k / K) for k in range(p - 1))
    d = np.abs(s) ** 2
    return np.where(d > 1e-300, 1.0 / np.maximum(d, 1e-300), 0.0)


def pme_apply(H, pos, v, K, p, alpha, rc, alpha_ref=None, ref_self=True):
    """M v by smooth PME with the same discretisation as the CUDA path:
    real-space pairs within rc (minimum image), self constant, and the
    reciprocal sum by spreading / FFT / influence / interpolation (the
    bead's own term included, as in the Ewald k-space sum).

    calcHI's tensor for overlapping beads (r < 2) depends on its split
    parameter; with alpha_ref the pairs closer than 2 get that dependence at
    alpha_ref instead of alpha, so the sum reproduces calcHI at alpha_ref.
    With ref_self the off-diagonal entries of the self block, which calcHI
    does not store, are removed."""
    pos = np.asarray(pos, float)
    v = np.asarray(v, float)
    N = len(pos)
    H = np.asarray(H, float)
    Hi = np.linalg.inv(H)
    V = abs(np.linalg.det(H))
    s = pos @ Hi.T
    s -= np.floor(s)
    u = s * K
    base = np.floor(u).astype(int)
    fr = u - base
    base %= K
    W = np.zeros((N, 3, p))
    for i in range(N):
        for d in range(3):
            W[i, d] = bspline_weights(fr[i, d], p)
    Q = np.zeros((3, K, K, K))
    idx = [(base[:, d][:, None] - np.arange(p)[None, :]) % K for d in range(3)]  # (N, p)
    wt = W[:, 0, :, None, None] * W[:, 1, None, :, None] * W[:, 2, None, None, :]  # (N,p,p,p)
    g0 = idx[0][:, :, None, None]
    g1 = idx[1][:, None, :, None]
    g2 = idx[2][:, None, None, :]
    for c in range(3):
        np.add.at(Q[c], (np.broadcast_to(g0, wt.shape), np.broadcast_to(g1, wt.shape),
                         np.broadcast_to(g2, wt.shape)), wt * v[:, c][:, None, None, None])
    F = np.fft.rfftn(Q, axes=(1, 2, 3))
    m0 = np.fft.fftfreq(K, 1.0 / K)
    m2 = np.arange(K // 2 + 1)
    M0, M1, M2 = np.meshgrid(m0, m0, m2, indexing="ij")
    k = 2 * math.pi * (M0[..., None] * Hi[0] + M1[..., None] * Hi[1] + M2[..., None] * Hi[2])
    kk = np.einsum("...i,...i->...", k, k)
    kk0 = np.where(kk > 0, kk, 1.0)
    bsq = bspline_moduli(K, p)
    f = phi_k(alpha, kk0) / V * bsq[np.arange(K)][:, None, None] * bsq[np.arange(K)][None, :, None] \
        * bsq[m2][None, None, :]
    f = np.where(kk > 0, f, 0.0)
    kF = sum(k[..., a] * F[a] for a in range(3))
    G = np.stack([f * (F[a] - k[..., a] * kF / kk0) for a in range(3)])
    Qb = np.fft.irfftn(G, s=(K, K, K), axes=(1, 2, 3)) * (K ** 3)
    out = np.zeros((N, 3))
    for c in range(3):
        out[:, c] = np.einsum("nabc,nabc->n", wt, Qb[c][g0, g1, g2])
    out += self_const(alpha) * v
    # real space within rc, lattice minimum image by fractional rounding
    for i in range(N):
        d = pos - pos[i]
        sd = d @ Hi.T
        sd -= np.rint(sd)
        d = sd @ H.T
        rr = np.einsum("nk,nk->n", d, d)
        mask = (rr < rc * rc) & (np.arange(N) != i)
        if not mask.any():
            continue
        dm, rrm = d[mask], rr[mask]
        t1, t2 = real_terms(alpha, rrm)
        if alpha_ref is not None:
            a1, a2 = real_terms(alpha_ref, rrm)
            b1, b2 = real_terms_far(alpha_ref, rrm)
            c1, c2 = real_terms_far(alpha, rrm)
            ovl = rrm < 4.0
            t1 = np.where(ovl, c1 + a1 - b1, t1)
            t2 = np.where(ovl, c2 + a2 - b2, t2)
        dv = np.einsum("nk,nk->n", dm, v[mask])
        out[i] += t1 @ v[mask] + (t2 / rrm * dv) @ dm
    if ref_self:
        # the k-space self sum's off-diagonal entries over the grid's own
        # half spectrum (multiplicity 2 off the m2 = 0 and Nyquist planes)
        mult = np.where((m2 == 0) | ((K % 2 == 0) & (m2 == K // 2)), 1.0, 2.0)[None, None, :]
        ph = np.where(kk > 0, phi_k(alpha, kk0) / V, 0.0) * mult
        w = (ph / kk0).reshape(-1)
        kf = k.reshape(-1, 3)
        S = -np.einsum("n,na,nb->ab", w, kf, kf)
        np.fill_diagonal(S, 0.0)
        out -= v @ S.T
    return out


def recip_self_offdiag(H, alpha, tol_exp=20.0):
    """Off-diagonal part of sum_{k != 0} (phi(k)/V)(I - k k^T/k^2): the self
    block's off-diagonal entries (the real-space self images beyond a
    cutoff below half the narrowest width are negligible)."""
    H = np.asarray(H, float)
    Hi = np.linalg.inv(H)
    V = abs(np.linalg.det(H))
    kcut = 2 * alpha * math.sqrt(tol_exp)
    B = 2 * math.pi * Hi.T
    mmax = [int(math.ceil(kcut / (2 * math.pi) * np.linalg.norm(H[:, d]))) + 1 for d in range(3)]
    g = np.mgrid[-mmax[0]:mmax[0] + 1, -mmax[1]:mmax[1] + 1, -mmax[2]:mmax[2] + 1].reshape(3, -1).T
    k = g @ B.T
    kk = np.einsum("ij,ij->i", k, k)
    keep = (kk > 0) & (kk < kcut * kcut)
    k, kk = k[keep], kk[keep]
    f = phi_k(alpha, kk) / V
    S = -np.einsum("n,na,nb->ab", f / kk, k, k)
    np.fill_diagonal(S, 0.0)
    return S
