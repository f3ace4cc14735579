"""FP64 torch restatement of the chained hot path, for reference gradients.

TEST INFRASTRUCTURE ONLY (oracle): the product never imports it. torch autograd over
this restatement gives the FP64 reference gradient the hand-written CUDA adjoint is
checked against; the restatement itself is pinned to the C oracle (p2r_oracle.cpp) and,
through it, to the reference's own CPU path.

Follows src/propagate-tor-test_tbb.cpp of cerati/p2r-tests ("TBB"):
  propagateToR  TBB:656-812     KalmanUpdate  TBB:433-642     sincos4  TBB:644-652
with the extensions of the C oracle: target radius hipo(hit) + dr[layer], run-time
kfact = 100/(-0.299792458*bz), chi2 = res^T inv(R) res summed over layers. Vectorised
over tracks; the convergence branch of the path derivatives (TBB:714) is a torch.where
(held fixed by autograd, like the CUDA adjoint).
"""
from __future__ import annotations

import torch


def _S6(i: int, j: int) -> int:
    return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i


def _sincos4(x):
    x2 = x * x
    omc = 0.5 * x2 - 0.04166667 * x2 * x2  # the float literals of TBB:650-651, widened
    return x - 0.16666667 * x * x2, 1.0 - omc, omc


def propagate(par, cov, k, r):
    """One propagateToR of every track (par (n,6), cov (n,21), k (n,), r (n,))."""
    x, y, z, ipt, phi, theta = par.unbind(1)
    kinv = 1.0 / k
    r0 = torch.sqrt(x * x + y * y)
    pt = 1.0 / ipt
    cosP, sinP = torch.cos(phi), torch.sin(phi)
    px, py = cosP * pt, sinP * pt
    pos = r0 > 0
    safe_r0 = torch.where(pos, r0, torch.ones_like(r0))
    dDdx = torch.where(pos, -x / safe_r0, torch.zeros_like(x))
    dDdy = torch.where(pos, -y / safe_r0, torch.zeros_like(y))
    dDdipt = torch.zeros_like(x)
    dDdphi = torch.zeros_like(x)
    D = torch.zeros_like(x)
    xo, yo = x, y
    for i in range(5):
        r0 = torch.sqrt(xo * xo + yo * yo)
        idd = r - r0
        D = D + idd
        sina, cosa, omc = _sincos4(idd * ipt * kinv)
        if i + 1 != 5:
            cond = (r0 > 0) & (torch.abs(r - r0) < 0.0001)
            oor0 = torch.where(cond, 1.0 / torch.where(cond, r0, torch.ones_like(r0)), torch.zeros_like(r0))
            dadipt = idd * kinv
            dadx = -xo * ipt * kinv * oor0
            dady = -yo * ipt * kinv * oor0
            pxca, pxsa, pyca, pysa = px * cosa, px * sina, py * cosa, py * sina
            tmp = k * dadx
            dDdx = dDdx - (xo * (1 + tmp * (pxca - pysa)) + yo * tmp * (pyca + pxsa)) * oor0
            tmp = k * dady
            dDdy = dDdy - (xo * tmp * (pxca - pysa) + yo * (1 + tmp * (pyca + pxsa))) * oor0
            tmp = dadipt * ipt
            dDdipt = dDdipt - k * (xo * (pxca * tmp - pysa * tmp - pyca - pxsa + py) +
                                   yo * (pyca * tmp + pxsa * tmp - pysa + pxca - px)) * pt * oor0
            dDdphi = dDdphi + k * (xo * (pysa - px + pxca) - yo * (pxsa - py + pyca)) * oor0
        xo = xo + k * (px * sina - py * omc)
        yo = yo + k * (py * sina + px * omc)
        px, py = px * cosa - py * sina, py * cosa + px * sina
    alpha = D * ipt * kinv
    dadx = dDdx * ipt * kinv
    dady = dDdy * ipt * kinv
    dadipt = (ipt * dDdipt + D) * kinv
    dadphi = dDdphi * ipt * kinv
    sina, cosa, omc = _sincos4(alpha)
    cosT, sinT = torch.cos(theta), torch.sin(theta)
    isT = 1.0 / sinT
    zero, one = torch.zeros_like(x), torch.ones_like(x)
    J = [[None] * 6 for _ in range(6)]
    for a in range(6):
        for b in range(6):
            J[a][b] = zero
    J[0][0] = 1 + k * dadx * (cosP * cosa - sinP * sina) * pt
    J[0][1] = k * dady * (cosP * cosa - sinP * sina) * pt
    J[0][3] = k * (cosP * (ipt * dadipt * cosa - sina) + sinP * (omc - ipt * dadipt * sina)) * pt * pt
    J[0][4] = k * (cosP * dadphi * cosa - sinP * dadphi * sina - sinP * sina + cosP * cosa - cosP) * pt
    J[1][0] = k * dadx * (sinP * cosa + cosP * sina) * pt
    J[1][1] = 1 + k * dady * (sinP * cosa + cosP * sina) * pt
    J[1][3] = k * (sinP * (ipt * dadipt * cosa - sina) + cosP * (ipt * dadipt * sina - omc)) * pt * pt
    J[1][4] = k * (sinP * dadphi * cosa + cosP * dadphi * sina + sinP * cosa + cosP * sina - sinP) * pt
    J[2][0] = k * cosT * dadx * pt * isT
    J[2][1] = k * cosT * dady * pt * isT
    J[2][2] = one
    J[2][3] = k * cosT * (ipt * dadipt - alpha) * pt * pt * isT
    J[2][4] = k * dadphi * cosT * pt * isT
    J[2][5] = -k * alpha * pt * isT * isT
    J[3][3] = one
    J[4][0], J[4][1], J[4][3], J[4][4] = dadx, dady, dadipt, 1 + dadphi
    J[5][5] = one
    Jm = torch.stack([torch.stack(row, 1) for row in J], 1)  # (n,6,6)
    C = torch.stack([torch.stack([cov[:, _S6(i, j)] for j in range(6)], 1) for i in range(6)], 1)
    Cn = Jm @ C @ Jm.transpose(1, 2)
    ncov = torch.stack([Cn[:, i, j] for i in range(6) for j in range(i + 1)], 1)
    npar = torch.stack([xo, yo, z + k * alpha * cosT * pt * isT, ipt, phi + alpha, theta], 1)
    return npar, ncov


def update(par, cov, hpos, hcov):
    """One KalmanUpdate of every track; returns (par, cov, chi2)."""
    hx, hy, hz = hpos.unbind(1)
    x, y, z = par[:, 0], par[:, 1], par[:, 2]
    r = torch.sqrt(hx * hx + hy * hy)
    R00 = -(hy + y) / (2 * r)
    R01 = (hx + x) / (2 * r)
    A = cov[:, :6] + hcov
    e0 = (R00 * A[:, 0] + R01 * A[:, 1]) * R00 + (R00 * A[:, 1] + R01 * A[:, 2]) * R01
    e1 = A[:, 3] * R00 + A[:, 4] * R01
    e2 = A[:, 5]
    s = 1.0 / (e0 * e2 - e1 * e1)
    i0, i1, i2 = s * e2, -s * e1, s * e0
    c = lambda i, j: cov[:, _S6(i, j)]
    K0 = torch.stack([c(m, 0) * (R00 * i0) + c(m, 1) * (R01 * i0) + c(m, 2) * i1 for m in range(6)], 1)
    K1 = torch.stack([c(m, 0) * (R00 * i1) + c(m, 1) * (R01 * i1) + c(m, 2) * i2 for m in range(6)], 1)
    res0 = R00 * (hx - x) + R01 * (hy - y)
    res1 = hz - z
    chi2 = i0 * res0 * res0 + 2 * i1 * res0 * res1 + i2 * res1 * res1
    npar = par + K0 * res0[:, None] + K1 * res1[:, None]
    ncov = torch.stack([c(i, j) - (K0[:, i] * R00 * c(0, j) + K0[:, i] * R01 * c(1, j) + K1[:, i] * c(2, j))
                        for i in range(6) for j in range(i + 1)], 1)
    return npar, ncov, chi2


def chained(par0, cov0, q, hpos, hcov, dr, bz, nlay=None):
    """All layers, chained. par0 (n,6), cov0 (n,21), q (n,), hpos (n,L,3), hcov (n,L,6),
    dr (L,), bz (0-dim). nlay (n,) optional per-track layer counts.
    Returns (par, cov, chi2 summed over layers)."""
    kfact = 100.0 / (-0.299792458 * bz)
    k = q.to(par0.dtype) * kfact
    par, cov = par0, cov0
    chi2 = torch.zeros(par0.shape[0], dtype=par0.dtype, device=par0.device)
    for l in range(hpos.shape[1]):
        hp, hc = hpos[:, l], hcov[:, l]
        r = torch.sqrt(hp[:, 0] ** 2 + hp[:, 1] ** 2) + dr[l]
        p2, c2 = propagate(par, cov, k, r)
        p3, c3, x2 = update(p2, c2, hp, hc)
        if nlay is None:
            par, cov, chi2 = p3, c3, chi2 + x2
        else:
            live = (l < nlay)[:, None]
            par = torch.where(live, p3, par)
            cov = torch.where(live, c3, cov)
            chi2 = chi2 + torch.where(live[:, 0], x2, torch.zeros_like(x2))
    return par, cov, chi2
