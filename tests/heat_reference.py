"""Quadrature references for the Gaussian heat source with zero boundary data.

At the centre of a disk / ball of radius R the solution of -Δu = f, u = 0 on
the boundary, is u(0) = ∫ G(0, y) f(y) dy with G(0, y) = ln(R/|y|) / (2π)
(2D) or (1/|y| - 1/R) / (4π) (3D).  For f = Q exp(-|y - x0|^2 / sigma^2) the
derivatives with respect to (Q, x0, sigma) are the integrals of G times
f/Q, f 2 (y - x0)/sigma^2 and f 2 |y - x0|^2 / sigma^3.  Computed with
Gauss-Legendre rules in the radius (and polar cosine) and the trapezoidal
rule in the azimuth.
"""
from __future__ import annotations

import numpy as np


def _terms(Y, x0, Q, sigma):
    d = Y - np.asarray(x0, dtype=np.float64)
    q = (d ** 2).sum(-1) / sigma ** 2
    f = Q * np.exp(-q)
    dQ = f / Q
    dx0 = f[..., None] * 2.0 * d / sigma ** 2
    dsig = f * 2.0 * q / sigma
    return f, dQ, dx0, dsig


def centre_value(dim: int, R: float, Q: float, x0, sigma: float, nr: int = 400,
                 nphi: int = 256, nt: int = 200) -> dict:
    """u(0) and du(0)/d(Q, x0, sigma) for the disk (dim 2) or ball (dim 3)."""
    x0 = np.asarray(x0, dtype=np.float64)
    gr, wr = np.polynomial.legendre.leggauss(nr)
    r = 0.5 * R * (gr + 1.0)
    wr = 0.5 * R * wr
    phi = np.arange(nphi) * (2 * np.pi / nphi)
    wphi = 2 * np.pi / nphi
    if dim == 2:
        rr, pp = np.meshgrid(r, phi, indexing="ij")
        Y = np.stack([rr * np.cos(pp), rr * np.sin(pp)], -1)
        G = np.log(R / rr) / (2 * np.pi)
        W = (wr[:, None] * wphi) * rr * G
    else:
        ct, wt = np.polynomial.legendre.leggauss(nt)
        rr, cc, pp = np.meshgrid(r, ct, phi, indexing="ij")
        st = np.sqrt(1.0 - cc ** 2)
        Y = np.stack([rr * st * np.cos(pp), rr * st * np.sin(pp), rr * cc], -1)
        G = (1.0 / rr - 1.0 / R) / (4 * np.pi)
        W = (wr[:, None, None] * wt[None, :, None] * wphi) * rr ** 2 * G
    f, dQ, dx0, dsig = _terms(Y, x0[:dim], Q, sigma)
    jac = np.zeros(5)
    jac[0] = (W * dQ).sum()
    jac[1:1 + dim] = (W[..., None] * dx0).reshape(-1, dim).sum(0)
    jac[4] = (W * dsig).sum()
    return {"u": float((W * f).sum()), "jacobian": jac}
