"""Exact solution of the 1D ideal-gas Riemann problem — TEST INFRASTRUCTURE.

Restates the exact Sod solver the reference uses for validation
(share/spearhed/ValidationSetups/SodShockTube/validate_sod.py:31-168, exact_sod):
the star-region pressure solves f_L(p) + f_R(p) + (u_R - u_L) = 0 with the
shock / rarefaction branches of each wave, by Newton iteration from the
two-rarefaction estimate; the solution is then sampled in x/t.  The golden
vectors in tests/golden/exact_sod.npz, produced by the reference's own solver,
pin this restatement.  Only tests/ import it.
"""
from __future__ import annotations

import numpy as np


def _wave(p, rho_k, p_k, g):
    """Jump function of one wave and its derivative in p."""
    c_k = np.sqrt(g * p_k / rho_k)
    if p > p_k:  # shock
        A = 2.0 / ((g + 1.0) * rho_k)
        B = (g - 1.0) / (g + 1.0) * p_k
        q = np.sqrt(A / (p + B))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (p + B))
    # rarefaction
    e = (g - 1.0) / (2.0 * g)
    return 2.0 * c_k / (g - 1.0) * ((p / p_k) ** e - 1.0), (p / p_k) ** (-(g + 1.0) / (2.0 * g)) / (rho_k * c_k)


def star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, g):
    c_l, c_r = np.sqrt(g * p_l / rho_l), np.sqrt(g * p_r / rho_r)
    e = (g - 1.0) / (2.0 * g)
    p = ((c_l + c_r - 0.5 * (g - 1.0) * (u_r - u_l)) / (c_l / p_l ** e + c_r / p_r ** e)) ** (1.0 / e)
    for _ in range(100):
        fl, dl = _wave(p, rho_l, p_l, g)
        fr, dr = _wave(p, rho_r, p_r, g)
        dp = (fl + fr + u_r - u_l) / (dl + dr)
        p = max(p - dp, 1e-14)
        if abs(dp) < 1e-12 * p:
            break
    fl, _ = _wave(p, rho_l, p_l, g)
    fr, _ = _wave(p, rho_r, p_r, g)
    u = 0.5 * (u_l + u_r) + 0.5 * (fr - fl)
    return p, u


def solve(x, t, gamma=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    """(rho, u, p, e) at positions x (interface at 0) and time t > 0."""
    rho_l, u_l, p_l = left
    rho_r, u_r, p_r = right
    g = gamma
    ps, us = star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, g)
    c_l, c_r = np.sqrt(g * p_l / rho_l), np.sqrt(g * p_r / rho_r)
    gm = (g - 1.0) / (g + 1.0)
    x = np.asarray(x, dtype=np.float64)
    s = x / t
    rho = np.empty_like(s)
    u = np.empty_like(s)
    p = np.empty_like(s)
    for i, xi in enumerate(s):
        if xi < us:  # left of the contact
            if ps > p_l:
                sl = u_l - c_l * np.sqrt((g + 1.0) / (2.0 * g) * ps / p_l + (g - 1.0) / (2.0 * g))
                if xi < sl:
                    rho[i], u[i], p[i] = rho_l, u_l, p_l
                else:
                    rho[i], u[i], p[i] = rho_l * (ps / p_l + gm) / (gm * ps / p_l + 1.0), us, ps
            else:
                cs = c_l * (ps / p_l) ** ((g - 1.0) / (2.0 * g))
                if xi < u_l - c_l:
                    rho[i], u[i], p[i] = rho_l, u_l, p_l
                elif xi > us - cs:
                    rho[i], u[i], p[i] = rho_l * (ps / p_l) ** (1.0 / g), us, ps
                else:
                    uf = 2.0 / (g + 1.0) * (c_l + 0.5 * (g - 1.0) * u_l + xi)
                    cf = 2.0 / (g + 1.0) * (c_l + 0.5 * (g - 1.0) * (u_l - xi))
                    pf = p_l * (cf / c_l) ** (2.0 * g / (g - 1.0))
                    rho[i], u[i], p[i] = g * pf / cf ** 2, uf, pf
        else:  # right of the contact
            if ps > p_r:
                sr = u_r + c_r * np.sqrt((g + 1.0) / (2.0 * g) * ps / p_r + (g - 1.0) / (2.0 * g))
                if xi > sr:
                    rho[i], u[i], p[i] = rho_r, u_r, p_r
                else:
                    rho[i], u[i], p[i] = rho_r * (ps / p_r + gm) / (gm * ps / p_r + 1.0), us, ps
            else:
                cs = c_r * (ps / p_r) ** ((g - 1.0) / (2.0 * g))
                if xi > u_r + c_r:
                    rho[i], u[i], p[i] = rho_r, u_r, p_r
                elif xi < us + cs:
                    rho[i], u[i], p[i] = rho_r * (ps / p_r) ** (1.0 / g), us, ps
                else:
                    uf = 2.0 / (g + 1.0) * (-c_r + 0.5 * (g - 1.0) * u_r + xi)
                    cf = 2.0 / (g + 1.0) * (c_r - 0.5 * (g - 1.0) * (u_r - xi))
                    pf = p_r * (cf / c_r) ** (2.0 * g / (g - 1.0))
                    rho[i], u[i], p[i] = g * pf / cf ** 2, uf, pf
    return rho, u, p, p / ((g - 1.0) * rho)


def binned_l1(x_particles, fields, t, gamma, lo, hi, bins):
    """L1 errors of bin-averaged particle fields against the exact solution,
    binned along x over [lo, hi] like validate_sod.py:205-262."""
    edges = np.linspace(lo, hi, bins + 1)
    centres = 0.5 * (edges[:-1] + edges[1:])
    idx = np.clip(np.digitize(x_particles, edges) - 1, 0, bins - 1)
    inside = (x_particles >= lo) & (x_particles <= hi)
    cnt = np.bincount(idx[inside], minlength=bins).astype(float)
    ex = dict(zip(("rho", "u", "p", "e"), solve(centres, t, gamma)))
    out = {}
    for name, vals in fields.items():
        sums = np.bincount(idx[inside], weights=vals[inside], minlength=bins)
        m = cnt > 0
        out[name] = float(np.mean(np.abs(sums[m] / cnt[m] - ex[name][m])))
    return out
