"""Seeded initial fields for the benchmark and test workloads.

Built with torch on any device (setup work, not part of the flow step).  Every
builder returns a flat tensor in the reference layout ``idx = y + x*ylen +
a*xlen*ylen`` and takes the resolved parameters ``rp`` of the theory.  Noise is
N(0, sigma) from a seeded ``numpy.random.default_rng``-independent torch generator
so that the same seed gives the same field on CPU and GPU.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _coords(rp, device, dtype=torch.float64):
    x = torch.arange(rp.xlen, device=device, dtype=dtype)[:, None] * rp.lsx
    y = torch.arange(rp.ylen, device=device, dtype=dtype)[None, :] * rp.lsy
    return x.expand(rp.xlen, rp.ylen), y.expand(rp.xlen, rp.ylen)


def _noise(shape, sigma, seed, device):
    if sigma == 0.0:
        return torch.zeros(shape, dtype=torch.float64, device=device)
    g = np.random.default_rng(seed)
    return torch.from_numpy(g.standard_normal(shape)).to(device) * sigma


def _finish_unit(m, rp, sigma, seed, device, ring=True):
    """Add noise to every component, renormalise, and set the 2-cell ring to the vacuum (0,0,1)."""
    m = m + _noise(m.shape, sigma, seed, device)
    m = m / torch.sqrt((m * m).sum(0, keepdim=True))
    if ring:
        h = int(rp.halo)
        for a, v in enumerate((0.0, 0.0, 1.0)):
            m[a, :h, :] = v
            m[a, -h:, :] = v
            m[a, :, :h] = v
            m[a, :, -h:] = v
    return m


def hedgehog(rp, charge=1, R=1.5, center=None, sigma=1e-3, seed=0, device="cpu"):
    """Baby Skyrme hedgehog m = (sin f cos B theta, sin f sin B theta, cos f), f = pi exp(-r/R)."""
    x, y = _coords(rp, device)
    cx, cy = center if center is not None else (0.5 * (rp.xlen - 1) * rp.lsx, 0.5 * (rp.ylen - 1) * rp.lsy)
    dx, dy = x - cx, y - cy
    r = torch.sqrt(dx * dx + dy * dy)
    th = torch.atan2(dy, dx)
    f = math.pi * torch.exp(-r / R)
    m = torch.stack([torch.sin(f) * torch.cos(charge * th), torch.sin(f) * torch.sin(charge * th), torch.cos(f)])
    return _finish_unit(m, rp, sigma, seed, device).reshape(-1)


def _anti(dx, dy, R):
    r = torch.sqrt(dx * dx + dy * dy)
    th = torch.atan2(dy, dx)
    f = math.pi * torch.exp(-r / R)
    # the reference's "anti" ansatz (chiral_magnet/initial_config.py, ansatz_anti branch)
    return torch.stack([-torch.sin(f) * torch.sin(th), -torch.sin(f) * torch.cos(th), torch.cos(f)])


def anti_skyrmion(rp, R=1.0, sigma=1e-3, seed=0, device="cpu"):
    """Chiral magnet anti-skyrmion at the centre, psi = 0 (4 components)."""
    x, y = _coords(rp, device)
    cx, cy = 0.5 * (rp.xlen - 1) * rp.lsx, 0.5 * (rp.ylen - 1) * rp.lsy
    m = _finish_unit(_anti(x - cx, y - cy, R), rp, sigma, seed, device)
    psi = torch.zeros((1, rp.xlen, rp.ylen), dtype=torch.float64, device=device)
    return torch.cat([m, psi]).reshape(-1)


def skyrmion_lattice(rp, n=8, R=1.0, jitter=0.25, sigma=1e-3, seed=0, device="cpu"):
    """n x n anti-skyrmions at seeded jittered lattice positions, composed by adding
    their stereographic coordinates w = (m1 + i m2)/(1 + m3) as the reference's
    create_skyrmion_kernel does (chiral_magnet/initial_config.py:286-386); psi = 0."""
    x, y = _coords(rp, device)
    g = np.random.default_rng(seed)
    Lx, Ly = (rp.xlen - 1) * rp.lsx, (rp.ylen - 1) * rp.lsy
    wr = torch.zeros_like(x)
    wi = torch.zeros_like(x)
    eps = 1e-12
    for i in range(n):
        for j in range(n):
            cx = (i + 0.5 + jitter * (g.random() - 0.5)) * Lx / n
            cy = (j + 0.5 + jitter * (g.random() - 0.5)) * Ly / n
            m = _anti(x - cx, y - cy, R)
            den = torch.clamp(1.0 + m[2], min=eps)
            wr = wr + m[0] / den
            wi = wi + m[1] / den
    nw = wr * wr + wi * wi
    m = torch.stack([2 * wr / (1 + nw), 2 * wi / (1 + nw), (1 - nw) / (1 + nw)])
    m = _finish_unit(m, rp, sigma, seed + 1, device)
    psi = torch.zeros((1, rp.xlen, rp.ylen), dtype=torch.float64, device=device)
    return torch.cat([m, psi]).reshape(-1)


def vortices(rp, n=4, sigma=0.0, seed=0, device="cpu"):
    """Abelian Higgs: n unit-winding vortices at seeded uniform positions in the
    central half, psi = u1 * prod tanh(r_i) e^{i theta_i}, A = 0."""
    x, y = _coords(rp, device)
    g = np.random.default_rng(seed)
    Lx, Ly = (rp.xlen - 1) * rp.lsx, (rp.ylen - 1) * rp.lsy
    re = torch.ones_like(x)
    im = torch.zeros_like(x)
    for _ in range(n):
        cx = (0.25 + 0.5 * g.random()) * Lx
        cy = (0.25 + 0.5 * g.random()) * Ly
        dx, dy = x - cx, y - cy
        r = torch.sqrt(dx * dx + dy * dy)
        th = torch.atan2(dy, dx)
        amp = torch.tanh(r)
        zr, zi = amp * torch.cos(th), amp * torch.sin(th)
        re, im = re * zr - im * zi, re * zi + im * zr
    u = float(getattr(rp, "u1", 1.0))
    F = torch.stack([torch.zeros_like(x), torch.zeros_like(x), u * re, u * im])
    if sigma:
        F = F + _noise(F.shape, sigma, seed + 1, device)
    return F.reshape(-1)


def vortex(rp, winding=1, center=None, device="cpu"):
    """Abelian Higgs: one vortex of winding n at `center` (default: the lattice centre),
    psi = u1 tanh(r)^|n| e^{i n theta}, A = 0 (a coalesced n-vortex for |n| > 1)."""
    x, y = _coords(rp, device)
    cx, cy = center if center is not None else (0.5 * (rp.xlen - 1) * rp.lsx, 0.5 * (rp.ylen - 1) * rp.lsy)
    dx, dy = x - cx, y - cy
    r = torch.sqrt(dx * dx + dy * dy)
    th = torch.atan2(dy, dx)
    amp = float(getattr(rp, "u1", 1.0)) * torch.tanh(r) ** abs(winding)
    F = torch.stack([torch.zeros_like(x), torch.zeros_like(x), amp * torch.cos(winding * th),
                     amp * torch.sin(winding * th)])
    return F.reshape(-1)
