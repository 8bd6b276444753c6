"""FP64 CPU restatement of soliton_solver's flow hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against; it is imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` and by nothing else.  The product
path (``soliton_solver_b200``) never imports it and has no CPU fallback.

It restates, vectorised over the lattice with numpy, the reference's Numba
kernels in the reference's own operation order, so that on the same inputs it
reproduces the reference's FP64 results to the last few ulps (pinned against
outputs of the reference itself, run under Numba's CUDA simulator, by
``tests/golden/make_golden.py`` and ``tests/test_oracle_golden.py``).

Array conventions
-----------------
A field is an array ``F`` of shape ``(nf, xlen, ylen)``; its C-order flattening
is the reference's device layout ``idx = y + x*ylen + a*xlen*ylen``
(soliton_solver/core/utils.py:17-42).  ``d1`` has shape ``(2, nf, X, Y)`` with
``d1[i, a]`` = d(field a)/d(coordinate i); ``d2`` has shape ``(2, 2, nf, X, Y)``.
(The reference stores derivatives x-contiguous, soliton_solver/core/utils.py:45-106;
only their values matter here.)  ``p_i`` / ``p_f`` are the packed parameter
arrays produced by the reference's ``pack_device_params``
(soliton_solver/core/params.py:229-249 and each theory's params.py).
"""
from __future__ import annotations

import math

import numpy as np

THEORIES = ("chiral_magnet", "baby_skyrme", "ginzburg_landau_superconductor",
            "anisotropic_superconductor")


# ----------------------------------------------------------------------------
# finite differences  (soliton_solver/core/derivatives.py)
# ----------------------------------------------------------------------------
def first_derivatives(F, p_i, p_f, comps=None):
    """4th-order central first derivatives, zero within ``halo`` of the edge.

    Follows soliton_solver/core/derivatives.py:14-57: d/dx is evaluated only for
    ``halo <= x <= xlen-halo-1`` (same for y) and is 0.0 elsewhere.
    """
    nf, X, Y = F.shape
    h = int(p_i[2])
    lsx, lsy = float(p_f[2]), float(p_f[3])
    d1 = np.zeros((2,) + F.shape)
    cs = range(nf) if comps is None else comps
    for a in cs:
        f = F[a]
        if X - 2 * h > 0:
            s = slice(h, X - h)
            d1[0, a, s, :] = ((1.0 / 12.0) * f[h - 2:X - h - 2, :] - (2.0 / 3.0) * f[h - 1:X - h - 1, :]
                              + (2.0 / 3.0) * f[h + 1:X - h + 1, :] - (1.0 / 12.0) * f[h + 2:X - h + 2, :]) / lsx
        if Y - 2 * h > 0:
            s = slice(h, Y - h)
            d1[1, a, :, s] = ((1.0 / 12.0) * f[:, h - 2:Y - h - 2] - (2.0 / 3.0) * f[:, h - 1:Y - h - 1]
                              + (2.0 / 3.0) * f[:, h + 1:Y - h + 1] - (1.0 / 12.0) * f[:, h + 2:Y - h + 2]) / lsy
    return d1


def second_derivatives(F, p_i, p_f, comps=None):
    """4th-order second derivatives including the reference's mixed-derivative ring.

    Follows soliton_solver/core/derivatives.py:60-115.  d2/dx2 and d2/dy2 use the
    5-point stencil and are zero within ``halo`` of the edge.  The mixed derivative
    is built from the main-diagonal 5-point stencil, ``diag/(2 dA) - dxx/2 - dyy/2``,
    and is nonzero only for ``halo < x < xlen-halo`` and ``halo < y < ylen-halo``
    (so x = halo is excluded but x = xlen-halo-1 is included).
    """
    nf, X, Y = F.shape
    h = int(p_i[2])
    lsx, lsy = float(p_f[2]), float(p_f[3])
    dA = float(p_f[4])
    d2 = np.zeros((2, 2) + F.shape)
    cs = range(nf) if comps is None else comps
    c1, c2, c3 = 1.0 / 12.0, 4.0 / 3.0, 5.0 / 2.0
    for a in cs:
        f = F[a]

        def sx(k, lo, hi):
            return f[lo + k:hi + k, :]

        def sy(k, lo, hi):
            return f[:, lo + k:hi + k]

        if X - 2 * h > 0:
            lo, hi = h, X - h
            d2[0, 0, a, lo:hi, :] = (-c1 * sx(-2, lo, hi) + c2 * sx(-1, lo, hi) - c3 * sx(0, lo, hi)
                                     + c2 * sx(1, lo, hi) - c1 * sx(2, lo, hi)) / (lsx * lsx)
        if Y - 2 * h > 0:
            lo, hi = h, Y - h
            d2[1, 1, a, :, lo:hi] = (-c1 * sy(-2, lo, hi) + c2 * sy(-1, lo, hi) - c3 * sy(0, lo, hi)
                                     + c2 * sy(1, lo, hi) - c1 * sy(2, lo, hi)) / (lsy * lsy)
        xl, xh, yl, yh = h + 1, X - h, h + 1, Y - h
        if xh > xl and yh > yl:
            def sd(k):
                return f[xl + k:xh + k, yl + k:yh + k]

            def sxx(k):
                return f[xl + k:xh + k, yl:yh]

            def syy(k):
                return f[xl:xh, yl + k:yh + k]

            diag = (-c1 * sd(-2) + c2 * sd(-1) - c3 * sd(0) + c2 * sd(1) - c1 * sd(2)) / (2.0 * dA)
            dxx_half = (-c1 * sxx(-2) + c2 * sxx(-1) - c3 * sxx(0) + c2 * sxx(1) - c1 * sxx(2)) / (2.0 * lsx * lsx)
            dyy_half = (-c1 * syy(-2) + c2 * syy(-1) - c3 * syy(0) + c2 * syy(1) - c1 * syy(2)) / (2.0 * lsy * lsy)
            d2[1, 0, a, xl:xh, yl:yh] = diag - dxx_half - dyy_half
        d2[0, 1, a] = d2[1, 0, a]
    return d2


# ----------------------------------------------------------------------------
# reductions  (soliton_solver/core/utils.py)
# ----------------------------------------------------------------------------
def reference_sum(v):
    """Block-tree sum of 1024-wide blocks, then numpy sum of the block partials.

    Restates reduce_sum_kernel + compute_sum (soliton_solver/core/utils.py:188-228,
    316-341) in the same association order.
    """
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
    n = v.size
    tpb = 1024
    blocks = (n + tpb - 1) // tpb
    s = np.zeros(blocks * tpb)
    s[:n] = v
    s = s.reshape(blocks, tpb)
    stride = tpb // 2
    while stride > 0:
        s[:, :stride] = s[:, :stride] + s[:, stride:2 * stride]
        stride //= 2
    return float(s[:, 0].copy().sum())


def reference_max(v):
    """Signed maximum over all entries (soliton_solver/core/utils.py:231-271, 343-368, 397-420)."""
    return float(np.max(np.asarray(v, dtype=np.float64)))


# ----------------------------------------------------------------------------
# shared unit-vector helpers (chiral_magnet/kernels.py:48-122, baby_skyrme/kernels.py:51-124)
# ----------------------------------------------------------------------------
def normalize_magnetization(F, nmag):
    """m /= |m| over the first ``nmag`` components, skipping sites with |m| == 0."""
    s = np.zeros(F.shape[1:])
    for a in range(nmag):
        s = s + F[a] * F[a]
    s = np.sqrt(s)
    nz = s != 0.0
    out = F.copy()
    for a in range(nmag):
        out[a] = np.where(nz, F[a] / np.where(nz, s, 1.0), F[a])
    return out


def project_orthogonal(G, F, nmag):
    """G -= (G.m) m over the first ``nmag`` components (m taken as given, not normalised)."""
    lm = np.zeros(F.shape[1:])
    for a in range(nmag):
        lm = lm + G[a] * F[a]
    out = G.copy()
    for a in range(nmag):
        out[a] = G[a] - lm * F[a]
    return out


def _levi(i, j, k):
    if (i, j, k) in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
        return 1.0
    if (i, j, k) in ((0, 2, 1), (2, 1, 0), (1, 0, 2)):
        return -1.0
    return 0.0


def _dmi_tensor(p_i):
    """DMI tensor selection, chiral_magnet/kernels.py:151-160 (first flag set wins)."""
    D00 = D01 = D10 = D11 = 0.0
    if p_i[11]:
        D00, D11 = -1.0, -1.0
    elif p_i[12]:
        D01, D10 = -1.0, 1.0
    elif p_i[13]:
        D00, D11 = 1.0, -1.0
    elif p_i[14]:
        s = 0.7071067811865476
        D00, D01, D10, D11 = -s, -s, s, -s
    return D00, D01, D10, D11


def _halo_mask(X, Y, h):
    x = np.arange(X)[:, None]
    y = np.arange(Y)[None, :]
    return (x < h) | (x > X - h - 1) | (y < h) | (y > Y - h - 1)


# ----------------------------------------------------------------------------
# chiral magnet  (soliton_solver/theories/chiral_magnet/kernels.py)
# ----------------------------------------------------------------------------
def chiral_energy_density(F, d1, p_i, p_f):
    """Per-site energy x dA, chiral_magnet/kernels.py:125-216."""
    dA = float(p_f[4])
    cK, ch, cmu = float(p_f[6]), float(p_f[7]), float(p_f[8])
    nc, nmag, demag = int(p_i[3]), int(p_i[10]), int(p_i[15])
    D00, D01, D10, D11 = _dmi_tensor(p_i)
    e = np.zeros(F.shape[1:])
    for a in range(nmag):
        for i in range(nc):
            e = e + 0.5 * d1[i, a] * d1[i, a]
    for i in range(nc):
        for j in range(nc):
            Dij = D00 if (j == 0 and i == 0) else (D01 if (j == 0 and i == 1) else (D10 if (j == 1 and i == 0) else D11))
            if Dij == 0.0:
                continue
            for k in range(nmag):
                mk = F[k]
                for l in range(nmag):
                    eps = _levi(j, k, l)
                    if eps != 0.0:
                        e = e + Dij * eps * mk * d1[i, l]
        if demag:
            e = e - (F[3] * d1[i, i] + d1[i, 3] * d1[i, 3] / (2.0 * cmu))
    mz = F[nmag - 1]
    e = e + ch * (1.0 - mz)
    e = e + cK * (1.0 - mz * mz)
    return e * dA


def chiral_gradient(F, d1, d2, p_i, p_f, raw=False):
    """Projected energy gradient, chiral_magnet/kernels.py:398-511 (before the l = -dt EG write).

    raw=True skips the halo zeroing and the projection and returns dE/dpsi for the
    demag row (the flow stores -coup_mu * dE/dpsi there)."""
    nf, X, Y = F.shape
    h = int(p_i[2])
    cK, ch, cmu = float(p_f[6]), float(p_f[7]), float(p_f[8])
    nc, nmag, demag = int(p_i[3]), int(p_i[10]), int(p_i[15])
    D00, D01, D10, D11 = _dmi_tensor(p_i)
    EG = np.zeros_like(F)
    for i in range(nmag):
        lap = np.zeros((X, Y))
        for j in range(nc):
            lap = lap + d2[j, j, i]
        EG[i] = EG[i] - lap
    if D00 != 0.0 or D01 != 0.0 or D10 != 0.0 or D11 != 0.0:
        for i in range(nmag):
            for j in range(nmag):
                eps = _levi(0, i, j)
                if eps != 0.0:
                    EG[i] = EG[i] + 2.0 * D00 * eps * d1[0, j]
                if eps != 0.0 and D01 != 0.0:
                    EG[i] = EG[i] + 2.0 * D01 * eps * d1[1, j]
                eps = _levi(1, i, j)
                if eps != 0.0 and D10 != 0.0:
                    EG[i] = EG[i] + 2.0 * D10 * eps * d1[0, j]
                if eps != 0.0 and D11 != 0.0:
                    EG[i] = EG[i] + 2.0 * D11 * eps * d1[1, j]
    last = nmag - 1
    mz = F[last]
    EG[last] = EG[last] - ch
    EG[last] = EG[last] - 2.0 * cK * mz
    if demag:
        for i in range(nc):
            EG[i] = EG[i] + d1[i, 3]
            EG[3] = EG[3] + (cmu * d1[i, i] - d2[i, i, 3])
    if raw:
        if demag:
            EG[3] = EG[3] * (-1.0 / cmu)
        return EG
    mask = _halo_mask(X, Y, h)
    EG[:, mask] = 0.0
    return project_orthogonal(EG, F, nmag)


def skyrmion_density(F, d1, p_i, p_f):
    """m . (dx m x dy m) dA / 4pi, chiral_magnet/kernels.py:254-291 (= baby_skyrme/kernels.py:237-270)."""
    dA = float(p_f[4])
    m1, m2, m3 = F[0], F[1], F[2]
    dm1dx, dm2dx, dm3dx = d1[0, 0], d1[0, 1], d1[0, 2]
    dm1dy, dm2dy, dm3dy = d1[1, 0], d1[1, 1], d1[1, 2]
    cx0 = dm2dx * dm3dy - dm3dx * dm2dy
    cx1 = dm3dx * dm1dy - dm1dx * dm3dy
    cx2 = dm1dx * dm2dy - dm2dx * dm1dy
    charge = m1 * cx0 + m2 * cx1 + m3 * cx2
    return charge * (dA / (4.0 * math.pi))


def magnetic_charge_density(F, d1, p_i, p_f):
    """-div m dA, chiral_magnet/kernels.py:329-360."""
    dA = float(p_f[4])
    c = np.zeros(F.shape[1:])
    for i in range(int(p_i[3])):
        c = c - d1[i, i]
    return c * dA


# ----------------------------------------------------------------------------
# baby Skyrme  (soliton_solver/theories/baby_skyrme/kernels.py)
# ----------------------------------------------------------------------------
def baby_skyrme_energy_density(F, d1, p_i, p_f):
    """baby_skyrme/kernels.py:127-199."""
    dA = float(p_f[4])
    mpi = float(p_f[6]); mpi2 = mpi * mpi
    kappa = float(p_f[7]); kappa2 = kappa * kappa
    m1, m2, m3 = F[0], F[1], F[2]
    dm1dx, dm1dy = d1[0, 0], d1[1, 0]
    dm2dx, dm2dy = d1[0, 1], d1[1, 1]
    dm3dx, dm3dy = d1[0, 2], d1[1, 2]
    gx = dm1dx * dm1dx + dm2dx * dm2dx + dm3dx * dm3dx
    gy = dm1dy * dm1dy + dm2dy * dm2dy + dm3dy * dm3dy
    e = 0.5 * (gx + gy)
    cx = dm2dx * dm3dy - dm3dx * dm2dy
    cy = dm3dx * dm1dy - dm1dx * dm3dy
    cz = dm1dx * dm2dy - dm2dx * dm1dy
    e = e + 0.5 * kappa2 * (cx * cx + cy * cy + cz * cz)
    N = int(p_i[19])
    if p_i[11]:
        e = e + mpi2 * (1.0 - m3)
    if p_i[12]:
        t = 1.0 - m3
        e = e + mpi2 * t * t * t * t
    if p_i[13]:
        e = e + 0.5 * mpi2 * m1 * m1
    if p_i[14]:
        e = e + 0.5 * mpi2 * (1.0 - m1 * m1) * (1.0 - m3 * m3)
    if p_i[15]:
        t = 1.0 - m3
        e = e + 0.5 * mpi2 * t * (1.0 + t * t * t)
    if p_i[16]:
        e = e + 16.0 * mpi2 * (1.0 - m3) * (1.0 + 3.0 * m3 * m3 + 3.0 * m1 * m2 * m2 - m1 * m1 * m1)
    if p_i[17]:
        zr, zi = m1, m2
        for _ in range(N - 1):
            zr, zi = zr * m1 - zi * m2, zr * m2 + zi * m1
        wr = 1.0 - zr
        wi = -zi
        e = e + mpi2 * (1.0 - m3) * (wr * wr + wi * wi)
    if p_i[18]:
        e = e + mpi2 * (1.0 - m3 * m3)
    return e * dA


def baby_skyrme_gradient(F, d1, d2, p_i, p_f, raw=False):
    """Projected gradient, baby_skyrme/kernels.py:308-458 (no halo zeroing in this theory);
    raw=True skips the projection."""
    mpi = float(p_f[6]); mpi2 = mpi * mpi
    kappa = float(p_f[7]); kappa2 = kappa * kappa
    N = int(p_i[19])
    m1, m2, m3 = F[0], F[1], F[2]
    F00, F01, F02 = d1[0, 0], d1[0, 1], d1[0, 2]
    F10, F11, F12 = d1[1, 0], d1[1, 1], d1[1, 2]
    S000, S001, S002 = d2[0, 0, 0], d2[0, 0, 1], d2[0, 0, 2]
    S110, S111, S112 = d2[1, 1, 0], d2[1, 1, 1], d2[1, 1, 2]
    S010, S011, S012 = d2[0, 1, 0], d2[0, 1, 1], d2[0, 1, 2]
    S100, S101, S102 = d2[1, 0, 0], d2[1, 0, 1], d2[1, 0, 2]
    sum_F0_sq = F00 * F00 + F01 * F01 + F02 * F02
    sum_F1_sq = F10 * F10 + F11 * F11 + F12 * F12
    z = np.zeros(F.shape[1:])
    g0, g1, g2 = z.copy(), z.copy(), z.copy()
    g0 = g0 - (S000 + S110)
    g1 = g1 - (S001 + S111)
    g2 = g2 - (S002 + S112)
    sum_all_sq = sum_F0_sq + sum_F1_sq
    g0 = g0 - kappa2 * S000 * sum_all_sq
    g1 = g1 - kappa2 * S001 * sum_all_sq
    g2 = g2 - kappa2 * S002 * sum_all_sq
    g0 = g0 + kappa2 * S000 * sum_F0_sq
    g1 = g1 + kappa2 * S001 * sum_F0_sq
    g2 = g2 + kappa2 * S002 * sum_F0_sq
    A0 = S010 * F10 - S110 * F00
    A1 = S011 * F11 - S111 * F01
    A2 = S012 * F12 - S112 * F02
    sumA = A0 + A1 + A2
    dot01 = F00 * F10 + F01 * F11 + F02 * F12
    g0 = g0 - kappa2 * (F00 * sumA - S010 * dot01)
    g1 = g1 - kappa2 * (F01 * sumA - S011 * dot01)
    g2 = g2 - kappa2 * (F02 * sumA - S012 * dot01)
    g0 = g0 - kappa2 * S110 * sum_all_sq
    g1 = g1 - kappa2 * S111 * sum_all_sq
    g2 = g2 - kappa2 * S112 * sum_all_sq
    g0 = g0 + kappa2 * S110 * sum_F1_sq
    g1 = g1 + kappa2 * S111 * sum_F1_sq
    g2 = g2 + kappa2 * S112 * sum_F1_sq
    B0 = S100 * F00 - S000 * F10
    B1 = S101 * F01 - S001 * F11
    B2 = S102 * F02 - S002 * F12
    sumB = B0 + B1 + B2
    g0 = g0 - kappa2 * (F10 * sumB - S100 * dot01)
    g1 = g1 - kappa2 * (F11 * sumB - S101 * dot01)
    g2 = g2 - kappa2 * (F12 * sumB - S102 * dot01)
    if p_i[11]:
        g2 = g2 - mpi2
    if p_i[12]:
        t = 1.0 - m3
        g2 = g2 - 4.0 * mpi2 * t * t * t
    if p_i[13]:
        g0 = g0 + mpi2 * m1
    if p_i[14]:
        g0 = g0 - mpi2 * (1.0 - m3 * m3) * m1
        g2 = g2 - mpi2 * (1.0 - m1 * m1) * m3
    if p_i[15]:
        t = 1.0 - m3
        t3 = t * t * t
        g2 = g2 - mpi2 * (0.5 * (1.0 + t3) + 1.5 * t3)
    if p_i[16]:
        g0 = g0 + 48.0 * mpi2 * (m2 * m2 - m1 * m1) * (1.0 - m3)
        g1 = g1 + 96.0 * mpi2 * m1 * m2 * (1.0 - m3)
        g2 = g2 - 16.0 * mpi2 * (-(m1 * m1 * m1) + 3.0 * m1 * (m2 * m2) + (1.0 - 3.0 * m3) * (1.0 - 3.0 * m3))
    if p_i[17]:
        r2 = m1 * m1 + m2 * m2
        theta = np.arctan2(m2, m1)
        with np.errstate(divide="ignore", invalid="ignore"):
            rN2 = r2 ** (0.5 * N)
            rN = r2 ** (1.0 * N)
            c = np.cos(N * theta)
            s = np.sin(N * theta)
            norm1mzN = 1.0 - 2.0 * c * rN2 + rN
            denom = np.sqrt(norm1mzN)
            ok = (denom != 0.0) & (r2 != 0.0)
            pref = 2.0 * mpi2 * N * np.sqrt(norm1mzN) * r2 ** (-1.0 + 0.5 * N) * (-1.0 + m3) / denom
            g0 = np.where(ok, g0 + pref * (s * m2 + m1 * (c - rN2)), g0)
            g1 = np.where(ok, g1 + -pref * (s * m1 + m2 * (-c + rN2)), g1)
        g2 = g2 - mpi2 * norm1mzN
    if p_i[18]:
        g2 = g2 - 2.0 * mpi2 * m3
    EG = np.stack([g0, g1, g2])
    if raw:
        return EG
    return project_orthogonal(EG, F, int(p_i[10]))


# ----------------------------------------------------------------------------
# Abelian Higgs / Ginzburg-Landau  (theories/ginzburg_landau_superconductor/kernels.py)
# ----------------------------------------------------------------------------
def abelian_higgs_energy_density(F, d1, p_i, p_f):
    """ginzburg_landau_superconductor/kernels.py:46-108.

    Reads u from p_f[9] (the vortex number slot), exactly as the reference does.
    """
    q, lam, u1 = float(p_f[6]), float(p_f[7]), float(p_f[9])
    dA = float(p_f[4])
    A1, A2, psi1, psi2 = F[0], F[1], F[2], F[3]
    dpsi1dx, dpsi1dy = d1[0, 2], d1[1, 2]
    dpsi2dx, dpsi2dy = d1[0, 3], d1[1, 3]
    dA1dy, dA2dx = d1[1, 0], d1[0, 1]
    psi_sq = psi1 * psi1 + psi2 * psi2
    A_sq = A1 * A1 + A2 * A2
    e = np.zeros(F.shape[1:])
    e = e + 0.5 * (dpsi1dx * dpsi1dx + dpsi1dy * dpsi1dy + dpsi2dx * dpsi2dx + dpsi2dy * dpsi2dy)
    e = e + q * A1 * (psi1 * dpsi2dx - psi2 * dpsi1dx)
    e = e + q * A2 * (psi1 * dpsi2dy - psi2 * dpsi1dy)
    e = e + 0.5 * q * q * A_sq * psi_sq
    e = e + lam / 8.0 * (u1 * u1 - psi_sq) * (u1 * u1 - psi_sq)
    curlA = dA2dx - dA1dy
    e = e + 0.5 * curlA * curlA
    return e * dA


def abelian_higgs_gradient(F, d1, d2, p_i, p_f):
    """ginzburg_landau_superconductor/kernels.py:343-419 (unconstrained, no halo zeroing)."""
    q, lam, u1 = float(p_f[6]), float(p_f[7]), float(p_f[8])
    A1, A2, psi1, psi2 = F[0], F[1], F[2], F[3]
    psi_sq = psi1 * psi1 + psi2 * psi2
    dA1dx, dA1dy = d1[0, 0], d1[1, 0]
    dA2dx, dA2dy = d1[0, 1], d1[1, 1]
    dpsi1dx, dpsi1dy = d1[0, 2], d1[1, 2]
    dpsi2dx, dpsi2dy = d1[0, 3], d1[1, 3]
    d2A1d2y = d2[1, 1, 0]
    d2A2d2x = d2[0, 0, 1]
    d2psi1d2x, d2psi1d2y = d2[0, 0, 2], d2[1, 1, 2]
    d2psi2d2x, d2psi2d2y = d2[0, 0, 3], d2[1, 1, 3]
    d2A1dxdy = d2[1, 0, 0]
    d2A2dxdy = d2[1, 0, 1]
    g0 = -d2A1d2y + d2A2dxdy + q * (psi1 * dpsi2dx - psi2 * dpsi1dx) + q * q * A1 * psi_sq
    g1 = -d2A2d2x + d2A1dxdy + q * (psi1 * dpsi2dy - psi2 * dpsi1dy) + q * q * A2 * psi_sq
    g2 = (-d2psi1d2x - d2psi1d2y + 2.0 * q * (A1 * dpsi2dx + A2 * dpsi2dy) + q * psi2 * (dA1dx + dA2dy)
          + q * q * (A1 * A1 + A2 * A2) * psi1 - lam / 2.0 * (u1 * u1 - psi_sq) * psi1)
    g3 = (-d2psi2d2x - d2psi2d2y - 2.0 * q * (A1 * dpsi1dx + A2 * dpsi1dy) - q * psi1 * (dA1dx + dA2dy)
          + q * q * (A1 * A1 + A2 * A2) * psi2 - lam / 2.0 * (u1 * u1 - psi_sq) * psi2)
    return np.stack([g0, g1, g2, g3])


def vortex_density(F, d1, p_i, p_f, q_index):
    """(dx A2 - dy A1) dA / (2 pi q), ginzburg_landau_superconductor/kernels.py:146-178
    (q = p_f[6]) and anisotropic_superconductor/kernels.py:208-240 (q = p_f[7])."""
    dA = float(p_f[4])
    q = float(p_f[q_index])
    b = d1[0, 1] - d1[1, 0]
    return b * (dA / (2.0 * math.pi * q))


# ----------------------------------------------------------------------------
# anisotropic s+id superconductor  (theories/anisotropic_superconductor/kernels.py)
# ----------------------------------------------------------------------------
def _gamma_entry(i, j, a, b, p_f):
    """anisotropic_superconductor/kernels.py:46-94."""
    g1, g2, g12 = float(p_f[14]), float(p_f[15]), float(p_f[16])
    if i == 0 and j == 0:
        if a == 0 and b == 0:
            return 2.0 * g1
        if (a, b) in ((0, 1), (1, 0)):
            return -2.0 * g12
        return 2.0 * g2
    if i == 1 and j == 1:
        if a == 0 and b == 0:
            return 2.0 * g1
        if (a, b) in ((0, 1), (1, 0)):
            return 2.0 * g12
        return 2.0 * g2
    return 0.0


def splusid_energy_density(F, d1, p_i, p_f):
    """anisotropic_superconductor/kernels.py:97-170 (vacuum energy subtracted)."""
    kappa, Q = float(p_f[6]), float(p_f[7])
    a1, a2 = float(p_f[8]), float(p_f[9])
    b1, b2, b3, b4 = float(p_f[10]), float(p_f[11]), float(p_f[12]), float(p_f[13])
    dA = float(p_f[4])
    u1, u2, th = float(p_f[17]), float(p_f[18]), float(p_f[19])
    A = (F[0], F[1])
    p1r, p1i, p2r, p2i = F[2], F[3], F[4], F[5]
    p1sq = p1r * p1r + p1i * p1i
    p2sq = p2r * p2r + p2i * p2i
    F_mag = 0.5 * kappa * kappa * (d1[0, 1] - d1[1, 0]) ** 2
    F_pot = np.zeros(F.shape[1:])
    F_pot = F_pot + (a1 * p1sq + a2 * p2sq)
    F_pot = F_pot + (b1 * p1sq * p1sq + b2 * p2sq * p2sq + b3 * p1sq * p2sq)
    F_pot = F_pot + 2.0 * b4 * (p1r * p1r * p2r * p2r + p1i * p1i * p2i * p2i - p1i * p1i * p2r * p2r
                                - p1r * p1r * p2i * p2i + 4.0 * p1r * p1i * p2r * p2i)
    F_kin = np.zeros(F.shape[1:])
    for i in range(int(p_i[3])):
        Ai = A[i]
        for j in range(int(p_i[3])):
            Aj = A[j]
            g00 = _gamma_entry(i, j, 0, 0, p_f)
            g01 = _gamma_entry(i, j, 0, 1, p_f)
            g10 = _gamma_entry(i, j, 1, 0, p_f)
            g11 = _gamma_entry(i, j, 1, 1, p_f)
            d1ri, d1rj = d1[i, 2], d1[j, 2]
            d1ii, d1ij = d1[i, 3], d1[j, 3]
            d2ri, d2rj = d1[i, 4], d1[j, 4]
            d2ii, d2ij = d1[i, 5], d1[j, 5]
            F_kin = F_kin + 0.5 * g00 * (d1ri * d1rj + d1ii * d1ij + Q * Ai * (p1r * d1ij - p1i * d1rj)
                                         + Q * Aj * (p1r * d1ii - p1i * d1ri) + Q * Q * Ai * Aj * p1sq)
            F_kin = F_kin + 0.5 * g01 * (d1ri * d2rj + d1ii * d2ij + Q * Ai * (p1r * d2ij - p1i * d2rj)
                                         + Q * Aj * (p2r * d1ii - p2i * d1ri)
                                         + Q * Q * Ai * Aj * (p1r * p2r + p1i * p2i))
            F_kin = F_kin + 0.5 * g10 * (d2ri * d1rj + d2ii * d1ij + Q * Ai * (p2r * d1ij - p2i * d1rj)
                                         + Q * Aj * (p1r * d2ii - p1i * d2ri)
                                         + Q * Q * Ai * Aj * (p2r * p1r + p2i * p1i))
            F_kin = F_kin + 0.5 * g11 * (d2ri * d2rj + d2ii * d2ij + Q * Ai * (p2r * d2ij - p2i * d2rj)
                                         + Q * Aj * (p2r * d2ii - p2i * d2ri) + Q * Q * Ai * Aj * p2sq)
    e = F_kin + F_mag + F_pot
    e = e - (a1 * u1 * u1 + a2 * u2 * u2 + b1 * u1 * u1 * u1 * u1 + b2 * u2 * u2 * u2 * u2
             + b3 * u1 * u1 * u2 * u2 + 2.0 * b4 * u1 * u1 * u2 * u2 * math.cos(2.0 * th))
    return e * dA


def splusid_gradient(F, d1, d2, p_i, p_f):
    """anisotropic_superconductor/kernels.py:556-658 (unconstrained, no halo zeroing)."""
    kappa, Q = float(p_f[6]), float(p_f[7])
    a1, a2 = float(p_f[8]), float(p_f[9])
    b1, b2, b3, b4 = float(p_f[10]), float(p_f[11]), float(p_f[12]), float(p_f[13])
    A = (F[0], F[1])
    p1r, p1i, p2r, p2i = F[2], F[3], F[4], F[5]
    z = np.zeros(F.shape[1:])
    EG = [z.copy() for _ in range(6)]
    nc = int(p_i[3])
    for j in range(nc):
        for k in range(nc):
            Ak = A[k]
            g00 = _gamma_entry(k, j, 0, 0, p_f)
            g01 = _gamma_entry(k, j, 0, 1, p_f)
            g10 = _gamma_entry(k, j, 1, 0, p_f)
            g11 = _gamma_entry(k, j, 1, 1, p_f)
            val = kappa * kappa * (d2[j, k, k] - d2[k, k, j])
            val = val - Q * g00 * (p1i * d1[k, 2] - p1r * d1[k, 3] - Q * Ak * (p1r * p1r + p1i * p1i))
            val = val - Q * g01 * (p2i * d1[k, 2] - p2r * d1[k, 3] - Q * Ak * (p1r * p2r + p1i * p2i))
            val = val - Q * g10 * (p1i * d1[k, 4] - p1r * d1[k, 5] - Q * Ak * (p2r * p1r + p2i * p1i))
            val = val - Q * g11 * (p2i * d1[k, 4] - p2r * d1[k, 5] - Q * Ak * (p2r * p2r + p2i * p2i))
            EG[j] = EG[j] + val
    p1sq = p1r * p1r + p1i * p1i
    p2sq = p2r * p2r + p2i * p2i
    EG[2] = EG[2] + 2.0 * (2.0 * a1 * p1r + 4.0 * b1 * p1r * p1sq + 2.0 * b3 * p1r * p2sq
                           + 2.0 * b4 * (2.0 * p1r * (p2r * p2r - p2i * p2i) + 4.0 * p1i * p2r * p2i))
    EG[3] = EG[3] + 2.0 * (2.0 * a1 * p1i + 4.0 * b1 * p1i * p1sq + 2.0 * b3 * p1i * p2sq
                           + 2.0 * b4 * (-2.0 * p1i * (p2r * p2r - p2i * p2i) + 4.0 * p1r * p2r * p2i))
    EG[4] = EG[4] + 2.0 * (2.0 * a2 * p2r + 4.0 * b2 * p2r * p2sq + 2.0 * b3 * p2r * p1sq
                           + 2.0 * b4 * (2.0 * p2r * (p1r * p1r - p1i * p1i) + 4.0 * p1r * p1i * p2i))
    EG[5] = EG[5] + 2.0 * (2.0 * a2 * p2i + 4.0 * b2 * p2i * p2sq + 2.0 * b3 * p2i * p1sq
                           + 2.0 * b4 * (-2.0 * p2i * (p1r * p1r - p1i * p1i) + 4.0 * p1r * p1i * p2r))
    for i in range(nc):
        Ai = A[i]
        for j in range(nc):
            Aj = A[j]
            gij00 = _gamma_entry(i, j, 0, 0, p_f)
            gij01 = _gamma_entry(i, j, 0, 1, p_f)
            gij10 = _gamma_entry(i, j, 1, 0, p_f)
            gij11 = _gamma_entry(i, j, 1, 1, p_f)
            dAij = d1[i, j]
            EG[2] = EG[2] - gij00 * (d2[i, j, 2] - Q * Q * Ai * Aj * p1r - Q * (p1i * dAij + Ai * d1[j, 3] + Aj * d1[i, 3]))
            EG[2] = EG[2] - gij01 * (d2[i, j, 4] - Q * Q * Ai * Aj * p2r - Q * (p2i * dAij + Ai * d1[j, 5] + Aj * d1[i, 5]))
            EG[3] = EG[3] - gij00 * (d2[i, j, 3] - Q * Q * Ai * Aj * p1i + Q * (p1r * dAij + Ai * d1[j, 2] + Aj * d1[i, 2]))
            EG[3] = EG[3] - gij01 * (d2[i, j, 5] - Q * Q * Ai * Aj * p2i + Q * (p2r * dAij + Ai * d1[j, 4] + Aj * d1[i, 4]))
            EG[4] = EG[4] - gij10 * (d2[i, j, 2] - Q * Q * Ai * Aj * p1r - Q * (p1i * dAij + Ai * d1[j, 3] + Aj * d1[i, 3]))
            EG[4] = EG[4] - gij11 * (d2[i, j, 4] - Q * Q * Ai * Aj * p2r - Q * (p2i * dAij + Ai * d1[j, 5] + Aj * d1[i, 5]))
            EG[5] = EG[5] - gij10 * (d2[i, j, 3] - Q * Q * Ai * Aj * p1i + Q * (p1r * dAij + Ai * d1[j, 2] + Aj * d1[i, 2]))
            EG[5] = EG[5] - gij11 * (d2[i, j, 5] - Q * Q * Ai * Aj * p2i + Q * (p2r * dAij + Ai * d1[j, 4] + Aj * d1[i, 4]))
    return np.stack(EG)


# ----------------------------------------------------------------------------
# theory dispatch
# ----------------------------------------------------------------------------
_GRAD = {
    "chiral_magnet": chiral_gradient,
    "baby_skyrme": baby_skyrme_gradient,
    "ginzburg_landau_superconductor": abelian_higgs_gradient,
    "anisotropic_superconductor": splusid_gradient,
}
_ENERGY = {
    "chiral_magnet": chiral_energy_density,
    "baby_skyrme": baby_skyrme_energy_density,
    "ginzburg_landau_superconductor": abelian_higgs_energy_density,
    "anisotropic_superconductor": splusid_energy_density,
}
CONSTRAINED = {"chiral_magnet": True, "baby_skyrme": True,
               "ginzburg_landau_superconductor": False, "anisotropic_superconductor": False}


def as_field(flat, p_i):
    """Reshape a flat reference-layout buffer into (nf, xlen, ylen)."""
    return np.asarray(flat, dtype=np.float64).reshape(int(p_i[4]), int(p_i[0]), int(p_i[1]))


def gradient_step(theory, F, p_i, p_f):
    """The reference's do_gradient_step_kernel (core/integrator.py:15-48): returns (l_out, EG)
    with ``l_out = -dt * EG``."""
    d1 = first_derivatives(F, p_i, p_f)
    d2 = second_derivatives(F, p_i, p_f)
    EG = _GRAD[theory](F, d1, d2, p_i, p_f)
    return -float(p_f[5]) * EG, EG


def raw_gradient(theory, F, p_i, p_f):
    """Unprojected functional derivative dE/dphi (the flow's stencil without projection or
    halo zeroing; true dE/dpsi for the chiral demag row)."""
    d1 = first_derivatives(F, p_i, p_f)
    d2 = second_derivatives(F, p_i, p_f)
    if theory in ("chiral_magnet", "baby_skyrme"):
        return _GRAD[theory](F, d1, d2, p_i, p_f, raw=True)
    return _GRAD[theory](F, d1, d2, p_i, p_f)


def energy_density(theory, F, p_i, p_f):
    """The reference's compute_energy_kernel output ``en`` (per-site energy x dA)."""
    d1 = first_derivatives(F, p_i, p_f)
    return _ENERGY[theory](F, d1, p_i, p_f)


def energy(theory, F, p_i, p_f):
    """observables.compute_energy (e.g. chiral_magnet/observables.py:15-57)."""
    return reference_sum(energy_density(theory, F, p_i, p_f))


def charge_density(theory, F, p_i, p_f, which):
    """Charge densities: 'skyrmion' (chiral, baby Skyrme), 'magnetic' (chiral), 'vortex' (GL, s+id).

    As in the reference kernels, derivatives are taken only of the components the
    density uses (magnetisation or gauge fields)."""
    if which == "skyrmion":
        d1 = first_derivatives(F, p_i, p_f, comps=range(int(p_i[10])))
        return skyrmion_density(F, d1, p_i, p_f)
    if which == "magnetic":
        d1 = first_derivatives(F, p_i, p_f, comps=range(int(p_i[10])))
        return magnetic_charge_density(F, d1, p_i, p_f)
    if which == "vortex":
        if theory == "ginzburg_landau_superconductor":
            d1 = first_derivatives(F, p_i, p_f, comps=range(int(p_i[11])))
            return vortex_density(F, d1, p_i, p_f, 6)
        d1 = first_derivatives(F, p_i, p_f, comps=range(int(p_i[12])))
        return vortex_density(F, d1, p_i, p_f, 7)
    raise ValueError(which)


def charge(theory, F, p_i, p_f, which):
    return reference_sum(charge_density(theory, F, p_i, p_f, which))


def field_density(theory, F, p_i, p_f, kind):
    """Diagnostic densities of the gauge theories (Simulation's output helpers).

    'higgs'      |psi|^2, ginzburg_landau_superconductor/kernels.py:218-272
    'higgs1'     |psi1|^2, anisotropic_superconductor/kernels.py:315-369
    'higgs2'     |psi2|^2, anisotropic_superconductor/kernels.py:372-426
    'phase'      cos(atan2(psi1) - atan2(psi2)), anisotropic_superconductor/kernels.py:497-553
    'supercurrent' (2, X, Y): (d2[1,0,A2] - d2[1,1,A1], d2[0,1,A1] - d2[0,0,A2]),
                 ginzburg_landau_superconductor/kernels.py:275-340 (second derivatives of
                 the gauge fields only, with the mixed-derivative ring)
    'magnetic'   the vortex density with which = 2 (compute_magnetic_field_kernel,
                 anisotropic_superconductor/kernels.py:280-312)
    """
    if kind in ("higgs", "higgs1", "higgs2"):
        a = 4 if kind == "higgs2" else 2
        return F[a] * F[a] + F[a + 1] * F[a + 1]
    if kind == "phase":
        return np.cos(np.arctan2(F[3], F[2]) - np.arctan2(F[5], F[4]))
    ng = int(p_i[11] if theory == "ginzburg_landau_superconductor" else p_i[12])
    if kind == "supercurrent":
        d2 = second_derivatives(F, p_i, p_f, comps=range(ng))
        return np.stack([d2[1, 0, 1] - d2[1, 1, 0], d2[0, 1, 0] - d2[0, 0, 1]])
    if kind == "magnetic":
        return charge_density(theory, F, p_i, p_f, "vortex")
    raise ValueError(kind)


def rk4_stage(V, l_in, F, k_prev, factor, p_f):
    """do_rk4_step_kernel, core/integrator.py:51-96: returns (k_out, Temp)."""
    dt = float(p_f[5])
    return dt * (V + factor * l_in), F + factor * k_prev


def rk4_finalize(theory, V, F, k1, k2, k3, k4, l1, l2, l3, l4, p_i):
    """do_rk4_kernel / do_rk4_kernel_no_constraint, core/integrator.py:99-189."""
    Vn = V + (1.0 / 6.0) * (l1 + 2.0 * l2 + 2.0 * l3 + l4)
    Fn = F + (1.0 / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    if CONSTRAINED[theory] and int(p_i[9]):
        nmag = int(p_i[10])
        Fn = normalize_magnetization(Fn, nmag)
        Vn = project_orthogonal(Vn, Fn, nmag)
    return Vn, Fn


def arrested_newton_flow_step(theory, F, V, prev_energy, p_i, p_f):
    """One step of do_arrested_newton_flow, core/integrator.py:217-348.

    Returns ``(F_new, V_new, E_new, err)``; err is the signed maximum of the
    stage-4 energy gradient over all nf*N entries.
    """
    k1, T = rk4_stage(V, V, F, F, 0.0, p_f)
    l1, _ = gradient_step(theory, T, p_i, p_f)
    k2, T = rk4_stage(V, l1, F, k1, 0.5, p_f)
    l2, _ = gradient_step(theory, T, p_i, p_f)
    k3, T = rk4_stage(V, l2, F, k2, 0.5, p_f)
    l3, _ = gradient_step(theory, T, p_i, p_f)
    k4, T = rk4_stage(V, l3, F, k3, 1.0, p_f)
    l4, EG = gradient_step(theory, T, p_i, p_f)
    Vn, Fn = rk4_finalize(theory, V, F, k1, k2, k3, k4, l1, l2, l3, l4, p_i)
    E = energy(theory, Fn, p_i, p_f)
    if int(p_i[7]) and E > prev_energy:
        Vn = np.zeros_like(Vn)
    return Fn, Vn, E, reference_max(EG)


def relax(theory, F, V, prev_energy, p_i, p_f, n_steps):
    """Run ``n_steps`` flow steps; returns (F, V, E_traj, err_traj)."""
    E_traj = np.empty(n_steps)
    err_traj = np.empty(n_steps)
    E = prev_energy
    for s in range(n_steps):
        F, V, E, err = arrested_newton_flow_step(theory, F, V, E, p_i, p_f)
        E_traj[s] = E
        err_traj[s] = err
    return F, V, E_traj, err_traj


def relax_replay(theory, F, V, arrests, p_i, p_f):
    """``len(arrests)`` flow steps of do_arrested_newton_flow (core/integrator.py:217-348)
    with the arrest decisions given instead of taken: V = 0 after step s iff arrests[s].
    An FP32 flow decides E' > E on FP32 energies, which cannot resolve the energy steps
    near an arrest (|dE|/E ~ 1e-9 in a few hundred steps); replaying its decisions lets
    its trajectory be compared step for step.  Returns (F, V, E_traj, err_traj)."""
    n_steps = len(arrests)
    E_traj = np.empty(n_steps)
    err_traj = np.empty(n_steps)
    for s in range(n_steps):
        F, V, E, err = arrested_newton_flow_step(theory, F, V, np.inf, p_i, p_f)
        if arrests[s]:
            V = np.zeros_like(V)
        E_traj[s] = E
        err_traj[s] = err
    return F, V, E_traj, err_traj
