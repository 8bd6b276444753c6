"""CPU restatement of the reference's initial-condition kernels (test infrastructure only).

The checker for ``ss_initialize`` / ``ss_insert_soliton`` of libsoliton_b200; the library
never imports it.  Vectorised over the lattice, in the reference's operation order
(FP64), it restates per theory ``theories/<theory>/initial_config.py``:

* ``position``, ``angle``, ``profile_function_*``  (chiral_magnet/initial_config.py:15-115,
  ginzburg_landau_superconductor/initial_config.py:13-112)
* ``create_ground_state_kernel``          (chiral :117-180, baby Skyrme :119-181,
  Abelian Higgs :114-178, s+id :116-190)
* ``create_initial_configuration_kernel`` (chiral :182-283, baby Skyrme :183-280,
  Abelian Higgs :180-257, s+id :192-280)
* ``create_skyrmion_kernel`` (chiral :285-386, baby Skyrme :282-383) and
  ``create_vortex_kernel`` (Abelian Higgs :259-313, s+id :282-347)
* ``compute_norm_magnetization`` (chiral_magnet/kernels.py:48-84)

Reference quirks kept: the chiral magnet reads the skyrmion number from p_f[9], the
baby Skyrme model from p_f[8]; the s+id ground state reads u1, u2 from p_f[11], p_f[12]
(beta2, beta3 in its packing) while its ansatz reads p_f[17], p_f[18].  One bug is
repaired: the Abelian Higgs ansatz reads ainf from p_f[11], one past the packed array;
here (and in the library) it reads the packed ainf, p_f[10].  Pinned to the outputs of
the reference's kernels (``tests/golden/init_*.npz``, ``tests/golden/make_golden_init.py``).
"""
from __future__ import annotations

import math

import numpy as np

MAGNETIC = {"chiral_magnet": 9, "baby_skyrme": 8}  # p_f slot of the skyrmion number
ANSATZ_NONE, ANSATZ_BLOCH, ANSATZ_NEEL, ANSATZ_ANTI = 0, 1, 2, 3


def _coords(p_i, p_f):
    X, Y = int(p_i[0]), int(p_i[1])
    gx = float(p_f[2]) * np.arange(X, dtype=np.float64)[:, None] * np.ones((1, Y))
    gy = float(p_f[3]) * np.arange(Y, dtype=np.float64)[None, :] * np.ones((X, 1))
    return gx, gy


def _centre(p_i, p_f):
    X, Y = int(p_i[0]), int(p_i[1])
    return (0.0 + float(p_f[2]) * float(X - 1)) / 2.0, (0.0 + float(p_f[3]) * float(Y - 1)) / 2.0


def _position_angle(gx, gy, xc, yc, orientation):
    dx, dy = gx - xc, gy - yc
    r = np.sqrt(dx * dx + dy * dy)
    ang = np.arctan2(dy, dx)
    ang = np.where(ang < 0.0, ang + 2.0 * math.pi, ang)
    th = np.where(r == 0.0, -orientation, -orientation + ang)
    return r, th


def _profile_m(r, max_r):
    t = 2.0 * r / max_r
    return np.where(r > max_r, 0.0, math.pi * np.exp(-(t * t)))


def _profile_s(r, max_r, value):
    return np.where(r > max_r, 1.0, np.tanh(value * r))


def _normalise(m):
    s = np.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])
    nz = s != 0.0
    return [np.where(nz, c / np.where(nz, s, 1.0), c) for c in m]


def _ansatz_m(ansatz, fm, th, skN):
    if ansatz == ANSATZ_BLOCH:
        return [-np.sin(fm) * np.sin(skN * th), np.sin(fm) * np.cos(skN * th), np.cos(fm)]
    if ansatz == ANSATZ_NEEL:
        return [np.sin(fm) * np.cos(skN * th), np.sin(fm) * np.sin(skN * th), np.cos(fm)]
    if ansatz == ANSATZ_ANTI:
        return [-np.sin(fm) * np.sin(skN * th), -np.sin(fm) * np.cos(skN * th), np.cos(fm)]
    return None


def ground(theory, p_i, p_f):
    """Field of create_ground_state_kernel, shape (nf, X, Y)."""
    X, Y, nf = int(p_i[0]), int(p_i[1]), int(p_i[4])
    F = np.zeros((nf, X, Y))
    if theory in MAGNETIC:
        F[2] = 1.0
    elif theory == "ginzburg_landau_superconductor":
        F[2] = float(p_f[8])
    else:
        u1, u2, td = float(p_f[11]), float(p_f[12]), float(p_f[19])
        F[2] = u1
        F[4] = u2 * math.cos(td)
        F[5] = u2 * math.sin(td)
    return F


def initial(theory, p_i, p_f, ansatz=ANSATZ_BLOCH, rotation=0.0, vortex_number=1.0):
    """Field of create_initial_configuration_kernel, shape (nf, X, Y)."""
    X, Y, nf = int(p_i[0]), int(p_i[1]), int(p_i[4])
    gx, gy = _coords(p_i, p_f)
    xc, yc = _centre(p_i, p_f)
    rmax = max(float(p_f[0]), float(p_f[1])) if float(p_f[0]) > float(p_f[1]) else float(p_f[1])
    F = np.zeros((nf, X, Y))
    if theory in MAGNETIC:
        skN = float(p_f[MAGNETIC[theory]])
        r, th = _position_angle(gx, gy, xc, yc, rotation)
        fm = _profile_m(r, rmax / 10.0 * skN)
        m = _ansatz_m(ansatz, fm, th, skN)
        if m is None:
            F[2] = 1.0
        else:
            F[:3] = np.stack(_normalise(m))
        return F
    r, th = _position_angle(gx, gy, xc, yc, 0.0)
    rr = np.where(r > 1e-12, r, 1e-12)
    if theory == "ginzburg_landau_superconductor":
        ainf, u1 = float(p_f[10]), float(p_f[8])
        fs = _profile_s(r, rmax, 0.2)
        F[0] = ainf * fs * np.sin(th) / rr
        F[1] = -ainf * fs * np.cos(th) / rr
        F[2] = u1 * fs * np.cos(vortex_number * th)
        F[3] = u1 * fs * np.sin(vortex_number * th)
        return F
    u1, u2, ainf = float(p_f[17]), float(p_f[18]), float(p_f[22])
    v1, v2 = float(p_f[23]), float(p_f[24])
    fs = _profile_s(r, rmax, 1.0)
    F[0] = ainf * fs * np.sin(th) / rr
    F[1] = -ainf * fs * np.cos(th) / rr
    F[2] = u1 * fs * np.cos(v1 * th)
    F[3] = u1 * fs * np.sin(v1 * th)
    F[4] = u2 * fs * np.cos(v2 * th)
    F[5] = u2 * fs * np.sin(v2 * th)
    return F


def insert(theory, F, p_i, p_f, pxi, pxj, ansatz=ANSATZ_BLOCH, rotation=0.0, vortex=True):
    """Field after create_skyrmion_kernel / create_vortex_kernel at lattice point (pxi, pxj)."""
    X, Y = int(p_i[0]), int(p_i[1])
    F = np.array(F, dtype=np.float64, copy=True)
    if not (0 <= pxi < X and 0 <= pxj < Y):
        return F
    gx, gy = _coords(p_i, p_f)
    xc, yc = float(p_f[2]) * float(pxi), float(p_f[3]) * float(pxj)
    rmax = float(p_f[0]) if float(p_f[0]) > float(p_f[1]) else float(p_f[1])
    if theory in MAGNETIC:
        skN = float(p_f[MAGNETIC[theory]])
        r, th = _position_angle(gx, gy, xc, yc, rotation)
        if skN == 0:
            fm = _profile_m(r, rmax / 10.0 * 2.0)
            m = _ansatz_m(ansatz, 2.0 * fm, th, 1.0)
        else:
            fm = _profile_m(r, rmax / 10.0 * skN)
            m = _ansatz_m(ansatz, fm, th, skN)
        if m is None:
            m = [np.zeros_like(r), np.zeros_like(r), np.ones_like(r)]
        eps = 1e-12
        den = np.maximum(1.0 + F[2], eps)
        old_wr, old_wi = F[0] / den, F[1] / den
        int_den = np.maximum(1.0 + m[2], eps)
        new_wr = old_wr + m[0] / int_den
        new_wi = old_wi + m[1] / int_den
        nw = new_wr * new_wr + new_wi * new_wi
        F[0] = 2.0 * new_wr / (1.0 + nw)
        F[1] = 2.0 * new_wi / (1.0 + nw)
        F[2] = (1.0 - nw) / (1.0 + nw)
        F[:3] = np.stack(_normalise([F[0], F[1], F[2]]))
        return F
    r, th = _position_angle(gx, gy, xc, yc, 0.0)
    phase = (-1.0 if vortex else 1.0) * th
    if theory == "ginzburg_landau_superconductor":
        u1, vn = float(p_f[8]), float(p_f[9])
        fs = _profile_s(r, rmax, 0.2)
        int_r = u1 * fs * np.cos(vn * phase)
        int_i = u1 * fs * np.sin(vn * phase)
        old_r, old_i = F[2].copy(), F[3].copy()
        F[2] = (old_r * int_r - old_i * int_i) / u1
        F[3] = (old_r * int_i + old_i * int_r) / u1
        return F
    vn, ainf = float(p_f[21]), float(p_f[22])
    fs = _profile_s(r, rmax, 2.0)
    rr = np.where(r > 1e-12, r, 1e-12)
    F[0] = F[0] - ainf * fs * np.sin(th) / rr
    F[1] = F[1] + ainf * fs * np.cos(th) / rr
    int_r = fs * np.cos(vn * phase)
    int_i = fs * np.sin(vn * phase)
    for a in (2, 4):
        old_r, old_i = F[a].copy(), F[a + 1].copy()
        F[a] = old_r * int_r - old_i * int_i
        F[a + 1] = old_r * int_i + old_i * int_r
    return F
