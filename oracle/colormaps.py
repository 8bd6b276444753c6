"""CPU restatement of the reference's colormap kernels (test infrastructure only).

This module is the checker for the headless RGBA kernels of libsoliton_b200
(``ss_render_rgba``); nothing in the library imports it.  It restates, per pixel and
in the reference's operation order with FP64 scalars,
``soliton_solver/core/colormaps.py``:

* ``clip_u8``                       (colormaps.py:14-40)
* ``_hsv_to_rgb``                   (colormaps.py:42-92)
* ``render_jet_density_to_rgba``    (colormaps.py:94-161)
* ``render_gray_density_to_rgba``   (colormaps.py:163-205)
* ``render_magnetization_to_rgba``  (colormaps.py:207-267)

Output layout as the reference's PBO: uint8 array (ylen, xlen, 4), pixel (y, x) from
field index ``y + x * ylen``.  Pinned to images the reference produced
(``tests/golden/colormap_*.npz``, ``tests/golden/make_golden_colormaps.py``).
"""
from __future__ import annotations

import math

import numpy as np


def clip_u8(x: float) -> int:
    if x < 0.0:
        return 0
    if x > 255.0:
        return 255
    return int(x)


def hsv_to_rgb(h: float, s: float, v: float):
    if h >= 360.0:
        h = 0.0
    h = h / 60.0
    i = int(h)
    ff = h - i
    p = v * (1.0 - s)
    r = v * (1.0 - (s * ff))
    t = v * (1.0 - (s * (1.0 - ff)))
    if i == 0:
        return v, t, p
    if i == 1:
        return r, v, p
    if i == 2:
        return p, v, t
    if i == 3:
        return p, r, v
    if i == 4:
        return t, p, v
    return v, p, r


def _hue(val: float, vmin: float, vmax: float) -> float:
    hue = (val - vmin) / (vmax - vmin + 1e-30)
    if hue < 0.0:
        hue = 0.0
    if hue > 1.0:
        hue = 1.0
    return hue


def jet_pixel(val: float, vmin: float, vmax: float):
    hue = _hue(val, vmin, vmax)
    if hue <= 1.0 / 8.0:
        r, g, b = 0.0, 0.0, (4.0 * hue + 0.5) * 255.0
    elif hue <= 3.0 / 8.0:
        r, g, b = 0.0, (4.0 * hue - 0.5) * 255.0, 255.0
    elif hue <= 5.0 / 8.0:
        r, g, b = (4.0 * hue - 1.5) * 255.0, 255.0, (-4.0 * hue + 2.5) * 255.0
    elif hue <= 7.0 / 8.0:
        r, g, b = 255.0, (-4.0 * hue + 3.5) * 255.0, 0.0
    else:
        r, g, b = (-4.0 * hue + 4.5) * 255.0, 0.0, 0.0
    return clip_u8(r), clip_u8(g), clip_u8(b), 255


def gray_pixel(val: float, vmin: float, vmax: float):
    c = clip_u8(_hue(val, vmin, vmax) * 255.0)
    return c, c, c, 255


def magnetization_pixel(m1: float, m2: float, m3: float):
    hue = (0.5 + (1.0 / (2.0 * math.pi)) * math.atan2(m1, m2)) * 360.0
    saturation = 0.5 - 0.5 * math.tanh(3.0 * (m3 - 0.5))
    value = 1.0 + m3
    R, G, B = hsv_to_rgb(hue, saturation, value)
    return clip_u8(R * 255.0), clip_u8(G * 255.0), clip_u8(B * 255.0), 255


def render_density(kind: str, density_flat, xlen: int, ylen: int, vmin: float, vmax: float) -> np.ndarray:
    """kind "jet" or "gray"; density_flat indexed y + x * ylen."""
    px = jet_pixel if kind == "jet" else gray_pixel
    d = np.asarray(density_flat, dtype=np.float64)
    out = np.zeros((ylen, xlen, 4), dtype=np.uint8)
    for x in range(xlen):
        for y in range(ylen):
            out[y, x] = px(float(d[y + x * ylen]), vmin, vmax)
    return out


def render_magnetization(field_flat, xlen: int, ylen: int) -> np.ndarray:
    """field_flat holds the planes m1, m2, m3 (stride xlen * ylen) first."""
    f = np.asarray(field_flat, dtype=np.float64)
    plane = xlen * ylen
    out = np.zeros((ylen, xlen, 4), dtype=np.uint8)
    for x in range(xlen):
        for y in range(ylen):
            b = y + x * ylen
            out[y, x] = magnetization_pixel(float(f[b]), float(f[b + plane]), float(f[b + 2 * plane]))
    return out
