"""Golden RGBA images from the reference's own colormap kernels.

Run in a container that has the reference checkout (it is NOT needed at test time):

    python tests/golden/make_golden_colormaps.py --ref <reference checkout> --out tests/golden

It imports ``soliton_solver.core.colormaps`` with Numba's CUDA simulator enabled
(``NUMBA_ENABLE_CUDASIM=1``; no GPU, no GL: the kernels write into a plain uint8
array of shape (ylen, xlen, 4)), launches ``render_jet_density_to_rgba``,
``render_gray_density_to_rgba`` and ``render_magnetization_to_rgba`` on seeded
inputs and writes ``colormap_*.npz`` (inputs, launch arguments, RGBA output).
Every input value is FP32-representable, so one image pins both the FP32 and the
FP64 input paths.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def _f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SOLITON_SOLVER_REF"), required="SOLITON_SOLVER_REF" not in os.environ,
                    help="root of the reference soliton_solver checkout (or set SOLITON_SOLVER_REF)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    sys.path.insert(0, args.ref)
    from soliton_solver.core import colormaps as cm

    def launch(kernel, xlen, ylen, *rest):
        out = np.zeros((ylen, xlen, 4), dtype=np.uint8)
        kernel[((xlen + 7) // 8, (ylen + 7) // 8), (8, 8)](out, *rest)
        return out

    rng = np.random.default_rng(2024)
    X, Y = 37, 29
    # densities: smooth + noise, with exact hits on vmin, vmax and the jet breakpoints
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    dens = _f32(1.5 * np.sin(2.3 * x) * np.cos(1.7 * y) + 0.3 * rng.standard_normal((X, Y)))
    flat = dens.reshape(-1).copy()
    specials = [-1.0, 2.0, -1.0 + 3.0 / 8, -1.0 + 9.0 / 8, -1.0 + 15.0 / 8, -1.0 + 21.0 / 8, 0.0, -5.0, 7.0]
    flat[: len(specials)] = _f32(specials)
    for name, kern in (("jet", cm.render_jet_density_to_rgba), ("gray", cm.render_gray_density_to_rgba)):
        for k, (vmin, vmax) in enumerate(((-1.0, 2.0), (0.25, 0.25), (3.0, -2.0), (-4.0, 4.0))):
            rgba = launch(kern, X, Y, flat, X, Y, vmin, vmax)
            np.savez_compressed(os.path.join(args.out, f"colormap_{name}_{k}.npz"), kind=name, density=flat,
                                xlen=X, ylen=Y, vmin=vmin, vmax=vmax, rgba=rgba)
    # magnetisation: unit vectors (a hedgehog with noise) plus a 4th plane, as a chiral field
    for k, (Xm, Ym) in enumerate(((37, 29), (16, 24))):
        xm = np.linspace(-1, 1, Xm)[:, None]
        ym = np.linspace(-1, 1, Ym)[None, :]
        r, th = np.hypot(xm, ym), np.arctan2(ym, xm)
        f = np.pi * np.exp(-r / 0.6)
        m = np.stack([np.sin(f) * np.cos(th), np.sin(f) * np.sin(th), np.cos(f)])
        m += 0.2 * rng.standard_normal(m.shape)
        m /= np.sqrt((m ** 2).sum(0))
        F = np.concatenate([m, 0.1 * rng.standard_normal((1, Xm, Ym))])
        F[:, 0, 0] = (0.0, 0.0, 1.0, 0.0)
        F[:, 0, 1] = (0.0, 0.0, -1.0, 0.0)
        F[:, 1, 0] = (1.0, 0.0, 0.0, 0.0)
        F[:, 1, 1] = (0.0, -1.0, 0.0, 0.0)
        F = _f32(F).reshape(-1)
        p_i = np.array([Xm, Ym], dtype=np.int32)
        rgba = launch(cm.render_magnetization_to_rgba, Xm, Ym, F, Xm, Ym, p_i)
        np.savez_compressed(os.path.join(args.out, f"colormap_magnetization_{k}.npz"), kind="magnetization",
                            field=F, xlen=Xm, ylen=Ym, rgba=rgba)
    print("wrote colormap fixtures to", args.out)


if __name__ == "__main__":
    main()
