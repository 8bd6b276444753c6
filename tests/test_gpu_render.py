"""ss_render_rgba (headless colormaps) against the reference's images and the oracle.

Byte-exact against every golden image, for FP64 and FP32 inputs (the golden inputs are
FP32-representable), through the reference-named launch adapters.  At larger sizes
against the oracle: density colormaps byte-exact; the magnetisation colormap calls
atan2 and tanh, whose CUDA and host libm results may differ in the last ulp, so at
most 1e-4 of the bytes may differ, by at most one level.
"""
import glob
import os

import numpy as np
import pytest
import torch

from oracle import colormaps as oc
from soliton_solver_b200.core import colormaps as cm

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "colormap_*.npz")))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[9:-4] for p in GOLDEN])
def test_render_matches_reference_images(path, dtype):
    g = np.load(path)
    kind, X, Y = str(g["kind"]), int(g["xlen"]), int(g["ylen"])
    out = torch.full((Y, X, 4), 7, dtype=torch.uint8, device="cuda")
    if kind == "magnetization":
        f = torch.tensor(g["field"], dtype=dtype, device="cuda")
        cm.render_magnetization_to_rgba[(1, 1), (8, 8)](out, f, X, Y, np.array([X, Y], dtype=np.int32))
    else:
        d = torch.tensor(g["density"], dtype=dtype, device="cuda")
        k = cm.render_jet_density_to_rgba if kind == "jet" else cm.render_gray_density_to_rgba
        k[(1, 1), (8, 8)](out, d, X, Y, float(g["vmin"]), float(g["vmax"]))
    np.testing.assert_array_equal(out.cpu().numpy(), g["rgba"])


@pytest.mark.parametrize("X,Y", [(173, 97), (64, 256)])
def test_render_larger_images_vs_oracle(X, Y):
    rng = np.random.default_rng(X)
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    dens = 2.0 * np.sin(3.1 * x) * np.cos(2.2 * y) + 0.2 * rng.standard_normal((X, Y))
    d = torch.tensor(dens.reshape(-1), dtype=torch.float64, device="cuda")
    for kind, k in (("jet", cm.render_jet_density_to_rgba), ("gray", cm.render_gray_density_to_rgba)):
        out = torch.empty((Y, X, 4), dtype=torch.uint8, device="cuda")
        k[None, None](out, d, X, Y, -1.5, 1.5)
        np.testing.assert_array_equal(out.cpu().numpy(), oc.render_density(kind, dens.reshape(-1), X, Y, -1.5, 1.5))
    r, th = np.hypot(x, y), np.arctan2(y, x)
    f = np.pi * np.exp(-r / 0.4)
    m = np.stack([np.sin(f) * np.cos(2 * th), np.sin(f) * np.sin(2 * th), np.cos(f)])
    m += 0.3 * rng.standard_normal(m.shape)
    m /= np.sqrt((m ** 2).sum(0))
    F = torch.tensor(m.reshape(-1), dtype=torch.float64, device="cuda")
    out = torch.empty((Y, X, 4), dtype=torch.uint8, device="cuda")
    cm.render_magnetization_to_rgba[None, None](out, F, X, Y, np.array([X, Y]))
    got = out.cpu().numpy().astype(np.int32)
    want = oc.render_magnetization(m.reshape(-1), X, Y).astype(np.int32)
    diff = np.abs(got - want)
    assert diff.max() <= 1 and (diff > 0).mean() <= 1e-4, (diff.max(), (diff > 0).mean())
