"""Headless colormaps with the reference's kernel names (core/colormaps.py:94-267).

``render_jet_density_to_rgba[grid, block](pbo_rgba, density_flat, xlen, ylen, vmin, vmax)``,
``render_gray_density_to_rgba[...]`` and ``render_magnetization_to_rgba[...](pbo_rgba, Field,
xlen, ylen, p_i)`` accept the reference's launch syntax (the launch configuration is
ignored) and write the same bytes through ``ss_render_rgba`` into ``pbo_rgba``: a
contiguous uint8 device buffer of shape (ylen, xlen, 4) (a torch tensor or anything
exposing ``__cuda_array_interface__``) instead of a mapped GL pixel buffer.  Fields and
densities may be FP32 or FP64; the arithmetic is FP64.  Work is queued on torch's
current stream of the buffer's device.
"""
from __future__ import annotations

import numpy as np
import torch

from soliton_solver_b200 import _native as nat
from soliton_solver_b200.core.hooks import Launch, as_tensor

_PREC = {torch.float32: nat.SS_FP32, torch.float64: nat.SS_FP64}


def _render(kind, pbo_rgba, src, xlen, ylen, vmin=0.0, vmax=1.0):
    out, s = as_tensor(pbo_rgba), as_tensor(src)
    xlen, ylen = int(xlen), int(ylen)
    if out.dtype != torch.uint8 or not out.is_contiguous() or out.numel() != 4 * xlen * ylen:
        raise ValueError("pbo_rgba must be a contiguous uint8 buffer of ylen * xlen * 4 bytes")
    if s.dtype not in _PREC or not s.is_contiguous() or s.device != out.device:
        raise ValueError("src must be a contiguous float32/float64 buffer on the same device")
    need = xlen * ylen * (3 if kind == nat.SS_RENDER_MAGNETIZATION else 1)
    if s.numel() < need:
        raise ValueError(f"src holds {s.numel()} values, the image needs {need}")
    with torch.cuda.device(out.device):
        stream = torch.cuda.current_stream(out.device).cuda_stream
        nat.check(nat.load().ss_render_rgba(kind, s.data_ptr(), _PREC[s.dtype], xlen, ylen, float(vmin),
                                            float(vmax), out.data_ptr(), stream))
    return out


def _jet(pbo_rgba, density_flat, xlen, ylen, vmin, vmax):
    return _render(nat.SS_RENDER_JET, pbo_rgba, density_flat, xlen, ylen, vmin, vmax)


def _gray(pbo_rgba, density_flat, xlen, ylen, vmin, vmax):
    return _render(nat.SS_RENDER_GRAY, pbo_rgba, density_flat, xlen, ylen, vmin, vmax)


def _magnetization(pbo_rgba, Field, xlen, ylen, p_i):
    # the reference takes the plane stride from p_i[0] * p_i[1]; it equals xlen * ylen
    p = np.asarray(p_i.cpu() if isinstance(p_i, torch.Tensor) else p_i)
    if int(p[0]) != int(xlen) or int(p[1]) != int(ylen):
        raise ValueError("p_i[0:2] must equal (xlen, ylen)")
    return _render(nat.SS_RENDER_MAGNETIZATION, pbo_rgba, Field, xlen, ylen)


render_jet_density_to_rgba = Launch(_jet, "render_jet_density_to_rgba")
render_gray_density_to_rgba = Launch(_gray, "render_gray_density_to_rgba")
render_magnetization_to_rgba = Launch(_magnetization, "render_magnetization_to_rgba")
