"""Plain-text .dat output of lattice arrays, formatted on the GPU.

Same functions, arguments and bytes as soliton_solver/core/io.py:16-240
(``_flat``, ``output_field_dat``, ``output_iteration_data_dat``,
``output_density_data_dat``, ``output_data_bundle_core``): every value as Python's
``format(v, ".{precision}g")`` followed by a tab, a newline after each lattice row and
a blank line after each field component.  The formatting runs in libsoliton_b200
(``ss_format_text``: exact decimal conversion per value on the device, a length scan,
one write pass); the text is copied to the host once and written with one call.
Arrays may be host numpy arrays or device tensors (FP32 or FP64).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from soliton_solver_b200 import _native as nat


def _flat(a: int, x: int, y: int, xlen: int, ylen: int) -> int:
    return y + x * ylen + a * xlen * ylen


def _device_values(values, device=None):
    if isinstance(values, torch.Tensor):
        t = values.detach()
        if t.dtype not in (torch.float32, torch.float64):
            t = t.to(torch.float64)
        if not t.is_cuda:
            t = t.to(device or "cuda")
        return t.contiguous().reshape(-1)
    a = np.asarray(values)
    if a.dtype != np.float32:
        a = a.astype(np.float64)
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(device or "cuda")


def format_text(values, precision: int = 32, row: int = 0, block: int = 0) -> bytes:
    """The .dat text of `values` (flat, in write order): each value formatted as
    format(v, f".{precision}g") plus a tab, a newline after every `row` values and
    another after every `block` values (0: none)."""
    v = _device_values(values)
    n = int(v.numel())
    if n == 0:
        return b""
    lib = nat.load()
    prec = nat.SS_FP32 if v.dtype == torch.float32 else nat.SS_FP64
    nbytes = ctypes.c_size_t()
    nat.check(lib.ss_text_workspace_bytes(n, ctypes.byref(nbytes)))
    with torch.cuda.device(v.device):
        ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=v.device)
        stream = torch.cuda.current_stream(v.device).cuda_stream
        length = ctypes.c_longlong()
        nat.check(lib.ss_format_text(v.data_ptr(), prec, n, int(precision), int(row), int(block), None, 0,
                                     ctypes.byref(length), ws.data_ptr(), ws.numel(), stream))
        out = torch.empty(max(int(length.value), 1), dtype=torch.uint8, device=v.device)
        nat.check(lib.ss_format_text(v.data_ptr(), prec, n, int(precision), int(row), int(block), out.data_ptr(),
                                     out.numel(), ctypes.byref(length), ws.data_ptr(), ws.numel(), stream))
        host = out[: int(length.value)].cpu()
    return host.numpy().tobytes()


def _select(arr, count: int, offset: int = 0):
    if isinstance(arr, torch.Tensor):
        return arr.reshape(-1)[offset: offset + count]
    return np.asarray(arr).reshape(-1)[offset: offset + count]


def output_field_dat(field_flat, path: str, xlen: int, ylen: int, nfields: int, precision: int = 32) -> None:
    n = int(xlen) * int(ylen)
    text = format_text(_select(field_flat, n * int(nfields)), precision, row=int(ylen), block=n)
    with open(path, "wb") as f:
        f.write(text)


def output_iteration_data_dat(values, path: str, precision: int = 32) -> None:
    vals = np.asarray([float(v) for v in values], dtype=np.float64)
    text = format_text(vals, precision) if vals.size else b""
    with open(path, "wb") as f:
        f.write(text)


def output_density_data_dat(density_flat, a: int, path: str, xlen: int, ylen: int, precision: int = 32) -> None:
    n = int(xlen) * int(ylen)
    text = format_text(_select(density_flat, n, int(a) * n), precision, row=int(ylen))
    with open(path, "wb") as f:
        f.write(text)


def output_data_bundle_core(output_dir: str, *, h_Field, h_grid, xlen: int, ylen: int, number_coordinates: int,
                            number_total_fields: int, precision: int, bundle_spec, arrays,
                            lattice_points_name: str = "LatticePoints.dat",
                            lattice_vectors_name: str = "LatticeVectors.dat",
                            field_dump_name: str = "d_Field.dat") -> None:
    """Lattice sizes, lattice vectors, the full field dump and the component grids
    named in `bundle_spec` ((array_key, component, filename) entries; missing or None
    arrays are skipped), as soliton_solver/core/io.py:185-240 writes them."""
    os.makedirs(output_dir, exist_ok=True)
    lattice_points = np.array([xlen, ylen], dtype=np.float64)
    g = _select(h_grid, 2 * int(xlen) * int(ylen))
    g = g.detach().cpu().numpy() if isinstance(g, torch.Tensor) else np.asarray(g)
    x_max = float(g[_flat(0, xlen - 1, ylen - 1, xlen, ylen)]) if number_coordinates >= 1 else 0.0
    y_max = float(g[_flat(1, xlen - 1, ylen - 1, xlen, ylen)]) if number_coordinates >= 2 else 0.0
    lattice_vectors = np.array([x_max, 0.0, 0.0, y_max], dtype=np.float64)
    output_iteration_data_dat(lattice_points[:number_coordinates], os.path.join(output_dir, lattice_points_name),
                              precision=precision)
    output_iteration_data_dat(lattice_vectors[:number_coordinates * number_coordinates],
                              os.path.join(output_dir, lattice_vectors_name), precision=precision)
    output_field_dat(h_Field, os.path.join(output_dir, field_dump_name), xlen, ylen, number_total_fields,
                     precision=precision)
    for array_key, a, filename in bundle_spec:
        if array_key not in arrays:
            continue
        arr = arrays[array_key]
        if arr is None:
            continue
        output_density_data_dat(arr, int(a), os.path.join(output_dir, filename), xlen, ylen, precision=precision)
