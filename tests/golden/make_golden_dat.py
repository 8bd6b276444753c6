"""Golden .dat files from the reference's own text writers (soliton_solver/core/io.py).

Run in a container that has the reference checkout (it is NOT needed at test time):

    python tests/golden/make_golden_dat.py --ref <reference checkout> --out tests/golden

The writers are plain Python (no GPU, no Numba kernel), so they are imported and
called directly: ``output_field_dat``, ``output_density_data_dat``,
``output_iteration_data_dat`` and ``output_data_bundle_core`` on seeded arrays that
mix random magnitudes across the whole double range with edge values (signed zeros,
subnormals, NaN, infinities, the fixed/scientific boundaries of the "g" format,
values that round up to a new power of ten, and exact binary fractions whose decimal
expansion ends in a 5 at the rounding digit).  Writes ``dat_values.npz`` (the inputs)
and the text files under ``dat/``.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def edge_values():
    v = [0.0, -0.0, 1.0, -1.0, 0.5, 1e16, 1e15, 9.999999999999999e15, 1e-4, 1e-5, 9.99999e-5, 0.00010000000000000002,
         123.456, -123.456, 1.0 / 3.0, 2.0 / 3.0, 5e-324, -5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
         -1.7976931348623157e308, 2.0 ** -46, 2.0 ** -49, 3 * 2.0 ** -52, 0.1, 0.2, 0.3, 1e22, 1e23, 123456789012345680.0,
         9.5, 0.95, 99.99999999999999, 1e100, 1e-100, float("nan"), float("inf"), float("-inf"), 6.02214076e23,
         np.float32(0.1).item(), np.float32(1e-30).item(), np.float32(3.4028235e38).item(), 4.9406564584124654e-324 * 7]
    return np.array(v, dtype=np.float64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SOLITON_SOLVER_REF"), required="SOLITON_SOLVER_REF" not in os.environ,
                    help="root of the reference soliton_solver checkout (or set SOLITON_SOLVER_REF)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    sys.path.insert(0, args.ref)
    from soliton_solver.core import io as rio

    rng = np.random.default_rng(77)
    X, Y, nf = 9, 7, 4
    n = X * Y * nf
    mags = 10.0 ** rng.uniform(-320, 308, n)
    field = rng.choice([-1.0, 1.0], n) * mags * rng.uniform(1, 10, n)
    e = edge_values()
    field[: e.size] = e
    dens = rng.standard_normal(2 * X * Y) * 10.0 ** rng.integers(-6, 6, 2 * X * Y)
    iters = np.array([12.566370614359172, 1.2e-7, -0.0, 3.0, 1e-5])
    grid = np.concatenate([(0.25 * np.arange(X)[:, None] * np.ones((1, Y))).reshape(-1),
                           (0.3 * np.arange(Y)[None, :] * np.ones((X, 1))).reshape(-1)])
    out = os.path.join(args.out, "dat")
    os.makedirs(out, exist_ok=True)
    np.savez_compressed(os.path.join(args.out, "dat_values.npz"), field=field, density=dens, iters=iters, grid=grid,
                        xlen=X, ylen=Y, nf=nf)
    for p in (32, 16, 8):
        rio.output_field_dat(field, os.path.join(out, f"field_p{p}.dat"), X, Y, nf, precision=p)
        rio.output_density_data_dat(dens, 1, os.path.join(out, f"density1_p{p}.dat"), X, Y, precision=p)
        rio.output_iteration_data_dat(iters, os.path.join(out, f"iters_p{p}.dat"), precision=p)
    rio.output_data_bundle_core(os.path.join(out, "bundle"), h_Field=field, h_grid=grid, xlen=X, ylen=Y,
                                number_coordinates=2, number_total_fields=nf, precision=32,
                                bundle_spec=[("grid", 0, "xGrid.dat"), ("grid", 1, "yGrid.dat"),
                                             ("Field", 2, "MagnetField3.dat"), ("Density", 1, "Density.dat"),
                                             ("Missing", 0, "Missing.dat")],
                                arrays={"grid": grid, "Field": field, "Density": dens},
                                field_dump_name="Field.dat")
    print("wrote", out)


if __name__ == "__main__":
    main()
