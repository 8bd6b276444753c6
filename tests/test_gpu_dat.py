"""GPU text formatting (ss_format_text, soliton_solver_b200.core.io) against the
reference's files and Python's own formatting: byte-identical.

The golden inputs mix random magnitudes over the whole double range with the edge cases
of the "g" format; a further random sweep (all exponents, FP64 and FP32 values, several
precisions) is compared with Python's format() directly.
"""
import os

import numpy as np
import pytest
import torch

from oracle import io as oio
from soliton_solver_b200.core import io as sio

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _read(*names):
    return open(os.path.join(GOLDEN, "dat", *names), "rb").read()


@pytest.mark.parametrize("p", [32, 16, 8])
def test_writers_match_reference_files(tmp_path, p):
    g = np.load(os.path.join(GOLDEN, "dat_values.npz"))
    X, Y, nf = int(g["xlen"]), int(g["ylen"]), int(g["nf"])
    sio.output_field_dat(g["field"], str(tmp_path / "f.dat"), X, Y, nf, precision=p)
    assert (tmp_path / "f.dat").read_bytes() == _read(f"field_p{p}.dat")
    sio.output_density_data_dat(torch.tensor(g["density"], device="cuda"), 1, str(tmp_path / "d.dat"), X, Y,
                                precision=p)
    assert (tmp_path / "d.dat").read_bytes() == _read(f"density1_p{p}.dat")
    sio.output_iteration_data_dat(list(g["iters"]), str(tmp_path / "i.dat"), precision=p)
    assert (tmp_path / "i.dat").read_bytes() == _read(f"iters_p{p}.dat")


def test_bundle_matches_reference(tmp_path):
    g = np.load(os.path.join(GOLDEN, "dat_values.npz"))
    X, Y, nf = int(g["xlen"]), int(g["ylen"]), int(g["nf"])
    out = tmp_path / "bundle"
    sio.output_data_bundle_core(str(out), h_Field=g["field"], h_grid=g["grid"], xlen=X, ylen=Y, number_coordinates=2,
                                number_total_fields=nf, precision=32,
                                bundle_spec=[("grid", 0, "xGrid.dat"), ("grid", 1, "yGrid.dat"),
                                             ("Field", 2, "MagnetField3.dat"), ("Density", 1, "Density.dat"),
                                             ("Missing", 0, "Missing.dat")],
                                arrays={"grid": g["grid"], "Field": g["field"], "Density": g["density"]},
                                field_dump_name="Field.dat")
    names = sorted(os.listdir(os.path.join(GOLDEN, "dat", "bundle")))
    assert sorted(os.listdir(out)) == names
    for n in names:
        assert (out / n).read_bytes() == _read("bundle", n), n


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("p", [1, 6, 17, 32, 40])
def test_random_sweep_vs_python_format(p, dtype):
    rng = np.random.default_rng(p)
    n = 20000
    if dtype == np.float64:
        bits = rng.integers(0, 2 ** 63, n, dtype=np.int64).view(np.float64)
        v = np.where(np.isfinite(bits), bits, 1.0) * rng.choice([-1.0, 1.0], n)  # every exponent, both signs
        v[:2000] = [round(float(x), int(d)) for x, d in zip(rng.standard_normal(2000), rng.integers(0, 12, 2000))]
        v[2000:4000] = rng.integers(-10 ** 6, 10 ** 6, 2000) * 2.0 ** rng.integers(-60, 10, 2000)  # dyadic
    else:
        bits = rng.integers(0, 2 ** 31, n, dtype=np.int32).view(np.float32)
        v = np.where(np.isfinite(bits), bits, np.float32(1.0)).astype(np.float32)
    got = sio.format_text(v, p, row=7, block=100)
    want = "".join(f"{{:.{p}g}}".format(float(x)) + "\t" + ("\n" if (i + 1) % 7 == 0 else "")
                   + ("\n" if (i + 1) % 100 == 0 else "") for i, x in enumerate(v)).encode()
    assert got == want


def test_save_output_bundle(tmp_path):
    """Simulation.save_output writes the theory's file set; the field dump and the
    energy density match the restatement of the writers byte for byte."""
    from soliton_solver_b200.core.simulation import Simulation
    from soliton_solver_b200.theories import load_theory
    th = load_theory("Chiral magnet")
    sim = Simulation(th.params.default_params(xlen=24, ylen=20, xsize=3.0, ysize=2.5), th, precision="fp64")
    sim.initialize({"mode": "initial", "ansatz": "neel"})
    sim.save_output(str(tmp_path), precision=32)
    names = sorted(os.listdir(tmp_path))
    assert names == sorted(["LatticePoints.dat", "LatticeVectors.dat", "Field.dat", "xGrid.dat", "yGrid.dat",
                            "MagnetField1.dat", "MagnetField2.dat", "MagnetField3.dat", "SkyrmionChargeDensity.dat",
                            "EnergyDensity.dat", "MagneticChargeDensity.dat"])
    F = sim.Field.cpu().numpy()
    assert (tmp_path / "Field.dat").read_bytes() == oio.field_text(F, 24, 20, 4, 32)
    en = sim.solver.energy_density(sim.Field).cpu().numpy()
    assert (tmp_path / "EnergyDensity.dat").read_bytes() == oio.density_text(en, 0, 24, 20, 32)
    assert (tmp_path / "LatticePoints.dat").read_bytes() == b"24\t20\t"
