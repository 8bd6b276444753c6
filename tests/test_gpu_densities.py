"""Diagnostic densities of the gauge theories on the GPU (ss_field_density) against the
reference's own outputs (tests/golden/density_*.npz, written by the reference's
Simulation helpers compute_higgs*_density, compute_phase_difference_density,
supercurrent and magnetic_field) and the oracle.

Tolerances: FP64 fields 1e-12 x max|reference| per entry (difference-form stencils and
libm ulps); FP32 fields against the oracle evaluated on the FP32-rounded field, 1e-12 x
max (the densities are evaluated in FP64 on the stored values).
"""
import glob
import os

import numpy as np
import pytest
import torch

from oracle import flow64 as ref
from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "density_*.npz")))
NAMES = {"ginzburg_landau_superconductor": "Abelian Higgs", "anisotropic_superconductor": "s+id superconductor"}
KINDS = ("higgs", "higgs1", "higgs2", "phase", "magnetic", "supercurrent")


def _close(got, want, what):
    got = np.asarray(got, np.float64).reshape(-1)
    want = np.asarray(want, np.float64).reshape(-1)
    scale = max(1.0, float(np.max(np.abs(want))))
    err = float(np.max(np.abs(got - want)))
    assert err <= 1e-12 * scale, f"{what}: max err {err:.3e} vs scale {scale:.3e}"


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[8:-4] for p in CASES])
def test_field_densities_vs_reference(path, prec):
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    F = np.asarray(g["field"], np.float64)
    if prec == "fp32":
        F = F.astype(np.float32).astype(np.float64)
    theory = load_theory(NAMES[th])
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f = torch.tensor(F, dtype=torch.float32 if prec == "fp32" else torch.float64, device="cuda")
    Fo = ref.as_field(F, p_i)
    for kind in (k for k in KINDS if k in g):
        got = s.field_density(f, kind).cpu().numpy()
        want = g[kind] if prec == "fp64" else ref.field_density(th, Fo, p_i, p_f, kind)
        _close(got, want, f"{kind} {prec}")


def test_density_kinds_are_checked_per_theory():
    th = load_theory("Abelian Higgs")
    rp = th.params.default_params(xlen=20, ylen=20).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
    f = torch.zeros(4 * 400, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="not defined"):
        s.field_density(f, "phase")


def test_simulation_helpers_hooks_and_output_bundle(tmp_path):
    """The Simulation methods and the kernels-module hooks give the same densities as
    the reference on the golden s+id field, and save_output writes the supercurrent and
    flux files from them."""
    g = np.load(os.path.join(GOLDEN, "density_sid_default.npz"))
    theory = load_theory("s+id superconductor")
    p_i = g["p_i"]
    kw = dict(xlen=int(p_i[0]), ylen=int(p_i[1]), xsize=2.4, ysize=1.8)
    sim = Simulation(theory.params.default_params(**kw), theory, precision="fp64")
    assert np.array_equal(sim.p_f_h, g["p_f"]) and np.array_equal(sim.p_i_h, p_i)
    sim.load_field(np.asarray(g["field"]))
    N = sim.rp.xlen * sim.rp.ylen
    for method, key in ((sim.compute_higgs1_density, "higgs1"), (sim.compute_higgs2_density, "higgs2"),
                        (sim.compute_phase_difference_density, "phase")):
        method()
        _close(sim.en.cpu().numpy(), g[key], key)
    _close(sim.magnetic_field().cpu().numpy()[:N], g["magnetic"], "magnetic_field")
    _close(sim.supercurrent().cpu().numpy()[:2 * N], g["supercurrent"], "supercurrent")
    # the reference-named hooks with the reference's argument orders
    k = theory.kernels
    out = torch.zeros(2 * N, dtype=torch.float64, device="cuda")
    k.compute_supercurrent_kernel[None, None](sim.Field, sim.d2fd2x, out, sim.p_i_d, sim.p_f_d)
    _close(out.cpu().numpy(), g["supercurrent"], "compute_supercurrent_kernel")
    k.compute_norm_higgs2_kernel[None, None](out, sim.Field, sim.p_i_d)
    _close(out.cpu().numpy()[:N], g["higgs2"], "compute_norm_higgs2_kernel")
    k.compute_magnetic_field_kernel[None, None](sim.Field, sim.d1fd1x, out, sim.p_i_d, sim.p_f_d)
    _close(out.cpu().numpy()[:N], g["magnetic"], "compute_magnetic_field_kernel")
    # scratch attributes of the reference's Simulation exist with its sizes
    assert sim.d1fd1x.numel() == 2 * 6 * N and sim.d2fd2x.numel() == 4 * 6 * N and sim.k1.numel() == 6 * N
    sim.save_output(str(tmp_path), precision=17)
    for name in ("Supercurrent1.dat", "Supercurrent2.dat", "ChargeDensity.dat"):
        assert (tmp_path / name).exists(), name
    rows = [r for r in (tmp_path / "Supercurrent2.dat").read_text().split("\n") if r.strip()]
    vals = np.array([[float(v) for v in r.split("\t") if v] for r in rows])
    _close(vals.reshape(-1), np.asarray(g["supercurrent"])[N:], "Supercurrent2.dat")


def test_abelian_higgs_has_no_magnetic_field_kernel():
    theory = load_theory("Abelian Higgs")
    sim = Simulation(theory.params.default_params(xlen=16, ylen=16), theory, precision="fp64")
    with pytest.raises(AttributeError):
        sim.magnetic_field()
    sim.compute_higgs_density()
    assert sim.supercurrent().numel() == 2 * 256
