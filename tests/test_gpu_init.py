"""Native initial-condition kernels (ss_initialize, ss_insert_soliton) against the
reference's kernels (golden) and the oracle.

Tolerances: FP64 fields 1e-13 relative to the largest magnitude (CUDA's and the host's
sin/cos/exp/atan2/tanh differ in the last ulp); FP32 fields 1e-6 (one rounding of an
FP64 value).  Velocity is zeroed by the ground state and the ansatz.  The calls go
through the reference-named hooks of each theory's initial_config module.
"""
import glob
import os

import numpy as np
import pytest
import torch

from oracle import init as oi
from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "init_*.npz")))
NAMES = {"chiral_magnet": "Chiral magnet", "baby_skyrme": "Baby Skyrme model",
         "ginzburg_landau_superconductor": "Ginzburg-Landau superconductor",
         "anisotropic_superconductor": "Anisotropic superconductor"}


def _flags(g):
    b, n, a = (bool(int(v)) for v in g["ansatz"]) if "ansatz" in g else (False, False, False)
    return b, n, a


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-4] for p in GOLDEN])
def test_init_matches_reference_kernels(path, dtype):
    g = np.load(path)
    key, p_i, p_f = str(g["theory"]), g["p_i"], g["p_f"]
    ic = load_theory(NAMES[key]).initial_config
    n = int(p_i[6])
    mode = int(g["mode"])
    V = torch.full((n,), 0.7, dtype=dtype, device="cuda")
    scratch = [torch.full((n,), 0.5, dtype=dtype, device="cuda") for _ in range(9)]
    if mode == 2:
        F = torch.tensor(g["before"], dtype=dtype, device="cuda")
        if key in ("chiral_magnet", "baby_skyrme"):
            ic.create_skyrmion_kernel[None, None](F, None, int(g["pxi"]), int(g["pxj"]), float(g["rotation"]),
                                                  *_flags(g), p_i, p_f)
        else:
            ic.create_vortex_kernel[None, None](F, None, int(g["pxi"]), int(g["pxj"]), bool(g["vortex"]), p_i, p_f)
    else:
        F = torch.full((n,), 0.3, dtype=dtype, device="cuda")
        if mode == 0:
            ic.create_ground_state_kernel[None, None](V, F, None, *scratch, p_i, p_f)
        elif key in ("chiral_magnet", "baby_skyrme"):
            ic.create_initial_configuration_kernel[None, None](V, F, None, *scratch, *_flags(g), float(g["rotation"]),
                                                               1.0, p_i, p_f)
        elif key == "ginzburg_landau_superconductor":
            ic.create_initial_configuration_kernel[None, None](V, F, None, *scratch, float(g["vortex_number"]), p_i,
                                                               p_f)
        else:
            ic.create_initial_configuration_kernel[None, None](V, F, None, *scratch, p_i, p_f)
        assert torch.count_nonzero(V).item() == 0
        assert all(torch.count_nonzero(b).item() == 0 for b in scratch)
    torch.cuda.synchronize()
    want = g["field"]
    tol = 1e-13 if dtype == torch.float64 else 1e-6
    got = F.double().cpu().numpy()
    assert np.max(np.abs(got - want)) <= tol * max(1.0, np.max(np.abs(want)))


@pytest.mark.parametrize("key,kw,cfg", [
    ("chiral_magnet", dict(xlen=200, ylen=160, xsize=20.0, ysize=16.0), {"mode": "initial", "ansatz": "neel",
                                                                         "skyrmion_rotation": 0.7}),
    ("baby_skyrme", dict(xlen=160, ylen=192, xsize=16.0, ysize=19.2, skyrmion_number=3.0), {}),
    ("ginzburg_landau_superconductor", dict(xlen=256, ylen=200, xsize=20.0, ysize=15.6), {"vortex_number": 3.0}),
    ("anisotropic_superconductor", dict(xlen=180, ylen=200, xsize=12.0, ysize=13.3), {}),
])
def test_simulation_initialize_vs_oracle(key, kw, cfg):
    """sim.initialize with the reference's default mode ("initial") and config keys,
    then a skyrmion / vortex inserted off centre, against the oracle."""
    th = load_theory(NAMES[key])
    sim = Simulation(th.params.default_params(**kw), th, precision="fp64")
    sim.initialize(cfg)
    p_i, p_f = sim.p_i_h, sim.p_f_h
    ansatz = {"bloch": oi.ANSATZ_BLOCH, "neel": oi.ANSATZ_NEEL, "anti": oi.ANSATZ_ANTI}[cfg.get("ansatz", "bloch")]
    want = oi.initial(key, p_i, p_f, ansatz, float(cfg.get("skyrmion_rotation", 0.0)),
                      float(cfg.get("vortex_number", 1.0)))
    got = sim.Field.cpu().numpy().reshape(want.shape)
    assert np.max(np.abs(got - want)) <= 1e-13 * max(1.0, np.max(np.abs(want)))
    pxi, pxj = kw["xlen"] // 3, kw["ylen"] // 4
    if key in ("chiral_magnet", "baby_skyrme"):
        th.initial_config.create_skyrmion_kernel[None, None](sim.Field, sim.grid, pxi, pxj, 0.2, False, False, True,
                                                             p_i, p_f)
        want = oi.insert(key, want, p_i, p_f, pxi, pxj, oi.ANSATZ_ANTI, 0.2)
    else:
        th.initial_config.create_vortex_kernel[None, None](sim.Field, sim.grid, pxi, pxj, True, p_i, p_f)
        want = oi.insert(key, want, p_i, p_f, pxi, pxj, vortex=True)
    torch.cuda.synchronize()
    got = sim.Field.cpu().numpy().reshape(want.shape)
    assert np.max(np.abs(got - want)) <= 1e-13 * max(1.0, np.max(np.abs(want)))
