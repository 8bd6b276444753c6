"""Simulation.minimize: relaxation to max|dE/dphi| < tol through the product API (GPU).

C2 (chiral magnet 320^2 over 10 x 10 J/D, Heusler, demag off, B = 0, anti-skyrmion, arrested
Newton flow): the default FP32 schedule ("fp32+fp64": FP32 flow until its energy plateaus
or it stalls at FP32 resolution, then FP64 on the projected state) must converge (err < 1e-6)
without reaching max_steps,
and its relaxed energy must equal the FP64-only minimum to 1e-6 relative (the metric's
accuracy gate; measured ~1e-11).  The FP32 phase's projected FP64 energy at the switch is
within 1e-6 as well.
"""
import math

import numpy as np
import pytest
import torch

from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.initial_conditions import anti_skyrmion, hedgehog
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu


def _c2(prec):
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=320, ylen=320, xsize=10.0, ysize=10.0, J=40e-12, K=0.8e6, D=4e-3, M=580e3,
                                 B=0.0, dmi_term="Heusler", demag=False, unit_magnetization=True, killkinen=True)
    sim = Simulation(p, th, precision=prec)
    sim.load_field(anti_skyrmion(sim.rp, R=1.0, sigma=1e-3, seed=0, device="cuda"))
    return sim


@pytest.fixture(scope="module")
def c2_fp64_minimum():
    sim = _c2("fp64")
    res = sim.minimize(tol=1e-6, max_steps=400_000)
    assert res["converged"] and res["phases"][0]["stop"] == "tol"
    return res["energy"]


def test_c2_default_schedule_meets_the_1e6_gate(c2_fp64_minimum):
    sim = _c2("fp32")
    res = sim.minimize(tol=1e-6, max_steps=400_000, record=True)
    assert res["schedule"] == "fp32+fp64"
    assert res["converged"] and res["steps"] < 400_000
    assert [ph["precision"] for ph in res["phases"]] == ["fp32", "fp64"]
    assert res["phases"][0]["stop"] == "plateau" and res["phases"][1]["stop"] == "tol"
    assert abs(res["energy"] - c2_fp64_minimum) <= 1e-6 * abs(c2_fp64_minimum), (res["energy"], c2_fp64_minimum)
    proj = res["trajectory"]["projected"]
    assert abs(proj[-1, 1] - c2_fp64_minimum) <= 1e-6 * abs(c2_fp64_minimum)
    # the relaxed state lands in the Simulation's FP32 buffers and, in FP64, in sim.Field64
    assert sim.Field64.dtype == torch.float64
    assert abs(sim.observables()["skyrmion_number"] - round(sim.observables()["skyrmion_number"])) < 1e-4
    # whole chunks are recorded; the run stops inside the last one, at the step below tol
    assert 0 <= len(res["trajectory"]["energy"]) - res["steps"] < 1000


def test_minimize_fp32_only_and_argument_checks():
    th = load_theory("Baby Skyrme")
    p = th.params.default_params(xlen=64, ylen=64, lsx=0.1, lsy=0.1, time_step=0.01, unit_magnetization=True,
                                 killkinen=True)
    sim = Simulation(p, th, precision="fp32")
    sim.load_field(hedgehog(sim.rp, charge=1, R=1.5, seed=0, device="cuda"))
    res = sim.minimize(tol=1e-3, max_steps=20_000, schedule="fp32", chunk=500)
    assert len(res["phases"]) == 1 and res["phases"][0]["precision"] == "fp32"
    assert res["steps"] <= 20_000 and math.isfinite(res["energy"])
    with pytest.raises(ValueError, match="schedule"):
        sim.minimize(schedule="fp16")
    sim64 = Simulation(p, th, precision="fp64")
    with pytest.raises(ValueError, match="FP32 Simulation"):
        sim64.minimize(schedule="fp32")
    off = Simulation(th.params.default_params(xlen=32, ylen=32, killkinen=False), th)
    with pytest.raises(ValueError, match="killkinen"):
        off.minimize()


def test_convert_field_round_trip_and_projection():
    """ss_convert_field: FP32 -> FP64 with the unit vectors renormalised in FP64, and back."""
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=40, ylen=36, unit_magnetization=True, demag=True)
    sim = Simulation(p, th, precision="fp32")
    g = torch.Generator(device="cuda").manual_seed(3)
    f = torch.randn(4, 40 * 36, device="cuda", generator=g)
    f[:3] /= f[:3].norm(dim=0)
    sim.Field.copy_(f.reshape(-1))
    F64 = torch.empty(sim.Field.numel(), dtype=torch.float64, device="cuda")
    sim.solver.convert(sim.Field, F64, project=True)
    m = F64.view(4, -1)
    want = sim.Field.view(4, -1).double()
    want_m = want[:3] / want[:3].norm(dim=0)
    assert torch.allclose(m[:3], want_m, rtol=0, atol=1e-15)
    assert torch.equal(m[3], want[3])
    assert float((m[:3].norm(dim=0) - 1).abs().max()) < 1e-15
    back = torch.empty_like(sim.Field)
    sim.solver.convert(F64, back, project=False)
    assert torch.equal(back.view(4, -1)[3], sim.Field.view(4, -1)[3])
    assert float((back - sim.Field).abs().max()) <= 3e-7
    raw = torch.empty_like(F64)
    sim.solver.convert(sim.Field, raw, project=False)
    assert torch.equal(raw, sim.Field.double())
    np.testing.assert_array_equal(raw.cpu().numpy(), sim.Field.double().cpu().numpy())
