"""Differentiable energy (torch.autograd with the gradient kernel as backward) and
coupling gradients at relaxed fields.

Tolerances:
  * backward vs dA x (FP64 oracle functional derivative): 1e-11 x max (FP64 fields);
  * backward vs central differences of the discrete energy along a smooth interior
    direction: 1e-3 relative (the kernel is the 4th-order functional derivative, the
    exact derivative of the discrete sum differs by O(h^4));
  * dE_min/dc from the coupling kernel at a relaxed FP64 field vs central differences
    of relaxed energies (dc = 1e-3 x c): 1e-4 relative.
"""
import math

import numpy as np
import pytest
import torch

from oracle import flow64 as ref
from soliton_solver_b200.autograd import coupling_gradients, energy
from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu

CASES = [
    ("Chiral magnet", "chiral_magnet", dict(xlen=64, ylen=72, xsize=4.0, ysize=4.5, dmi_term="Heusler",
                                             demag=True, B=0.2, unit_magnetization=True)),
    ("Baby Skyrme", "baby_skyrme", dict(xlen=60, ylen=64, xsize=6.0, ysize=6.4, unit_magnetization=True)),
    ("Abelian Higgs", "ginzburg_landau_superconductor", dict(xlen=64, ylen=68, xsize=6.3, ysize=6.7)),
    ("s+id superconductor", "anisotropic_superconductor", dict(xlen=56, ylen=60, xsize=5.5, ysize=5.9)),
]


def _smooth(rp, key, seed):
    rng = np.random.default_rng(seed)
    X, Y, nf = rp.xlen, rp.ylen, rp.number_total_fields
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    F = np.stack([0.3 * np.sin(2 * x + rng.normal()) * np.cos(1.5 * y + rng.normal()) for _ in range(nf)])
    if key in ("chiral_magnet", "baby_skyrme"):
        F[2] += 1.0
        F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    return F


@pytest.mark.parametrize("name,key,kw", CASES, ids=[c[1] for c in CASES])
def test_backward_is_the_gradient_kernel(name, key, kw):
    th = load_theory(name)
    rp = th.params.default_params(**kw).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    F = _smooth(rp, key, 3)
    s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
    f = torch.tensor(F.reshape(-1), dtype=torch.float64, device="cuda", requires_grad=True)
    E = energy(f, s)
    assert abs(E.item() - ref.energy(key, F, p_i, p_f)) <= 1e-11 * abs(ref.energy(key, F, p_i, p_f))
    (3.0 * E).backward()
    want = 3.0 * float(p_f[4]) * ref.raw_gradient(key, F, p_i, p_f).reshape(-1)
    got = f.grad.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-11 * np.max(np.abs(want))


@pytest.mark.parametrize("name,key,kw", CASES, ids=[c[1] for c in CASES])
def test_backward_matches_discrete_energy_differences(name, key, kw):
    th = load_theory(name)
    rp = th.params.default_params(**kw).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    F = _smooth(rp, key, 5)
    X, Y = rp.xlen, rp.ylen
    x = np.linspace(0, 1, X)[:, None]
    y = np.linspace(0, 1, Y)[None, :]
    bump = (np.sin(np.pi * x) * np.sin(np.pi * y)) ** 8        # smooth, vanishes near the boundary
    D = np.stack([bump * np.cos(3 * a + 2 * x + y) for a in range(rp.number_total_fields)])
    if key == "anisotropic_superconductor":
        # the reference's s+id condensate rows are not the derivative of its energy
        # (tests/test_oracle_golden.py::test_splusid_condensate_rows_are_not_dE_dpsi);
        # the flow gradient is checked on the gauge rows only
        D[2:] = 0.0
    s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
    f = torch.tensor(F.reshape(-1), dtype=torch.float64, device="cuda", requires_grad=True)
    energy(f, s).backward()
    ad = float(np.dot(f.grad.cpu().numpy(), D.reshape(-1)))
    eps = 1e-5
    fd = (ref.energy(key, F + eps * D, p_i, p_f) - ref.energy(key, F - eps * D, p_i, p_f)) / (2 * eps)
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd)


def _relaxed_energy(th, kw, F0, steps):
    sim = Simulation(th.params.default_params(**kw), th, precision="fp64")
    sim.load_field(F0)
    E0 = sim.observables()["energy"]
    E, err = sim.relax(steps, E0)
    return sim, float(E[-1]), float(np.abs(err[-1]))


def test_lambda_gradient_at_relaxed_vortex():
    """Abelian Higgs: dE_min/dLambda from the coupling kernel vs central differences of
    relaxed energies (single centred vortex)."""
    th = load_theory("Abelian Higgs")
    kw = dict(xlen=96, ylen=96, xsize=12.0, ysize=12.0, Lambda=1.0, q=1.0, u1=1.0, vortex_number=1.0)
    rp = th.params.default_params(**kw).resolved()
    X, Y = rp.xlen, rp.ylen
    x = (np.arange(X) - (X - 1) / 2)[:, None] * rp.lsx
    y = (np.arange(Y) - (Y - 1) / 2)[None, :] * rp.lsy
    r, t = np.hypot(x, y), np.arctan2(y, x)
    F0 = np.stack([0 * r, 0 * r, np.tanh(r) * np.cos(t), np.tanh(r) * np.sin(t)])  # A = 0, one vortex
    steps = 20000
    sim, E, err = _relaxed_energy(th, kw, F0, steps)
    g = coupling_gradients(sim)["Lambda"]
    d = 1e-3
    _, Ep, _ = _relaxed_energy(th, dict(kw, Lambda=1.0 + d), F0, steps)
    _, Em, _ = _relaxed_energy(th, dict(kw, Lambda=1.0 - d), F0, steps)
    fd = (Ep - Em) / (2 * d)
    assert abs(g - fd) <= 1e-4 * abs(fd), (g, fd, err)
