"""The exact derivative of the discrete energy sum and the discretisation-consistent adjoint (GPU).

1. ss_energy_gradient_exact against directional derivatives of the oracle's FP64 energy
   (the reference's compute_energy restated): for a random direction v, dA <X, v> equals
   the Richardson-extrapolated central difference (4 D(eps/2) - D(eps)) / 3 of E_h, which
   is exact for energies of degree <= 4 in the field (all four theories) up to rounding;
   tolerance 1e-9 relative.  The residual X - S (S: the flow's stencil derivative) shrinks
   like h^4 under refinement in the interior.
2. relaxed_coupling_gradients on the chiral magnet at h = 10/255, where the envelope value at
   the flow's relaxed state is off by ~4.6e-4 (the flow's stencil gradient is not the
   derivative of the discrete energy: O(h^4) inside, O(1/h) next to the frozen ring): with
   the adjoint's linear-response correction (one MINRES solve) dE_min/dB matches central
   differences of relaxed energies to 1e-5.
3. ss_set_forcing adds a fixed field to the flow's gradient in every stage.
"""
import numpy as np
import pytest
import torch

from oracle import flow64 as ref
from soliton_solver_b200.autograd import coupling_gradients, relaxed_coupling_gradients
from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.initial_conditions import anti_skyrmion
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu

CASES = [
    ("Chiral magnet", "chiral_magnet", dict(xlen=22, ylen=19, xsize=2.0, ysize=1.7, dmi_term="Hybrid", demag=True,
                                            B=0.2, unit_magnetization=True)),
    ("Baby Skyrme", "baby_skyrme", dict(xlen=20, ylen=21, xsize=2.1, ysize=2.2, potential="Standard", kappa=1.3,
                                        unit_magnetization=True)),
    ("Abelian Higgs", "ginzburg_landau_superconductor", dict(xlen=19, ylen=20, xsize=2.0, ysize=2.1, Lambda=0.7,
                                                             q=1.2)),
    ("s+id superconductor", "anisotropic_superconductor", dict(xlen=18, ylen=20, xsize=1.9, ysize=2.1, beta4=-0.3,
                                                               gamma12=0.3)),
]


@pytest.mark.parametrize("name,key,kw", CASES, ids=[c[1] for c in CASES])
def test_exact_gradient_is_the_derivative_of_the_energy_sum(name, key, kw):
    th = load_theory(name)
    rp = th.params.default_params(**kw).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    rng = np.random.default_rng(5)
    F = 0.3 * rng.standard_normal((rp.number_total_fields, rp.xlen, rp.ylen))
    F[2] += 0.8
    if key in ("chiral_magnet", "baby_skyrme"):
        F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
    f = torch.tensor(F.reshape(-1), device="cuda")
    s.bind(f, torch.zeros_like(f))
    X = s.energy_gradient_exact(f).cpu().numpy()
    dA = float(p_f[4])
    for seed in (1, 2):
        v = np.random.default_rng(seed).standard_normal(F.shape)

        def D(eps):
            return (ref.energy(key, F + eps * v, p_i, p_f) - ref.energy(key, F - eps * v, p_i, p_f)) / (2 * eps)

        fd = (4 * D(5e-4) - D(1e-3)) / 3
        an = dA * float(np.dot(X, v.reshape(-1)))
        assert abs(an - fd) <= 1e-9 * max(abs(fd), 1e-3), (an, fd)


def _smooth_skyrmion(rp, R=1.0):
    """The Belavin-Polyakov skyrmion m = (2 R x, 2 R y, r^2 - R^2) / (r^2 + R^2): analytic
    everywhere (profiles such as pi exp(-r/R) or pi exp(-r^2/2) leave non-analytic terms at
    the centre, where the 4th-order stencils' error does not shrink like h^4)."""
    x = (torch.arange(rp.xlen, dtype=torch.float64) - (rp.xlen - 1) / 2)[:, None] * rp.lsx
    y = (torch.arange(rp.ylen, dtype=torch.float64) - (rp.ylen - 1) / 2)[None, :] * rp.lsy
    x, y = x.expand(rp.xlen, rp.ylen), y.expand(rp.xlen, rp.ylen)
    d = x * x + y * y + R * R
    m = torch.stack([2 * R * x / d, 2 * R * y / d, (x * x + y * y - R * R) / d, torch.zeros_like(d)])
    return m.reshape(-1).cuda()


def test_stencil_residual_shrinks_like_h4():
    """X - S for a smooth chiral field sampled at two spacings: the interior residual falls
    by ~2^4 when h halves (the stencil gradient is the 4th-order functional derivative)."""
    th = load_theory("Chiral magnet")
    res = []
    for n in (64, 128):
        kw = dict(xlen=n, ylen=n, xsize=6.0, ysize=6.0, dmi_term="Heusler", demag=False, unit_magnetization=True)
        rp = th.params.default_params(**kw).resolved()
        p_i, p_f = th.params.pack_device_params(rp)
        s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
        f = _smooth_skyrmion(rp)
        s.bind(f, torch.zeros_like(f))
        r = s.energy_gradient_exact(f, minus_stencil=True).view(4, n, n)[:3]
        q = n // 4
        res.append(float(r[:, q:3 * q, q:3 * q].abs().max()))
    ratio = res[0] / res[1]
    assert 10.0 < ratio < 24.0, res


def _relaxed(th, kw, field, steps):
    sim = Simulation(th.params.default_params(**kw), th, precision="fp64")
    sim.load_field(field(sim.rp))
    E, _ = sim.relax(steps, sim.observables()["energy"])
    return sim, float(E[-1])


def test_corrected_chiral_adjoint_matches_finite_differences():
    th = load_theory("Chiral magnet")
    kw = dict(xlen=256, ylen=256, xsize=10.0, ysize=10.0, J=40e-12, K=0.8e6, D=4e-3, M=580e3, B=0.2,
              dmi_term="Heusler", demag=False, unit_magnetization=True)
    sim, _ = _relaxed(th, kw, lambda rp: anti_skyrmion(rp, R=1.0, seed=0, device="cuda"), 150000)
    plain = coupling_gradients(sim)["B"]
    g, info = relaxed_coupling_gradients(sim, names=("B",))
    F = sim.Field.clone()
    d = 2e-3 * kw["B"]  # central-difference truncation ~d^2/6 relative: 7e-7
    _, Ep = _relaxed(th, dict(kw, B=kw["B"] + d), lambda rp: F, 40000)
    _, Em = _relaxed(th, dict(kw, B=kw["B"] - d), lambda rp: F, 40000)
    fd = (Ep - Em) / (2 * d)
    assert abs(plain - fd) > 1e-4 * abs(fd)  # the discretisation gap this spacing shows uncorrected
    assert abs(g["B"] - fd) <= 1e-5 * abs(fd), (g["B"], plain, fd, info)
    assert info["minres_iterations"] < 20000


def test_forcing_is_added_to_the_flow_gradient():
    """ss_set_forcing: FP64 flow steps with a fixed field f added to the gradient rows equal
    the oracle's arrested-Newton steps with EG + f in every RK4 stage (Abelian Higgs: no
    projection, no halo zeroing, no row scaling), to 1e-12; removing it restores the flow."""
    th = load_theory("Abelian Higgs")
    rp = th.params.default_params(xlen=24, ylen=20, xsize=2.3, ysize=1.9, Lambda=0.7).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    rng = np.random.default_rng(8)
    F = 0.3 * rng.standard_normal((4, 24, 20))
    F[2] += 0.8
    f = 0.1 * rng.standard_normal(F.shape)
    dt = float(p_f[5])

    def forced_step(F, V, prev):
        def l(T):
            return -dt * (ref.gradient_step("ginzburg_landau_superconductor", T, p_i, p_f)[1] + f)
        k1, T = ref.rk4_stage(V, V, F, F, 0.0, p_f)
        l1 = l(T)
        k2, T = ref.rk4_stage(V, l1, F, k1, 0.5, p_f)
        l2 = l(T)
        k3, T = ref.rk4_stage(V, l2, F, k2, 0.5, p_f)
        l3 = l(T)
        k4, T = ref.rk4_stage(V, l3, F, k3, 1.0, p_f)
        l4 = l(T)
        Vn, Fn = ref.rk4_finalize("ginzburg_landau_superconductor", V, F, k1, k2, k3, k4, l1, l2, l3, l4, p_i)
        E = ref.energy("ginzburg_landau_superconductor", Fn, p_i, p_f)
        return Fn, (np.zeros_like(Vn) if E > prev else Vn), E

    s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
    fd = torch.tensor(F.reshape(-1), device="cuda")
    vd = torch.zeros_like(fd)
    s.bind(fd, vd)
    s.set_forcing(torch.tensor(f.reshape(-1), device="cuda"))
    E, _ = s.step(2, 1e300)
    Fo, Vo, prev = F, np.zeros_like(F), 1e300
    for k in range(2):
        Fo, Vo, prev = forced_step(Fo, Vo, prev)
        assert abs(E[k] - prev) <= 1e-12 * abs(prev)
    np.testing.assert_allclose(fd.cpu().numpy(), Fo.reshape(-1), rtol=0, atol=1e-12)
    s.set_forcing(None)
    E2, _ = s.step(1, float("nan"))
    Fu, _, Eu, _ = ref.relax("ginzburg_landau_superconductor", Fo, Vo, prev, p_i, p_f, 1)
    assert abs(E2[0] - Eu[0]) <= 1e-12 * abs(Eu[0])
