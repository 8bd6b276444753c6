"""Pin the FP64 oracle to golden vectors produced by the reference itself.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py``,
which runs the reference's own Numba kernels (under Numba's CUDA simulator) on
seeded random fields.  The oracle restates those kernels in the same operation
order, so agreement is expected to the last few ulps.
"""
import glob
import os

import numpy as np
import pytest

from oracle import flow64 as ref

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
HOOKS = sorted(glob.glob(os.path.join(GOLDEN, "hook_*.npz")))
TRAJS = sorted(glob.glob(os.path.join(GOLDEN, "traj_*.npz")))

# Relative to the largest magnitude of the compared array: the oracle follows the
# reference's association order, so the only differences are libm ulps.
RTOL = 1e-13


def _close(a, b, rtol=RTOL):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(1.0, float(np.max(np.abs(b)))) if b.size else 1.0
    err = float(np.max(np.abs(a - b))) if b.size else 0.0
    assert err <= rtol * scale, f"max abs err {err:.3e} > {rtol:.1e} * {scale:.3e}"


def test_fixtures_present():
    assert len(HOOKS) >= 20 and len(TRAJS) >= 5


@pytest.mark.parametrize("path", HOOKS, ids=[os.path.basename(p)[5:-4] for p in HOOKS])
def test_hooks(path):
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    F = ref.as_field(g["field"], p_i)
    V = ref.as_field(g["velocity"], p_i)
    l_out, EG = ref.gradient_step(th, F, p_i, p_f)
    _close(EG.reshape(-1), g["energy_gradient"])
    _close(l_out.reshape(-1), g["l_out"])
    _close(ref.energy_density(th, F, p_i, p_f).reshape(-1), g["energy_density"])
    E = ref.energy(th, F, p_i, p_f)
    assert abs(E - float(g["energy"])) <= 1e-13 * max(1.0, abs(float(g["energy"])))
    assert abs(E - float(g["obs_energy"])) <= 1e-13 * max(1.0, abs(float(g["energy"])))
    if "skyrmion_density" in g:
        d = ref.charge_density(th, F, p_i, p_f, "skyrmion")
        _close(d.reshape(-1), g["skyrmion_density"])
        assert abs(ref.reference_sum(d) - float(g["obs_skyrmion_number"])) <= 1e-13
    if "magnetic_charge_density" in g:
        d = ref.charge_density(th, F, p_i, p_f, "magnetic")
        _close(d.reshape(-1), g["magnetic_charge_density"])
        assert abs(ref.reference_sum(d) - float(g["obs_magnetic_charge"])) <= 1e-13
    if "vortex_density" in g:
        d = ref.charge_density(th, F, p_i, p_f, "vortex")
        _close(d.reshape(-1), g["vortex_density"])
        assert abs(ref.reference_sum(d) - float(g["obs_vortex_number"])) <= 1e-13
    ks = [ref.as_field(k, p_i) for k in g["rk4_k"]]
    ls = [ref.as_field(v, p_i) for v in g["rk4_l"]]
    k_out, temp = ref.rk4_stage(V, ls[0], F, ks[0], 0.5, p_f)
    _close(k_out.reshape(-1), g["rk4_stage_k_out"])
    _close(temp.reshape(-1), g["rk4_stage_temp"])
    Vn, Fn = ref.rk4_finalize(th, V, F, *ks, *ls, p_i)
    _close(Vn.reshape(-1), g["rk4_final_velocity"])
    _close(Fn.reshape(-1), g["rk4_final_field"])


@pytest.mark.parametrize("path", TRAJS, ids=[os.path.basename(p)[:-4] for p in TRAJS])
def test_trajectories(path):
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    F = ref.as_field(g["field"], p_i)
    V = ref.as_field(g["velocity"], p_i)
    F, V, E, err = ref.relax(th, F, V, float(g["prev_energy"]), p_i, p_f, int(g["n_steps"]))
    np.testing.assert_allclose(E, g["energy_traj"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(err, g["err_traj"], rtol=1e-12, atol=1e-14)
    _close(F.reshape(-1), g["final_field"], 1e-12)
    _close(V.reshape(-1), g["final_velocity"], 1e-12)


def _fd_vs_gradient(key, kw, comps):
    from soliton_solver_b200.theories import load_theory
    names = {"anisotropic_superconductor": "s+id superconductor", "ginzburg_landau_superconductor": "Abelian Higgs"}
    th = load_theory(names[key])
    rp = th.params.default_params(**kw).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    rng = np.random.default_rng(5)
    X, Y, nf = rp.xlen, rp.ylen, rp.number_total_fields
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    F = np.stack([0.3 * np.sin(2 * x + rng.normal()) * np.cos(1.5 * y + rng.normal()) for _ in range(nf)])
    bump = (np.sin(np.pi * (x + 1) / 2) * np.sin(np.pi * (y + 1) / 2)) ** 8
    g = ref.raw_gradient(key, F, p_i, p_f) * float(p_f[4])
    out = []
    for a in comps:
        D = np.zeros_like(F)
        D[a] = bump * np.cos(2 * x + y)
        eps = 1e-5
        fd = (ref.energy(key, F + eps * D, p_i, p_f) - ref.energy(key, F - eps * D, p_i, p_f)) / (2 * eps)
        out.append((float((g * D).sum()), fd))
    return out


def test_splusid_condensate_rows_are_not_dE_dpsi():
    """Pins a property of the reference: the s+id gradient rows of the condensates
    (anisotropic_superconductor/kernels.py:617-650) are not the derivative of its
    energy (kernels.py:97-170), while the gauge rows are (to O(h^4)).  The flow, the
    kernels and the autograd backward follow the reference's rows."""
    kw = dict(xlen=56, ylen=60, xsize=5.5, ysize=5.9)
    gauge = _fd_vs_gradient("anisotropic_superconductor", kw, (0, 1))
    for ad, fd in gauge:
        assert abs(ad - fd) <= 1e-3 * abs(fd)
    cond = _fd_vs_gradient("anisotropic_superconductor", kw, (2, 3, 4, 5))
    assert all(abs(ad - fd) > 0.1 * abs(fd) for ad, fd in cond)   # off by 25% to 80x
    assert any(abs(ad - fd) > 10 * abs(fd) for ad, fd in cond)
    # the Abelian Higgs rows are all consistent
    for ad, fd in _fd_vs_gradient("ginzburg_landau_superconductor", dict(xlen=64, ylen=68, xsize=6.3, ysize=6.7),
                                  (0, 1, 2, 3)):
        assert abs(ad - fd) <= 1e-3 * abs(fd)


DENSITIES = sorted(glob.glob(os.path.join(GOLDEN, "density_*.npz")))


@pytest.mark.parametrize("path", DENSITIES, ids=[os.path.basename(p)[8:-4] for p in DENSITIES])
def test_field_densities(path):
    """Higgs norms, phase difference, supercurrent and magnetic field of the gauge theories
    against the reference's Simulation helpers (compute_higgs*_density, supercurrent,
    magnetic_field, compute_phase_difference_density)."""
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    F = ref.as_field(g["field"], p_i)
    kinds = [k for k in ("higgs", "higgs1", "higgs2", "phase", "magnetic", "supercurrent") if k in g]
    assert "supercurrent" in kinds and len(kinds) >= 2
    for k in kinds:
        _close(ref.field_density(th, F, p_i, p_f, k).reshape(-1), g[k])


def test_relax_replay_with_the_oracles_own_decisions_is_relax():
    """relax_replay (the oracle with given arrest decisions, used to check FP32 runs whose
    decisions FP32 energies take) reproduces relax exactly when given relax's own
    decisions: V = 0 after step s iff E[s] > E[s-1] (the first step compares with the
    caller's previous energy, here +inf).  A run with arrests: Baby Skyrme from a field
    with a large random velocity."""
    from soliton_solver_b200.theories import load_theory

    th = load_theory("Baby Skyrme")
    rp = th.params.default_params(xlen=24, ylen=20, lsx=0.2, lsy=0.2, time_step=0.05,
                                  unit_magnetization=True, killkinen=True).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    rng = np.random.default_rng(3)
    F = rng.standard_normal((3, 24, 20))
    F /= np.sqrt((F ** 2).sum(0))
    V = 0.5 * rng.standard_normal(F.shape)
    Fo, Vo, E, err = ref.relax("baby_skyrme", F, V, np.inf, p_i, p_f, 12)
    arrests = np.concatenate([[False], np.diff(E) > 0])
    assert arrests.any() and not arrests.all()
    Fr, Vr, Er, errr = ref.relax_replay("baby_skyrme", F, V, arrests, p_i, p_f)
    np.testing.assert_array_equal(Fr, Fo)
    np.testing.assert_array_equal(Vr, Vo)
    np.testing.assert_array_equal(Er, E)
    np.testing.assert_array_equal(errr, err)
