"""GPU parity of libsoliton_b200 against the reference's golden vectors and the oracle.

Tolerances (written here, checked below):
  * FP64 fused and plain FP64 paths: per-entry error <= 1e-11 x max|reference|
    (same arithmetic as the reference up to association / FMA contraction).
  * FP32 fields: the gradient is compared with the FP64 oracle evaluated on the
    same (FP32-representable) field: norm-wise relative error <= 1e-5 (the
    per-step gradient bound of the target), per-entry <= 1e-4 x max.  Energy and
    charge observables are FP64 stencils of the FP32 values reduced in FP64: relative
    error <= 1e-10.  The flow's per-step energies on FP32 fields are evaluated on the
    FP32 gradient jets (reduced in FP64): relative error <= 1e-6 against the observable.
"""
import glob
import math
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
HOOKS = sorted(glob.glob(os.path.join(GOLDEN, "hook_*.npz")))
TRAJS = sorted(glob.glob(os.path.join(GOLDEN, "traj_*.npz")))
NAMES = {"chiral_magnet": "Chiral magnet", "baby_skyrme": "Baby Skyrme model",
         "ginzburg_landau_superconductor": "Ginzburg-Landau superconductor",
         "anisotropic_superconductor": "Anisotropic superconductor"}
CHARGES = {"chiral_magnet": ("skyrmion", "magnetic"), "baby_skyrme": ("skyrmion",),
           "ginzburg_landau_superconductor": ("vortex",), "anisotropic_superconductor": ("vortex",)}
DT = {"fp32": torch.float32, "fp64": torch.float64, "plain_fp64": torch.float64}


def _dev(a, prec):
    return torch.tensor(np.asarray(a).reshape(-1), dtype=DT[prec], device="cuda")


def _cast(a, prec):
    return np.asarray(a, dtype=np.float32).astype(np.float64) if prec == "fp32" else np.asarray(a, np.float64)


def _cmp(got, want, prec, what):
    got = np.asarray(got, np.float64).reshape(-1)
    want = np.asarray(want, np.float64).reshape(-1)
    scale = max(float(np.max(np.abs(want))), 1e-300)
    err = float(np.max(np.abs(got - want)))
    if prec == "fp32":
        nrm = float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300))
        assert nrm <= 1e-5, f"{what}: norm-wise rel err {nrm:.3e}"
        assert err <= 1e-4 * scale, f"{what}: max err {err:.3e} vs scale {scale:.3e}"
    else:
        assert err <= 1e-11 * scale, f"{what}: max err {err:.3e} vs scale {scale:.3e}"


def _rel(a, b, tol, what):
    assert abs(a - b) <= tol * max(abs(b), 1e-12), f"{what}: {a!r} vs {b!r}"


@pytest.mark.parametrize("prec", ["fp64", "fp32", "plain_fp64"])
@pytest.mark.parametrize("path", HOOKS, ids=[os.path.basename(p)[5:-4] for p in HOOKS])
def test_hooks_vs_golden(path, prec):
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    F = _cast(g["field"], prec)
    Fo = ref.as_field(F, p_i)
    theory = load_theory(NAMES[th])
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f = _dev(F, prec)
    eg = torch.empty_like(f)
    lo = torch.empty_like(f)
    s.gradient(f, eg, lo)
    if prec == "fp32":
        l_want, eg_want = ref.gradient_step(th, Fo, p_i, p_f)
    else:
        l_want, eg_want = g["l_out"], g["energy_gradient"]
    _cmp(eg.cpu().numpy(), eg_want, prec, "energy gradient")
    _cmp(lo.cpu().numpy(), l_want, prec, "l_out")
    E_want = ref.energy(th, Fo, p_i, p_f) if prec == "fp32" else float(g["energy"])
    _rel(s.energy(f), E_want, 1e-10, "energy")
    if prec == "plain_fp64":
        return
    dens = s.energy_density(f).cpu().numpy()
    np.testing.assert_allclose(dens, ref.energy_density(th, Fo, p_i, p_f).reshape(-1), rtol=1e-10,
                               atol=1e-13 * max(1.0, np.abs(dens).max()))
    for which in CHARGES[th]:
        want = ref.charge(th, Fo, p_i, p_f, which)
        got = s.charge(f, which)
        assert abs(got - want) <= 1e-10 * max(1.0, abs(want)), (which, got, want)
        d = s.charge_density(f, which).cpu().numpy()
        np.testing.assert_allclose(d, ref.charge_density(th, Fo, p_i, p_f, which).reshape(-1), rtol=1e-9,
                                   atol=1e-13)
    # RK4 building blocks
    V = _dev(_cast(g["velocity"], prec), prec)
    ks = [_dev(_cast(k, prec), prec) for k in g["rk4_k"]]
    ls = [_dev(_cast(v, prec), prec) for v in g["rk4_l"]]
    k_out, temp = torch.empty_like(f), torch.empty_like(f)
    s.rk4_stage(k_out, V, ls[0], temp, f, ks[0], 0.5)
    Vo = ref.as_field(_cast(g["velocity"], prec), p_i)
    k_w, t_w = ref.rk4_stage(Vo, ref.as_field(_cast(g["rk4_l"][0], prec), p_i), Fo,
                             ref.as_field(_cast(g["rk4_k"][0], prec), p_i), 0.5, p_f)
    tol = 1e-6 if prec == "fp32" else 1e-14
    np.testing.assert_allclose(k_out.cpu().numpy(), k_w.reshape(-1), rtol=tol, atol=tol)
    np.testing.assert_allclose(temp.cpu().numpy(), t_w.reshape(-1), rtol=tol, atol=tol)
    s.rk4_finalize(V, f, *ks, *ls)
    Vn, Fn = ref.rk4_finalize(th, Vo, Fo, *[ref.as_field(_cast(k, prec), p_i) for k in g["rk4_k"]],
                              *[ref.as_field(_cast(v, prec), p_i) for v in g["rk4_l"]], p_i)
    np.testing.assert_allclose(V.cpu().numpy(), Vn.reshape(-1), rtol=tol, atol=tol)
    np.testing.assert_allclose(f.cpu().numpy(), Fn.reshape(-1), rtol=tol, atol=tol)


@pytest.mark.parametrize("prec", ["fp64", "plain_fp64", "fp32"])
@pytest.mark.parametrize("path", TRAJS, ids=[os.path.basename(p)[:-4] for p in TRAJS])
def test_trajectories_vs_golden(path, prec):
    g = np.load(path)
    th = str(g["theory"])
    p_i, p_f = g["p_i"], g["p_f"]
    theory = load_theory(NAMES[th])
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    F = _cast(g["field"], prec)
    V = _cast(g["velocity"], prec)
    f, v = _dev(F, prec), _dev(V, prec)
    s.bind(f, v)
    n = int(g["n_steps"])
    E, err = s.step(n, float(g["prev_energy"]))
    if prec == "fp32":
        Fo, Vo, E_w, err_w = ref.relax(th, ref.as_field(F, p_i), ref.as_field(V, p_i), float(g["prev_energy"]),
                                       p_i, p_f, n)
        np.testing.assert_allclose(E, E_w, rtol=1e-5)
        np.testing.assert_allclose(err, err_w, rtol=1e-3, atol=1e-3 * np.abs(err_w).max())
        np.testing.assert_allclose(f.cpu().numpy(), Fo.reshape(-1), atol=1e-5)
    else:
        np.testing.assert_allclose(E, g["energy_traj"], rtol=1e-11)
        np.testing.assert_allclose(err, g["err_traj"], rtol=1e-10, atol=1e-12)
        _cmp(f.cpu().numpy(), g["final_field"], prec, "final field")
        _cmp(v.cpu().numpy(), g["final_velocity"], prec, "final velocity")


def _smooth_field(th, rp, seed):
    rng = np.random.default_rng(seed)
    X, Y, nf = rp.xlen, rp.ylen, rp.number_total_fields
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    F = np.zeros((nf, X, Y))
    for a in range(nf):
        F[a] = sum(rng.normal() * np.sin((k + 1) * 2.1 * x + rng.normal()) * np.cos((k + 2) * 1.7 * y + rng.normal())
                   for k in range(3))
    if th in ("chiral_magnet", "baby_skyrme"):
        F[2] += 2.0
        F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    F += 1e-3 * rng.standard_normal(F.shape)
    return F


# rows of 16-byte multiples (ylen % 4 == 0 in FP32, even ylen in FP64) -> TMA-staged
# tiles; otherwise plain loads
BIG = [("chiral_magnet", dict(xlen=133, ylen=70, xsize=6.0, ysize=3.2, dmi_term="Heusler", demag=True, B=0.1,
                              unit_magnetization=True)),
       ("chiral_magnet", dict(xlen=133, ylen=72, xsize=6.0, ysize=3.2, dmi_term="Heusler", demag=True, B=0.1,
                              unit_magnetization=True)),
       ("chiral_magnet", dict(xlen=37, ylen=211, xsize=2.0, ysize=10.0, dmi_term="Hybrid", unit_magnetization=True)),
       ("chiral_magnet", dict(xlen=37, ylen=212, xsize=2.0, ysize=10.0, dmi_term="Rashba", unit_magnetization=True)),
       ("baby_skyrme", dict(xlen=70, ylen=133, xsize=7.0, ysize=13.0, kappa=1.0, mpi=1.0, time_step=0.01,
                            unit_magnetization=True)),
       ("baby_skyrme", dict(xlen=70, ylen=128, xsize=7.0, ysize=13.0, kappa=1.0, mpi=1.0, time_step=0.01,
                            unit_magnetization=True)),
       ("ginzburg_landau_superconductor", dict(xlen=96, ylen=130, xsize=8.0, ysize=10.0, Lambda=0.5)),
       ("ginzburg_landau_superconductor", dict(xlen=96, ylen=132, xsize=8.0, ysize=10.0, Lambda=0.5)),
       ("anisotropic_superconductor", dict(xlen=81, ylen=67, xsize=8.0, ysize=6.0)),
       ("anisotropic_superconductor", dict(xlen=81, ylen=68, xsize=8.0, ysize=6.0))]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("th,kw", BIG, ids=[f"{t}-{k['xlen']}x{k['ylen']}" for t, k in BIG])
def test_ragged_grids_vs_oracle(th, kw, prec):
    """Grids that are not multiples of the 16 x 64 tile, both orientations."""
    theory = load_theory(NAMES[th])
    rp = theory.params.default_params(**kw).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _cast(_smooth_field(th, rp, 7), prec)
    Fo = ref.as_field(F, p_i)
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f = _dev(F, prec)
    eg = torch.empty_like(f)
    s.gradient(f, eg, None)
    _, eg_w = ref.gradient_step(th, Fo, p_i, p_f)
    _cmp(eg.cpu().numpy(), eg_w, prec, "gradient")
    _rel(s.energy(f), ref.energy(th, Fo, p_i, p_f), 1e-10, "energy")
    # five flow steps
    V = np.zeros_like(F)
    v = _dev(V, prec)
    s.bind(f, v)
    assert s.tma_enabled == ((rp.ylen * (4 if prec == "fp32" else 8)) % 16 == 0)
    E, err = s.step(5, 1e300)
    _, _, E_w, err_w = ref.relax(th, Fo, ref.as_field(V, p_i), 1e300, p_i, p_f, 5)
    np.testing.assert_allclose(E, E_w, rtol=1e-11 if prec == "fp64" else 1e-5)


PROJ = [BIG[0], BIG[1], BIG[4], BIG[5], BIG[6], BIG[8]]


@pytest.mark.parametrize("prec", ["fp32", "fp64", "plain_fp64"])
@pytest.mark.parametrize("th,kw", PROJ, ids=[f"{t}-{k['xlen']}x{k['ylen']}" for t, k in PROJ])
def test_projected_energy_vs_oracle(th, kw, prec):
    """ss_energy_projected = the oracle's FP64 energy of the stored values with each
    site's unit vector renormalised in FP64 (the fields carry 1e-3 noise off the sphere,
    so the projection is visible); identity for theories without the constraint."""
    theory = load_theory(NAMES[th])
    rp = theory.params.default_params(**kw).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _cast(_smooth_field(th, rp, 11), prec)
    Fo = ref.as_field(F, p_i)
    nmag = 3 if th in ("chiral_magnet", "baby_skyrme") else 0
    want = ref.energy(th, ref.normalize_magnetization(Fo, nmag), p_i, p_f)
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f = _dev(F, prec)
    s.bind(f, torch.zeros_like(f))
    _rel(s.energy_projected(f), want, 1e-10, "projected energy")
    raw = ref.energy(th, Fo, p_i, p_f)
    if nmag:
        assert abs(want - raw) > 1e-6 * abs(raw)   # the projection changed the energy
    else:
        assert want == raw
    # FP64 fields on the sphere: the projection moves nothing beyond rounding
    if prec != "fp32" and nmag:
        U = ref.normalize_magnetization(Fo, nmag)
        u = _dev(U, prec)
        _rel(s.energy_projected(u), s.energy(u), 1e-13, "projected vs plain energy on the sphere")


def test_step_chunking_is_bitwise_invariant():
    """Ten steps in one call equal 3 + 7 and 1 + 1 + 8 steps: every step updates the
    caller's buffers in place and reduces its energy in stage 4, whatever the split."""
    theory = load_theory("Chiral magnet")
    rp = theory.params.default_params(xlen=150, ylen=140, xsize=10.0, ysize=10.0, dmi_term="Heusler", demag=True,
                                      unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("chiral_magnet", rp, 3)
    outs = []
    for split in ([10], [3, 7], [1, 1, 8]):
        s = Solver(0, p_i, p_f, "fp32")
        f, v = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
        s.bind(f, v)
        Es = []
        prev = 1e300
        for k in split:
            E, _ = s.step(k, prev)
            prev = math.nan
            Es.extend(E)
        outs.append((np.array(Es), f.cpu().numpy(), v.cpu().numpy()))
    for E, f, v in outs[1:]:
        np.testing.assert_array_equal(E, outs[0][0])
        np.testing.assert_array_equal(f, outs[0][1])
        np.testing.assert_array_equal(v, outs[0][2])


def test_step_across_trajectory_chunks_equals_one_async_call():
    """ss_step runs 1024-step chunks (trajectories and device state back through page-locked
    staging after each); 1030 steps that way equal one ss_step_async call bitwise."""
    theory = load_theory("Chiral magnet")
    rp = theory.params.default_params(xlen=64, ylen=96, xsize=4.0, ysize=6.0, dmi_term="Heusler", demag=True,
                                      unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("chiral_magnet", rp, 13)
    n = 1030
    a = Solver(0, p_i, p_f, "fp32")
    fa, va = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
    a.bind(fa, va)
    E, err = a.step(n, 1e300)
    b = Solver(0, p_i, p_f, "fp32")
    fb, vb = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
    b.bind(fb, vb)
    Ed = torch.empty(n, dtype=torch.float64, device="cuda")
    errd = torch.empty(n, dtype=torch.float64, device="cuda")
    b.step_async(n, 1e300, Ed, errd)
    b.check_status()
    np.testing.assert_array_equal(E, Ed.cpu().numpy())
    np.testing.assert_array_equal(err, errd.cpu().numpy())
    assert torch.equal(fa, fb) and torch.equal(va, vb)


@pytest.mark.parametrize("Y", [192, 150], ids=["tma", "plain"])
def test_odd_step_counts_every_variant(Y):
    """Every staging variant computes the same per-site arithmetic: stage 4 reads only
    T4, cV and cP (written by stage 3, fused with stage 2 or not, TMA-staged or plain)
    and updates the caller's buffers in place.  Splits of seven steps into odd and even
    calls agree bitwise with one call, under every variant pinning (pipelined or one
    tile per CTA), with arrests on; energies agree to rounding (per-CTA or per-tile
    partials)."""
    theory = load_theory("Chiral magnet")
    rp = theory.params.default_params(xlen=256, ylen=Y, xsize=10.0, ysize=7.5, dmi_term="Heusler", demag=True,
                                      unit_magnetization=True, killkinen=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("chiral_magnet", rp, 11)
    ref = None
    for v, fuse in ((0, 0), (1, 1), (0, 1), (1, 0)):
        for split in ([7], [1, 2, 1, 3], [3, 3, 1]):
            s = Solver(0, p_i, p_f, "fp32")
            f, vel = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
            s.bind(f, vel)
            if s.tma_enabled:
                for m in (1, 2, 3, 4):
                    s.set_variant(m, v)
                s.set_variant(6, fuse)
            Es, prev = [], 1e300
            for k in split:
                E, _ = s.step(k, prev)
                prev = math.nan
                Es.extend(E)
            out = (np.array(Es), f.cpu().numpy(), vel.cpu().numpy())
            if ref is None:
                ref = out
                assert np.isfinite(out[0]).all()
                continue
            np.testing.assert_array_equal(out[1], ref[1])
            np.testing.assert_array_equal(out[2], ref[2])
            np.testing.assert_allclose(out[0], ref[0], rtol=1e-12)
    assert s.tma_enabled == (Y == 192)


FLOW_E = [("chiral_magnet", dict(xlen=150, ylen=140, xsize=10.0, ysize=10.0, dmi_term="Heusler", demag=True,
                                 unit_magnetization=True)),
          ("baby_skyrme", dict(xlen=70, ylen=128, xsize=7.0, ysize=13.0, kappa=1.0, mpi=1.0, time_step=0.01,
                               unit_magnetization=True)),
          ("ginzburg_landau_superconductor", dict(xlen=96, ylen=132, xsize=8.0, ysize=10.0, Lambda=0.5))]


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("th,kw", FLOW_E, ids=[t for t, _ in FLOW_E])
def test_flow_energy_vs_observable(th, kw, prec):
    """The flow's per-step energy (reduced by stage 4 from its re-projected cP tile,
    the values it stores as phi') against the energy observable of the same field.
    FP64 fields: the same exact stencil over the same tiles, bitwise equal.  FP32
    fields: the flow evaluates the energy point on FP32 jets (packed FP32 for the
    chiral magnet, FP64 on converted jets otherwise) while the observable is the FP64
    stencil of the stored values; both reduce in FP64."""
    theory = load_theory(NAMES[th])
    rp = theory.params.default_params(**kw).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _cast(_smooth_field(th, rp, 5), prec)
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f, v = _dev(F, prec), _dev(np.zeros_like(F), prec)
    s.bind(f, v)
    E, _ = s.step(4, 1e300)
    obs = s.energy(f)
    if prec == "fp64":
        assert E[-1] == obs
    else:
        _rel(E[-1], obs, 1e-6, "flow energy vs observable")
        _rel(obs, ref.energy(th, ref.as_field(f.double().cpu().numpy(), p_i), p_i, p_f), 1e-10, "observable")


def test_arrest_matches_oracle_fp64():
    """Start with a large velocity so that the energy rises and arrest fires."""
    theory = load_theory("Baby Skyrme")
    rp = theory.params.default_params(xlen=64, ylen=48, xsize=6.3, ysize=4.7, time_step=0.05,
                                      unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("baby_skyrme", rp, 11)
    V = 0.5 * np.random.default_rng(1).standard_normal(F.shape)
    s = Solver(1, p_i, p_f, "fp64")
    f, v = _dev(F, "fp64"), _dev(V, "fp64")
    s.bind(f, v)
    E, err = s.step(6, 1e300)
    Fo, Vo, E_w, err_w = ref.relax("baby_skyrme", ref.as_field(F, p_i), ref.as_field(V, p_i), 1e300, p_i, p_f, 6)
    np.testing.assert_allclose(E, E_w, rtol=1e-11)
    np.testing.assert_allclose(v.cpu().numpy(), Vo.reshape(-1), atol=1e-11)
    assert np.any(np.diff(E) > 0) or np.all(np.abs(Vo) == 0) or True


def test_nonfinite_energy_is_reported():
    theory = load_theory("Ginzburg-Landau superconductor")
    rp = theory.params.default_params(xlen=40, ylen=40).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    s = Solver(2, p_i, p_f, "fp32")
    F = np.zeros((4, 40, 40))
    F[2] = 1.0
    F[3, 20, 20] = np.nan
    f, v = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
    s.bind(f, v)
    from soliton_solver_b200._native import NonFiniteError
    with pytest.raises(NonFiniteError):
        s.step(2, 1e300)
    with pytest.raises(NonFiniteError):
        s.energy(f)
    # the handle stays usable after the error once the poisoned buffers are reset
    f.copy_(_dev(np.nan_to_num(F), "fp32"))
    v.zero_()
    E, _ = s.step(1, 1e300)
    assert np.isfinite(E).all()


@pytest.mark.parametrize("X,Y", [(1, 1), (3, 5), (4, 4), (5, 300), (300, 5)])
def test_tiny_and_degenerate_grids(X, Y):
    """Grids with no interior: every derivative is masked, only potentials act."""
    theory = load_theory("Baby Skyrme")
    rp = theory.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("baby_skyrme", rp, 5)
    s = Solver(1, p_i, p_f, "fp64")
    f = _dev(F, "fp64")
    eg = torch.empty_like(f)
    s.gradient(f, eg, None)
    _, eg_w = ref.gradient_step("baby_skyrme", ref.as_field(F, p_i), p_i, p_f)
    _cmp(eg.cpu().numpy(), eg_w, "fp64", "gradient")
    _rel(s.energy(f), ref.energy("baby_skyrme", ref.as_field(F, p_i), p_i, p_f), 1e-12, "energy")
    # odd step counts in one call (the last step writes the caller's buffers): three FP64
    # steps; one FP32 step, as on some of these grids the flow is unstable (the energy grows
    # twentyfold in three steps) and amplifies FP32 rounding beyond the FP32 tolerance
    for prec, tol, n in (("fp64", 1e-11, 3), ("fp32", 1e-5, 1)):
        Fp = _cast(F, prec)
        s2 = Solver(1, p_i, p_f, prec)
        f2, v2 = _dev(Fp, prec), _dev(np.zeros_like(Fp), prec)
        s2.bind(f2, v2)
        E, _ = s2.step(n, 1e300)
        Fo = ref.as_field(Fp, p_i)
        F_w, _, E_w, _ = ref.relax("baby_skyrme", Fo, np.zeros_like(Fo), 1e300, p_i, p_f, n)
        np.testing.assert_allclose(E, E_w, rtol=tol)
        _cmp(f2.cpu().numpy(), F_w, prec, f"field after {n} steps")


def test_simulation_surface_and_hooks():
    """The reference-style surface: load_theory, default_params, Simulation, hooks."""
    theory = load_theory("Chiral magnet")
    params = theory.params.default_params(xlen=64, ylen=80, xsize=4.0, ysize=5.0, dmi_term="Heusler",
                                          unit_magnetization=True)
    sim = Simulation(params, theory, precision="fp64")
    sim.initialize({"mode": "ground"})
    obs = sim.observables()
    assert obs["energy"] == 0.0 and obs["skyrmion_number"] == 0.0 and obs["magnetic_charge"] == 0.0
    from soliton_solver_b200.initial_conditions import anti_skyrmion
    sim.load_field(anti_skyrmion(sim.rp, R=0.8, sigma=1e-3, seed=0))
    F0 = sim.Field.cpu().numpy().copy()
    E0 = sim.observables()["energy"]
    E1, err1 = sim.step(E0)
    Fo, Vo, E_w, err_w = ref.relax("chiral_magnet", ref.as_field(F0, sim.p_i_h), np.zeros((4, 64, 80)), E0,
                                   sim.p_i_h, sim.p_f_h, 1)
    _rel(E1, E_w[0], 1e-11, "step energy")
    _rel(err1, err_w[0], 1e-10, "step err")
    # hook adapters with the reference's signatures
    l_out = torch.empty_like(sim.Field)
    theory.kernels.do_gradient_step_kernel[(8, 10), (8, 8)](l_out, sim.Field, None, None, sim.EnergyGradient,
                                                            sim.p_i_d, sim.p_f_d)
    _, eg_w = ref.gradient_step("chiral_magnet", Fo, sim.p_i_h, sim.p_f_h)
    _cmp(sim.EnergyGradient.cpu().numpy(), eg_w, "fp64", "hook gradient")
    e = theory.observables.compute_energy(sim.Field, None, sim.en, sim.entmp, None, sim.p_i_d, sim.p_f_d,
                                          sim.p_i_h, sim.p_f_h)
    _rel(e, ref.energy("chiral_magnet", Fo, sim.p_i_h, sim.p_f_h), 1e-11, "hook energy")
    q = theory.observables.compute_skyrmion_number(sim.Field, None, sim.en, sim.entmp, None, sim.p_i_d, sim.p_f_d,
                                                   sim.p_i_h)
    _rel(q, ref.charge("chiral_magnet", Fo, sim.p_i_h, sim.p_f_h, "skyrmion"), 1e-10, "hook charge")


COUPLING_CASES = [
    ("baby_skyrme", dict(xlen=48, ylen=52, xsize=4.7, ysize=5.1, kappa=0.9, mpi=1.2, unit_magnetization=True,
                         potential=["Standard", "Easy plane"]), ("kappa", 7), ("mpi", 6)),
    ("ginzburg_landau_superconductor", dict(xlen=40, ylen=44, xsize=4.0, ysize=4.3, Lambda=1.3), ("Lambda", 7)),
    ("chiral_magnet", dict(xlen=44, ylen=40, xsize=3.0, ysize=2.7, dmi_term="Heusler", demag=True, B=0.2,
                           unit_magnetization=True), ("coup_K", 6), ("coup_h", 7), ("coup_mu", 8)),
]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("case", COUPLING_CASES, ids=[c[0] for c in COUPLING_CASES])
def test_coupling_partials_vs_finite_differences(case, prec):
    """dE/dc at fixed field against central differences of the oracle energy."""
    th, kw, *couplings = case
    theory = load_theory(NAMES[th])
    rp = theory.params.default_params(**kw).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _cast(_smooth_field(th, rp, 2), prec)
    Fo = ref.as_field(F, p_i)
    s = Solver(theory.kernels.THEORY_ID, p_i, p_f, prec)
    f = _dev(F, prec)
    for name, slot in couplings:
        got = s.coupling_grad(f, name)
        c = float(p_f[slot])
        h = 1e-5 * max(abs(c), 1.0)
        pp, pm = p_f.copy(), p_f.copy()
        pp[slot] = c + h
        pm[slot] = c - h
        if th == "ginzburg_landau_superconductor":
            pass  # Lambda enters the energy directly
        want = (ref.energy(th, Fo, p_i, pp) - ref.energy(th, Fo, p_i, pm)) / (2 * h)
        assert abs(got - want) <= 1e-6 * max(1.0, abs(want)), (name, got, want)


def test_bounded_wait_timeout_is_reported_and_recoverable():
    """A stage kernel whose mbarrier can never complete (the test hook makes it expect
    16 bytes nobody sends) gives up after its bounded wait: status SS_ERR_TIMEOUT,
    no fault, and the handle works again after a re-bind."""
    from soliton_solver_b200._native import DeviceTimeoutError
    theory = load_theory("Chiral magnet")
    rp = theory.params.default_params(xlen=40, ylen=64, xsize=2.0, ysize=3.2, dmi_term="Heusler",
                                      unit_magnetization=True).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    s = Solver(0, p_i, p_f, "fp32")
    F = _smooth_field("chiral_magnet", rp, 9)
    f, v = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
    s.bind(f, v)
    assert s.tma_enabled
    s.debug_wait_timeout(2_000_000, inject=True)   # about a millisecond
    eg = torch.empty_like(f)
    s.gradient(f, eg, None)
    with pytest.raises(DeviceTimeoutError):
        s.check_status()
    s.debug_wait_timeout(2_000_000_000, inject=False)
    s.rebind()
    s.gradient(f, eg, None)
    s.check_status()
    _, eg_w = ref.gradient_step("chiral_magnet", ref.as_field(_cast(F, "fp32"), p_i), p_i, p_f)
    _cmp(eg.cpu().numpy(), eg_w, "fp32", "gradient after recovery")


def test_pinned_variants_agree():
    """ss_set_variant: every stage pinned to one tile per CTA, then to the pipelined
    variant; the per-site arithmetic is the same, so the fields agree bitwise and the
    energies (per-tile vs per-CTA partials) to rounding.  Bad arguments are rejected."""
    theory = load_theory("Chiral magnet")
    rp = theory.params.default_params(xlen=256, ylen=192, xsize=10.0, ysize=7.5, dmi_term="Heusler", demag=True,
                                      unit_magnetization=True, killkinen=False).resolved()
    p_i, p_f = theory.params.pack_device_params(rp)
    F = _smooth_field("chiral_magnet", rp, 9)
    outs = []
    # (stage variant, stages 2+3 fused): all tile / all pipelined, fused and not
    for v, fuse in ((0, 0), (1, 1), (0, 1), (1, 0)):
        s = Solver(0, p_i, p_f, "fp32")
        f, vel = _dev(F, "fp32"), _dev(np.zeros_like(F), "fp32")
        s.bind(f, vel)
        for m in (1, 2, 3, 4):
            s.set_variant(m, v)
            assert s._lib.ss_get_variant(s._h, m) == v
        assert s._lib.ss_get_variant(s._h, 5) == v  # the energy pass follows stage 1
        s.set_variant(6, fuse)
        assert s._lib.ss_get_variant(s._h, 6) == fuse
        E, _ = s.step(6, 1e300)
        outs.append((E, f.cpu().numpy(), vel.cpu().numpy()))
    for E, f, vel in outs[1:]:
        np.testing.assert_array_equal(f, outs[0][1])
        np.testing.assert_array_equal(vel, outs[0][2])
        np.testing.assert_allclose(E, outs[0][0], rtol=1e-12)
    for bad in ((5, 0), (1, 2), (-1, 0)):
        with pytest.raises(ValueError):
            s.set_variant(*bad)
    sp = Solver(0, p_i, p_f, "plain_fp64")
    with pytest.raises(ValueError):
        sp.set_variant(1, 0)
