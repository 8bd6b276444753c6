"""The headline lattice at full size: chiral magnet 4096 x 4096, FP32 fields, Heusler DMI,
demag on, B = 0.2 T, 64 anti-skyrmions on a jittered lattice, arrested Newton flow.

  * whole lattice: one full FP32 step of the 16.8 M-site lattice against the FP64
    oracle's step of the same (FP32-rounded) field, computed over 16 stripes of 256
    rows with 12 rows of overlap on each cut side (a step's result at a row depends on
    the rows within 4 stages x 2 cells, and the cut's masks reach 2 more): every site
    of the new field to 1e-5 absolute (the FP32 trajectory tolerance of the parity
    tests), the stage-4 err to 1e-4 x its scale, and the step's flow energy against
    the oracle's FP64 energy of its new field: the projected FP64 energy of the stored result
    to 1e-7, the flow's FP32-jet energy to 5e-6 (its stored-pole bias, 2.1e-6 here).

Size-independent properties besides:

  * locality: the gradient at a site depends on its 5 x 5 neighbourhood only, so the
    full-lattice gradient on windows deep inside the lattice must equal the oracle's
    gradient of the window cut out with a margin (FP32 tolerance of the parity tests:
    norm-wise 1e-5, per entry 1e-4 x max);
  * chunking: 5 steps in one call equal 2 + 3 and 1 + 1 + 3 bitwise (the odd-count
    calls end in the caller's buffers);
  * the flow energy (FP32 jets, FP64 sum) equals the FP64 observable of the same field
    to 1e-6, and the sum of the FP64 energy density equals the reduced energy to 1e-12;
  * unit norm of the magnetisation after the steps to 1e-6, and the topological
    charge of 64 anti-skyrmions (|Q| within 0.05 of 64).
"""
import math

import numpy as np
import pytest
import torch

from oracle import flow64 as ref
from soliton_solver_b200.core.simulation import Simulation
from soliton_solver_b200.initial_conditions import skyrmion_lattice
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu

X = Y = 4096
XSIZE = 128.0
PHYS = dict(J=40e-12, K=0.8e6, D=4e-3, M=580e3, B=0.2, dmi_term="Heusler", demag=True, unit_magnetization=True,
            killkinen=True)


def _params(th, xlen, ylen, **kw):
    return th.params.default_params(xlen=xlen, ylen=ylen, **PHYS, **kw)


@pytest.fixture(scope="module")
def full():
    th = load_theory("Chiral magnet")
    p = _params(th, X, Y, xsize=XSIZE, ysize=XSIZE)
    sim = Simulation(p, th, precision="fp32")
    F0 = skyrmion_lattice(sim.rp, n=8, R=1.0, seed=1000, device=sim.device).to(torch.float32)
    return th, p, sim, F0


def _run(sim, F0, split):
    sim.load_field(F0)
    Es, prev = [], 1e300
    for k in split:
        E, _ = sim.relax(k, prev)
        prev = math.nan
        Es.extend(E)
    return np.array(Es), sim.Field.cpu().numpy(), sim.Velocity.cpu().numpy()


def test_fullsize_chunking_energy_norm_charge(full):
    th, p, sim, F0 = full
    outs = [_run(sim, F0, split) for split in ([5], [2, 3], [1, 1, 3])]
    for E, f, v in outs[1:]:
        np.testing.assert_array_equal(E, outs[0][0])
        np.testing.assert_array_equal(f, outs[0][1])
        np.testing.assert_array_equal(v, outs[0][2])
    E, f, _ = outs[0]
    assert np.isfinite(E).all()
    # the flow energy of the final field against the FP64 observable of the same field
    obs = sim.observables()
    assert abs(E[-1] - obs["energy"]) <= 1e-6 * abs(obs["energy"])
    # checksum: the FP64 energy density sums to the reduced energy
    dens = sim.solver.energy_density(sim.Field)
    assert abs(float(dens.sum()) - obs["energy"]) <= 1e-12 * abs(obs["energy"]) + 1e-9
    # unit norm after the re-projection of every step
    m = f.reshape(4, X, Y)[:3].astype(np.float64)
    assert float(np.max(np.abs(np.sqrt((m ** 2).sum(0)) - 1.0))) <= 1e-6
    # 64 anti-skyrmions
    assert abs(abs(obs["skyrmion_number"]) - 64.0) <= 0.05


@pytest.mark.parametrize("seed", [0, 1])
def test_fullsize_gradient_windows_vs_oracle(full, seed):
    th, p, sim, F0 = full
    sim.load_field(F0)
    sim.relax(3, 1e300)  # a field the flow has touched
    eg = sim.gradient().cpu().numpy().reshape(4, X, Y)
    F = sim.Field.cpu().numpy().astype(np.float64).reshape(4, X, Y)
    rp = sim.rp
    rng = np.random.default_rng(seed)
    w, mg = 48, 4
    for _ in range(3):
        x0 = int(rng.integers(8, X - w - 8))
        y0 = int(rng.integers(8, Y - w - 8))
        win = F[:, x0 - mg:x0 + w + mg, y0 - mg:y0 + w + mg]
        pw = _params(th, w + 2 * mg, w + 2 * mg, lsx=rp.lsx, lsy=rp.lsy, time_step=rp.time_step,
                     xsize=rp.lsx * (w + 2 * mg - 1), ysize=rp.lsy * (w + 2 * mg - 1))
        p_i, p_f = th.params.pack_device_params(pw.resolved())
        _, eg_w = ref.gradient_step("chiral_magnet", win, p_i, p_f)
        got = eg[:, x0:x0 + w, y0:y0 + w].reshape(-1)
        want = eg_w[:, mg:mg + w, mg:mg + w].reshape(-1)
        scale = float(np.max(np.abs(want)))
        nrm = float(np.linalg.norm(got - want) / np.linalg.norm(want))
        assert nrm <= 1e-5, f"window ({x0}, {y0}): norm-wise rel err {nrm:.3e}"
        assert float(np.max(np.abs(got - want))) <= 1e-4 * scale


def test_fullsize_gradient_corners_vs_oracle(full):
    """Windows at the four corners share the lattice's real edges with the oracle's
    window (derivative masks and the halo zeroing of the chiral magnet); only the
    window's inner sides are artificial and are excluded by the margin."""
    th, p, sim, F0 = full
    sim.load_field(F0)
    sim.relax(2, 1e300)
    eg = sim.gradient().cpu().numpy().reshape(4, X, Y)
    F = sim.Field.cpu().numpy().astype(np.float64).reshape(4, X, Y)
    rp = sim.rp
    w, mg = 40, 4
    n = w + mg
    pw = _params(th, n, n, lsx=rp.lsx, lsy=rp.lsy, time_step=rp.time_step, xsize=rp.lsx * (n - 1),
                 ysize=rp.lsy * (n - 1))
    p_i, p_f = th.params.pack_device_params(pw.resolved())
    for lo_x in (True, False):
        for lo_y in (True, False):
            xs = slice(0, n) if lo_x else slice(X - n, X)
            ys = slice(0, n) if lo_y else slice(Y - n, Y)
            _, eg_w = ref.gradient_step("chiral_magnet", F[:, xs, ys], p_i, p_f)
            cx = slice(0, w) if lo_x else slice(mg, n)  # the lattice edge side, away from the cut
            cy = slice(0, w) if lo_y else slice(mg, n)
            want = eg_w[:, cx, cy]
            gx = slice(0, w) if lo_x else slice(X - w, X)
            gy = slice(0, w) if lo_y else slice(Y - w, Y)
            got = eg[:, gx, gy]
            scale = float(np.max(np.abs(want)))
            assert scale > 0
            nrm = float(np.linalg.norm(got - want) / np.linalg.norm(want))
            assert nrm <= 1e-5, f"corner ({lo_x}, {lo_y}): norm-wise rel err {nrm:.3e}"
            assert float(np.max(np.abs(got - want))) <= 1e-4 * scale
            # the halo ring of the lattice edge is zeroed
            edge_x = got[:, :2, :] if lo_x else got[:, -2:, :]
            assert not np.any(edge_x)


def _oracle_step_window(args):
    """One oracle RK4 step of a window; returns the new field and the stage-4 gradient."""
    win, p_i, p_f = args
    V = np.zeros_like(win)
    k1, T = ref.rk4_stage(V, V, win, win, 0.0, p_f)
    l1, _ = ref.gradient_step("chiral_magnet", T, p_i, p_f)
    k2, T = ref.rk4_stage(V, l1, win, k1, 0.5, p_f)
    l2, _ = ref.gradient_step("chiral_magnet", T, p_i, p_f)
    k3, T = ref.rk4_stage(V, l2, win, k2, 0.5, p_f)
    l3, _ = ref.gradient_step("chiral_magnet", T, p_i, p_f)
    k4, T = ref.rk4_stage(V, l3, win, k3, 1.0, p_f)
    l4, EG = ref.gradient_step("chiral_magnet", T, p_i, p_f)
    _, Fn = ref.rk4_finalize("chiral_magnet", V, win, k1, k2, k3, k4, l1, l2, l3, l4, p_i)
    return Fn, EG


def test_fullsize_whole_lattice_step_vs_oracle(full):
    import concurrent.futures as cf
    th, p, sim, F0 = full
    sim.load_field(F0)
    E, err = sim.relax(1, 1e300)
    got = sim.Field.cpu().numpy().astype(np.float64).reshape(4, X, Y)
    Fin = F0.cpu().numpy().astype(np.float64).reshape(4, X, Y)
    rp = sim.rp
    S, H = 256, 12
    jobs, spans = [], []
    for x0 in range(0, X, S):
        x1 = x0 + S
        lo, hi = max(0, x0 - H), min(X, x1 + H)
        pw = _params(th, hi - lo, Y, lsx=rp.lsx, lsy=rp.lsy, time_step=rp.time_step, xsize=rp.lsx * (hi - lo - 1),
                     ysize=rp.lsy * (Y - 1))
        p_i, p_f = th.params.pack_device_params(pw.resolved())
        jobs.append((np.ascontiguousarray(Fin[:, lo:hi, :]), p_i, p_f))
        spans.append((x0, x1, lo))
    want = np.empty_like(Fin)
    err_want = -np.inf
    with cf.ThreadPoolExecutor(8) as ex:
        for (x0, x1, lo), (Fn, EG) in zip(spans, ex.map(_oracle_step_window, jobs)):
            want[:, x0:x1, :] = Fn[:, x0 - lo:x1 - lo, :]
            err_want = max(err_want, float(EG[:, x0 - lo:x1 - lo, :].max()))
    assert float(np.max(np.abs(got - want))) <= 1e-5
    assert abs(float(err[0]) - err_want) <= 1e-4 * max(abs(err_want), 1.0)
    p_i, p_f = th.params.pack_device_params(rp)
    E_want = ref.energy("chiral_magnet", want, p_i, p_f)
    # the FP64 energy of the stored FP32 result with its unit vectors renormalised in FP64
    assert abs(sim.projected_energy() - E_want) <= 1e-7 * abs(E_want)
    # the flow's own energy (FP32 jets) carries the stored-pole bias of the FP32 vacuum
    # (m3 rounds to 1 where |m_perp| < 2.4e-4): 2.1e-6 relative on this lattice
    assert abs(float(E[0]) - E_want) <= 5e-6 * abs(E_want)
