"""Batched lattices (ss_batch_*) against single-lattice solvers.

Each lattice in a batch must follow exactly the trajectory a single-lattice Solver
gives it: FP64 energies and fields to 1e-13 relative, FP32 energies to 1e-10.
Lattices differ in size (TMA-aligned and not), couplings, seeds and arrest history.
"""
import numpy as np
import pytest
import torch

from oracle import flow64 as ref
from soliton_solver_b200.core.batch import BatchSolver
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu


def _hedgehog(rp, B, R, seed):
    rng = np.random.default_rng(seed)
    X, Y = rp.xlen, rp.ylen
    x = (np.arange(X) - (X - 1) / 2)[:, None] * rp.lsx
    y = (np.arange(Y) - (Y - 1) / 2)[None, :] * rp.lsy
    r, t = np.hypot(x, y), np.arctan2(y, x)
    f = np.pi * np.exp(-r / R)
    m = np.stack([np.sin(f) * np.cos(B * t), np.sin(f) * np.sin(B * t), np.cos(f)])
    m += 1e-3 * rng.standard_normal(m.shape)
    return m / np.sqrt((m ** 2).sum(0))


SIZES = [(64, 64), (72, 96), (128, 128), (40, 200), (96, 64), (33, 70), (50, 91), (61, 45)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("aligned", [True, False])
def test_batch_matches_single_lattices(precision, aligned):
    th = load_theory("Baby Skyrme")
    sizes = [s for s in SIZES if (s[1] % 4 == 0) == aligned] or SIZES[:1]
    rng = np.random.default_rng(7)
    params = [th.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for X, Y in sizes]
    b = BatchSolver(th, params, precision)
    assert b.tma_enabled == all(Y * (4 if precision == "fp32" else 8) % 16 == 0 for _, Y in sizes)
    fields = [_hedgehog(p.resolved(), B=i % 4 + 1, R=float(rng.uniform(1, 3)), seed=i) for i, p in enumerate(params)]
    for i, F in enumerate(fields):
        b.load(i, F)
    prev = np.full(len(sizes), 1e300)
    prev[1] = -1e300  # arrest fires for this lattice
    E, err = b.step(6, prev)
    dt = torch.float32 if precision == "fp32" else torch.float64
    for i, p in enumerate(params):
        rp = p.resolved()
        p_i, p_f = th.params.pack_device_params(rp)
        s = Solver(th.kernels.THEORY_ID, p_i, p_f, precision)
        f = torch.tensor(fields[i].reshape(-1), dtype=dt, device="cuda")
        v = torch.zeros_like(f)
        s.bind(f, v)
        Ei, erri = s.step(6, float(prev[i]))
        tol = 1e-13 if precision == "fp64" else 1e-10
        np.testing.assert_allclose(E[i], Ei, rtol=tol)
        np.testing.assert_allclose(err[i], erri, rtol=1e-6 if precision == "fp32" else 1e-12)
        np.testing.assert_allclose(b.fields[i].cpu().numpy(), f.cpu().numpy(), rtol=0,
                                   atol=1e-12 if precision == "fp64" else 1e-6)
    # a second call continues from the device state of every lattice
    E2, _ = b.step(3)
    assert np.all(np.isfinite(E2))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("aligned", [True, False], ids=["tma", "plain"])
def test_batch_odd_step_counts_are_bitwise_invariant(aligned, precision):
    """Batched steps update every lattice's buffers in place (stage 4 reads only T4, cV
    and cP): seven steps split into odd and even calls equal one call bitwise, arrests
    included."""
    th = load_theory("Baby Skyrme")
    sizes = [s for s in SIZES if (s[1] % 4 == 0) == aligned]
    rng = np.random.default_rng(11)
    params = [th.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for X, Y in sizes]
    fields = [_hedgehog(p.resolved(), B=i % 4 + 1, R=float(rng.uniform(1, 3)), seed=i) for i, p in enumerate(params)]
    prev = np.full(len(sizes), 1e300)
    prev[0] = -1e300  # arrest fires for this lattice
    outs = []
    for split in ([7], [1, 2, 1, 3], [3, 3, 1]):
        b = BatchSolver(th, params, precision)
        es = 4 if precision == "fp32" else 8
        assert b.tma_enabled == all(Y * es % 16 == 0 for _, Y in sizes)
        for i, F in enumerate(fields):
            b.load(i, F)
        Es = []
        for j, k in enumerate(split):
            E, _ = b.step(k, prev if j == 0 else None)
            Es.append(E)
        outs.append((np.concatenate(Es, axis=1), [f.cpu().numpy() for f in b.fields],
                     [v.cpu().numpy() for v in b.velocities]))
    for E, fs, vs in outs[1:]:
        np.testing.assert_array_equal(E, outs[0][0])
        for a, c in zip(fs, outs[0][1]):
            np.testing.assert_array_equal(a, c)
        for a, c in zip(vs, outs[0][2]):
            np.testing.assert_array_equal(a, c)


def test_batch_trajectories_across_chunks():
    """A call longer than the 1024-step trajectory chunk: every lattice's energy and err
    rows (returned per chunk in one 2-D copy for all lattices) equal a single-lattice
    solver's, and the fields end equal."""
    th = load_theory("Baby Skyrme")
    sizes = [(24, 32), (40, 36), (33, 20)]
    rng = np.random.default_rng(3)
    params = [th.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for X, Y in sizes]
    fields = [_hedgehog(p.resolved(), B=1 + i, R=1.5, seed=i) for i, p in enumerate(params)]
    b = BatchSolver(th, params, "fp64")
    for i, F in enumerate(fields):
        b.load(i, F)
    n = 1030
    E, err = b.step(n, np.full(len(sizes), 1e300))
    assert E.shape == (len(sizes), n) and np.isfinite(E).all()
    for i, p in enumerate(params):
        p_i, p_f = th.params.pack_device_params(p.resolved())
        s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp64")
        f = torch.tensor(fields[i].reshape(-1), dtype=torch.float64, device="cuda")
        v = torch.zeros_like(f)
        s.bind(f, v)
        Ei, erri = s.step(n, 1e300)
        np.testing.assert_allclose(E[i], Ei, rtol=1e-12)
        np.testing.assert_allclose(err[i], erri, rtol=1e-10, atol=1e-300)
        np.testing.assert_allclose(b.fields[i].cpu().numpy(), f.cpu().numpy(), rtol=0, atol=1e-11)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_trajectories_vs_oracle(precision):
    """Each lattice of a batch against the FP64 oracle's own arrested-Newton steps from the
    same field (not through the single-lattice solver): FP64 energies 1e-12 relative and
    fields 1e-12; FP32 (oracle on the FP32-rounded field) energies 1e-6, fields 1e-5."""
    th = load_theory("Baby Skyrme")
    sizes = [(64, 64), (40, 200), (33, 70)]
    rng = np.random.default_rng(21)
    params = [th.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for X, Y in sizes]
    fields = [_hedgehog(p.resolved(), B=i + 1, R=float(rng.uniform(1, 3)), seed=i) for i, p in enumerate(params)]
    if precision == "fp32":
        fields = [F.astype(np.float32).astype(np.float64) for F in fields]
    b = BatchSolver(th, params, precision)
    for i, F in enumerate(fields):
        b.load(i, F)
    prev = np.full(len(sizes), 1e300)
    prev[2] = -1e300  # arrest fires for this lattice
    n = 5
    E, err = b.step(n, prev)
    tol_E, tol_F = (1e-12, 1e-12) if precision == "fp64" else (1e-6, 1e-5)
    for i, p in enumerate(params):
        p_i, p_f = th.params.pack_device_params(p.resolved())
        Fo, _, Ew, errw = ref.relax("baby_skyrme", fields[i], np.zeros_like(fields[i]), float(prev[i]), p_i, p_f, n)
        np.testing.assert_allclose(E[i], Ew, rtol=tol_E)
        assert float(np.max(np.abs(b.fields[i].double().cpu().numpy() - Fo.reshape(-1)))) <= tol_F
        np.testing.assert_allclose(err[i], errw, rtol=1e-4 if precision == "fp32" else 1e-10)


def test_batch_sweep_config_shape():
    """256 lattices with sizes from {64, 128, 256, 512}^2, random couplings and charges
    (the batched baby Skyrme sweep), FP32: runs and keeps every energy finite, and three
    sampled lattices (one of each of the three smaller sizes) follow the FP64 oracle's
    steps from the same FP32 field (energies 1e-6 relative)."""
    th = load_theory("Baby Skyrme")
    rng = np.random.default_rng(4)
    edges = rng.choice([64, 128, 256, 512], size=256)
    params = [th.params.default_params(xlen=int(e), ylen=int(e), lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for e in edges]
    b = BatchSolver(th, params, "fp32")
    assert b.tma_enabled
    for i, p in enumerate(params):
        b.load(i, _hedgehog(p.resolved(), B=1, R=1.5, seed=i))
    F0 = [f.double().cpu().numpy() for f in b.fields]
    E, err = b.step(20, 1e300)
    assert np.all(np.isfinite(E)) and E.shape == (256, 20)
    for e in (64, 128, 256):
        i = int(np.nonzero(edges == e)[0][0])
        p_i, p_f = th.params.pack_device_params(params[i].resolved())
        _, _, Ew, _ = ref.relax("baby_skyrme", ref.as_field(F0[i], p_i), np.zeros((3, e, e)), 1e300, p_i, p_f, 3)
        np.testing.assert_allclose(E[i, :3], Ew, rtol=1e-6)


def test_graph_replay_equals_stream_steps():
    """A captured n-step graph, replayed twice, gives the same fields and energies as
    2 x n steps issued on the stream (single lattice and batch)."""
    th = load_theory("Chiral magnet")
    p = th.params.default_params(xlen=160, ylen=128, xsize=5.0, ysize=4.0, dmi_term="Heusler", demag=True,
                                 unit_magnetization=True)
    rp = p.resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    from soliton_solver_b200.initial_conditions import anti_skyrmion
    F = anti_skyrmion(rp, R=0.8, seed=1).numpy()
    outs = []
    for use_graph in (False, True):
        s = Solver(th.kernels.THEORY_ID, p_i, p_f, "fp32")
        f = torch.tensor(F, dtype=torch.float32, device="cuda")
        v = torch.zeros_like(f)
        s.bind(f, v)
        s.step(1, 1e300)  # seeds the device-side energy
        if use_graph:
            E = torch.empty(7, dtype=torch.float64, device="cuda")
            s.capture(7, E, None)
            s.replay()
            s.replay()
            torch.cuda.synchronize()
            last = E.cpu().numpy()
        else:
            s.step(7)
            Es, _ = s.step(7)
            last = Es
        outs.append((f.cpu().numpy(), last))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])

    bth = load_theory("Baby Skyrme")
    params = [bth.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02, unit_magnetization=True)
              for X, Y in ((64, 64), (96, 128))]
    res = []
    for use_graph in (False, True):
        b = BatchSolver(bth, params, "fp32")
        for i, q in enumerate(params):
            b.load(i, _hedgehog(q.resolved(), B=1, R=1.5, seed=i))
        b.step(1, 1e300)
        if use_graph:
            b.capture(5)
            b.replay()
            b.replay()
            E, _ = b.trajectory()
        else:
            b.step(5)
            E, _ = b.step(5)
        res.append(([t.cpu().numpy() for t in b.fields], E))
    for a, c in zip(res[0][0], res[1][0]):
        np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_batch_tile_shapes_autotune_and_agree():
    """The autotuner times every size class in both tile shapes (16 x 64 and 8 x 32 sites)
    and keeps one per class; whatever the shapes, every lattice's fields after five steps are
    bitwise those of the 16 x 64 run (the per-site arithmetic does not depend on the tile),
    and the energies agree to rounding (the per-tile partials are summed in another order)."""
    th = load_theory("Baby Skyrme")
    sizes = [(64, 64), (64, 64), (128, 96), (96, 128), (128, 96)]
    rng = np.random.default_rng(9)
    params = [th.params.default_params(xlen=X, ylen=Y, lsx=0.1, lsy=0.1, time_step=0.02,
                                       kappa=float(rng.uniform(0.5, 2)), mpi=float(rng.uniform(0.5, 2)),
                                       unit_magnetization=True) for X, Y in sizes]
    fields = [_hedgehog(p.resolved(), B=i % 3 + 1, R=1.5, seed=i) for i, p in enumerate(params)]
    runs = []
    for mode in ("shape0", "shape1", "tuned"):
        b = BatchSolver(th, params, "fp32")
        assert b.tma_enabled
        if mode == "shape1":
            for i in range(len(sizes)):
                b.set_shape(i, 1)
            assert all(b.shape(i) == 1 for i in range(len(sizes)))
        elif mode == "tuned":
            tuned = b.autotune(2)
            assert set(tuned) == {(64, 64), (128, 96), (96, 128)}
            for ms0, ms1, chosen in tuned.values():
                assert ms0 > 0 and ms1 > 0 and chosen == (1 if ms1 < ms0 else 0)
        for i, F in enumerate(fields):
            b.load(i, F)
        E, _ = b.step(5, 1e300)
        runs.append((E, [f.cpu().numpy() for f in b.fields]))
    for E, fs in runs[1:]:
        np.testing.assert_allclose(E, runs[0][0], rtol=1e-12)
        for a, c in zip(fs, runs[0][1]):
            np.testing.assert_array_equal(a, c)


def test_batch_small_shape_rejected_without_tma():
    th = load_theory("Baby Skyrme")
    params = [th.params.default_params(xlen=33, ylen=70, lsx=0.1, lsy=0.1, unit_magnetization=True)]
    b = BatchSolver(th, params, "fp32")
    assert not b.tma_enabled
    with pytest.raises(ValueError, match="TMA"):
        b.set_shape(0, 1)
    tuned = b.autotune(1)
    assert list(tuned.values())[0][2] == 0
