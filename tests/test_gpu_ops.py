"""The torch.library custom ops of soliton_b200 against the direct Solver calls.

Each op must return what the native call it wraps returns (bitwise: same kernels, same
inputs), flow_step must advance exactly the buffers it is given, and torch.library.opcheck's
schema and fake-tensor checks must pass (the schema check also verifies that
flow_step mutates field and velocity and nothing else).
"""
import numpy as np
import pytest
import torch

from soliton_solver_b200 import autograd as ops
from soliton_solver_b200.core.solver import Solver
from soliton_solver_b200.theories import load_theory

pytestmark = pytest.mark.gpu


def _setup(prec="fp32"):
    th = load_theory("Chiral magnet")
    rp = th.params.default_params(xlen=96, ylen=128, xsize=6.0, ysize=8.0, dmi_term="Heusler", demag=True, B=0.2,
                                  unit_magnetization=True).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    rng = np.random.default_rng(5)
    x = np.linspace(-1, 1, rp.xlen)[:, None]
    y = np.linspace(-1, 1, rp.ylen)[None, :]
    F = np.stack([0.4 * np.sin(2 * x + rng.normal()) * np.cos(1.5 * y + rng.normal()) for _ in range(4)])
    F[2] += 1.0
    F[:3] /= np.sqrt((F[:3] ** 2).sum(0))
    dt = torch.float32 if prec == "fp32" else torch.float64
    f = torch.tensor(F.reshape(-1), dtype=dt, device="cuda")
    return th, p_i, p_f, f


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_ops_equal_direct_calls(prec):
    th, p_i, p_f, f = _setup(prec)
    s = Solver(0, p_i, p_f, prec)
    key = ops.register(s)
    eg = torch.empty_like(f)
    s.gradient(f, eg, None)
    assert torch.equal(torch.ops.soliton_b200.gradient(f, key), eg)
    assert torch.equal(torch.ops.soliton_b200.energy_gradient(f, key), s.energy_gradient(f))
    assert torch.ops.soliton_b200.energy(f, key).item() == s.energy(f)
    for which in ("skyrmion", "magnetic"):
        assert torch.ops.soliton_b200.charge(f, key, which).item() == s.charge(f, which)
    for c in ("coup_K", "coup_h", "coup_mu"):
        assert torch.ops.soliton_b200.coupling_grad(f, key, c).item() == s.coupling_grad(f, c)


def test_flow_step_op_advances_the_bound_buffers():
    th, p_i, p_f, f0 = _setup()
    a = Solver(0, p_i, p_f, "fp32")
    fa, va = f0.clone(), torch.zeros_like(f0)
    a.bind(fa, va)
    key = ops.register(a)
    E, err = torch.ops.soliton_b200.flow_step(fa, va, key, 5, 1e300)
    b = Solver(0, p_i, p_f, "fp32")
    fb, vb = f0.clone(), torch.zeros_like(f0)
    b.bind(fb, vb)
    Eb, errb = b.step(5, 1e300)
    np.testing.assert_array_equal(E.cpu().numpy(), Eb)
    np.testing.assert_array_equal(err.cpu().numpy(), errb)
    assert torch.equal(fa, fb) and torch.equal(va, vb)
    # other buffers are bound first and advanced like a fresh solver's
    fc, vc = f0.clone(), torch.zeros_like(f0)
    Ec, _ = torch.ops.soliton_b200.flow_step(fc, vc, key, 5, 1e300)
    np.testing.assert_array_equal(Ec.cpu().numpy(), Eb)
    assert torch.equal(fc, fb) and torch.equal(vc, vb)
    assert a.field is fc


def test_opcheck_schema_and_fake():
    th, p_i, p_f, f = _setup()
    s = Solver(0, p_i, p_f, "fp32")
    key = ops.register(s)
    utils = ("test_schema", "test_faketensor")
    torch.library.opcheck(ops.gradient_op, (f, key), test_utils=utils)
    torch.library.opcheck(ops.charge_op, (f, key, "skyrmion"), test_utils=utils)
    torch.library.opcheck(ops.coupling_grad_op, (f, key, "coup_h"), test_utils=utils)
    fs, vs = f.clone(), torch.zeros_like(f)
    s.bind(fs, vs)
    torch.library.opcheck(ops.flow_step_op, (fs, vs, key, 2, 1e300), test_utils=utils)
