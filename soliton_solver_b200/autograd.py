"""Differentiable discrete energy and coupling gradients.

``energy(field, solver)`` is E[phi] = sum_sites e(phi) dA as a torch scalar whose
backward is the hand-written gradient kernel: dE/dphi = dA * (functional
derivative), the same stencil that drives the flow, evaluated without the unit-norm
projection and with the demag psi row as the true dE/dpsi (ss_energy_gradient).
It agrees with the derivative of the discrete sum up to O(h^4) interior terms and
the masked boundary ring; ``tests/test_autograd.py`` states the tolerance.

The native calls are registered as torch.library custom ops so they compose with
torch's dispatcher (fake tensors, opcheck); solvers are passed by an integer key of
``register()``:

  soliton_b200::energy(field, key) -> f64 scalar          ss_energy (differentiable)
  soliton_b200::energy_gradient(field, key) -> like field  ss_energy_gradient
  soliton_b200::gradient(field, key) -> like field         ss_gradient (projected EG)
  soliton_b200::charge(field, key, which) -> f64 scalar    ss_charge
  soliton_b200::coupling_grad(field, key, name) -> f64     ss_coupling_grad
  soliton_b200::flow_step(field!, velocity!, key, n_steps, prev_energy) -> (E, err)
                                                           ss_step_async on field and
                                                           velocity (mutated in place)

``coupling_gradients(sim, names)`` returns dE/dc at the current field for the
couplings of the theory (kappa, mpi for the baby Skyrme model, Lambda for
Ginzburg-Landau, B, K, D for the chiral magnet through the reduced couplings).  At a
relaxed field this is dE_min/dc (envelope theorem).
"""
from __future__ import annotations

import itertools

import torch

_SOLVERS: dict = {}
_KEYS = itertools.count(1)


def register(solver) -> int:
    """Integer key under which the custom ops find `solver`."""
    key = getattr(solver, "_op_key", None)
    if key is None:
        key = next(_KEYS)
        solver._op_key = key
        _SOLVERS[key] = solver
    return key


@torch.library.custom_op("soliton_b200::energy", mutates_args=())
def energy_op(field: torch.Tensor, key: int) -> torch.Tensor:
    s = _SOLVERS[key]
    return torch.tensor(s.energy(field.contiguous()), dtype=torch.float64, device=field.device)


@energy_op.register_fake
def _(field, key):
    return field.new_empty((), dtype=torch.float64)


@torch.library.custom_op("soliton_b200::energy_gradient", mutates_args=())
def energy_gradient_op(field: torch.Tensor, key: int) -> torch.Tensor:
    s = _SOLVERS[key]
    return s.energy_gradient(field.contiguous())


@energy_gradient_op.register_fake
def _(field, key):
    return torch.empty_like(field)


@torch.library.custom_op("soliton_b200::gradient", mutates_args=())
def gradient_op(field: torch.Tensor, key: int) -> torch.Tensor:
    s = _SOLVERS[key]
    out = torch.empty_like(field)
    s.gradient(field.contiguous(), out, None)
    return out


@gradient_op.register_fake
def _(field, key):
    return torch.empty_like(field)


@torch.library.custom_op("soliton_b200::charge", mutates_args=())
def charge_op(field: torch.Tensor, key: int, which: str) -> torch.Tensor:
    s = _SOLVERS[key]
    return torch.tensor(s.charge(field.contiguous(), which), dtype=torch.float64, device=field.device)


@charge_op.register_fake
def _(field, key, which):
    return field.new_empty((), dtype=torch.float64)


@torch.library.custom_op("soliton_b200::coupling_grad", mutates_args=())
def coupling_grad_op(field: torch.Tensor, key: int, name: str) -> torch.Tensor:
    s = _SOLVERS[key]
    return torch.tensor(s.coupling_grad(field.contiguous(), name), dtype=torch.float64, device=field.device)


@coupling_grad_op.register_fake
def _(field, key, name):
    return field.new_empty((), dtype=torch.float64)


@torch.library.custom_op("soliton_b200::flow_step", mutates_args=("field", "velocity"))
def flow_step_op(field: torch.Tensor, velocity: torch.Tensor, key: int, n_steps: int,
                 prev_energy: float) -> tuple[torch.Tensor, torch.Tensor]:
    """n_steps arrested-Newton-flow steps of `field` and `velocity` in place; energy and
    err trajectories stay on the device (no host synchronisation).  Buffers other than
    the solver's bound ones are bound first (which starts a fresh arrest history, as
    Solver.bind does)."""
    s = _SOLVERS[key]
    if s.field is None or field.data_ptr() != s.field.data_ptr() or velocity.data_ptr() != s.velocity.data_ptr():
        s.bind(field, velocity)
    E = torch.empty(n_steps, dtype=torch.float64, device=field.device)
    err = torch.empty(n_steps, dtype=torch.float64, device=field.device)
    s.step_async(n_steps, prev_energy, E, err)
    return E, err


@flow_step_op.register_fake
def _(field, velocity, key, n_steps, prev_energy):
    return (field.new_empty((n_steps,), dtype=torch.float64), field.new_empty((n_steps,), dtype=torch.float64))


def _setup(ctx, inputs, output):
    field, key = inputs
    ctx.save_for_backward(field)
    ctx.key = key


def _backward(ctx, grad_E):
    (field,) = ctx.saved_tensors
    s = _SOLVERS[ctx.key]
    g = energy_gradient_op(field, ctx.key)
    dA = float(s.p_f[4])
    return (g * (grad_E.to(g.dtype) * dA)), None


energy_op.register_autograd(_backward, setup_context=_setup)


def energy(field: torch.Tensor, solver) -> torch.Tensor:
    """Differentiable total energy of `field` (flat, reference layout, solver's dtype)."""
    return energy_op(field, register(solver))


_REDUCED = {"chiral_magnet": ("coup_K", "coup_h", "coup_mu")}


def _partials(sim, solver, field, names):
    """dE/dc of `field` for the theory's couplings (chiral magnet: B, K, D through the
    reduced couplings' chain rule, plus the reduced ones)."""
    mod = sim.theory.__name__.rsplit(".", 1)[-1]
    if mod == "chiral_magnet":
        red = {c: solver.coupling_grad(field, c) for c in _REDUCED[mod]}
        chain = sim.theory.params.coupling_chain(sim.rp)
        out = dict(red)
        for phys, parts in chain.items():
            out[phys] = sum(red[c] * d for c, d in parts.items())
        if names is not None:
            out = {k: out[k] for k in names}
        return out
    avail = {"baby_skyrme": ("kappa", "mpi"), "ginzburg_landau_superconductor": ("Lambda",)}.get(mod, ())
    names = avail if names is None else names
    return {c: solver.coupling_grad(field, c) for c in names}


def coupling_gradients(sim, names=None) -> dict:
    """dE/dc at sim.Field for the named couplings (all the theory supports by default)."""
    return _partials(sim, sim.solver, sim.Field, names)


def relaxed_coupling_gradients(sim, names=None, max_steps: int = 20000, chunk: int = 500, rtol: float = 1e-9):
    """dE_min/dc at a relaxed field, consistent with the discrete energy sum.

    The flow relaxes to the zero of the reference's stencil gradient G, which differs
    from the exact derivative of the discrete energy sum E_h by an O(h^4) residual r.
    The relaxed energy E_min(c) = E_h(phi*(c)) differs from E_h at the stationary point
    of E_h only by O(h^8), so dE_min/dc is dE_h/dc there (envelope theorem), while dE_h/dc
    at phi* itself is off by O(h^4).  This runs the FP64 flow from the relaxed state
    (sim.Field64 after a mixed-precision minimize, else sim.Field) with the frozen
    residual r(phi*) added to its gradient (ss_energy_gradient_exact, ss_set_forcing):
    its stationary point is that of E_h to O(h^8).  It stops when every coupling
    derivative moves by less than rtol (relative) over a chunk, or after max_steps.
    Returns (grads, info) with info = steps, the uncorrected envelope values and the
    relative size of the correction.  The Simulation's own state is not modified."""
    import math

    import numpy as np
    import torch

    from soliton_solver_b200.core.solver import Solver

    src = getattr(sim, "Field64", None) if sim.precision == "fp32" else sim.Field
    if src is None:
        raise ValueError("an FP32 Simulation needs its FP64 relaxed state (sim.minimize with an FP64 phase)")
    p_i = np.array(sim.p_i_h, dtype=np.int32, copy=True)
    p_i[7] = 1  # the arrested flow
    s64 = Solver(sim.kernels.THEORY_ID, p_i, sim.p_f_h, "fp64", sim.device)
    F = src.detach().clone().to(torch.float64)
    V = torch.zeros_like(F)
    s64.bind(F, V)
    g0 = _partials(sim, s64, F, names)
    r = s64.energy_gradient_exact(F, minus_stencil=True)
    s64.set_forcing(r)
    E0 = s64.energy(F)
    g_prev, steps = g0, 0
    try:
        while steps < max_steps:
            s64.step(chunk, E0 if steps == 0 else math.nan)
            steps += chunk
            g = _partials(sim, s64, F, names)
            if all(abs(g[k] - g_prev[k]) <= rtol * max(abs(g[k]), 1e-300) for k in g):
                break
            g_prev = g
    finally:
        s64.set_forcing(None)
    rel = {k: abs(g[k] - g0[k]) / max(abs(g[k]), 1e-300) for k in g}
    return g, {"steps": steps, "uncorrected": g0, "correction_rel": rel, "residual_max": float(r.abs().max())}
