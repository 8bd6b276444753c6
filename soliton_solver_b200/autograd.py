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


def coupling_gradients(sim, names=None) -> dict:
    """dE/dc at sim.Field for the named couplings (all the theory supports by default)."""
    mod = sim.theory.__name__.rsplit(".", 1)[-1]
    solver = sim.solver
    if mod == "chiral_magnet":
        red = {c: solver.coupling_grad(sim.Field, c) for c in _REDUCED[mod]}
        chain = sim.theory.params.coupling_chain(sim.rp)
        out = dict(red)
        for phys, parts in chain.items():
            out[phys] = sum(red[c] * d for c, d in parts.items())
        if names is not None:
            out = {k: out[k] for k in names}
        return out
    avail = {"baby_skyrme": ("kappa", "mpi"), "ginzburg_landau_superconductor": ("Lambda",)}.get(mod, ())
    names = avail if names is None else names
    return {c: solver.coupling_grad(sim.Field, c) for c in names}
