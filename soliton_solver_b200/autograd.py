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


def _minres(apply, b, tol, max_iter, monitor=None, every=200, precond=None):
    """Preconditioned MINRES (Paige and Saunders) for the symmetric, possibly indefinite
    A x = b from x = 0, with the symmetric positive definite preconditioner precond(v) =
    M^-1 v (identity when None); returns (x, iterations, relative preconditioned residual).
    monitor(x, it) is called every `every` iterations and ends the solve when it returns
    True."""
    import torch
    minv = precond if precond is not None else (lambda v: v)
    x = torch.zeros_like(b)
    r1 = b.clone()
    y = minv(r1)
    beta1 = float(torch.dot(r1, y)) ** 0.5 if float(torch.dot(r1, y)) > 0 else 0.0
    if beta1 == 0.0:
        return x, 0, 0.0
    r2 = r1.clone()
    w = torch.zeros_like(b)
    w2 = torch.zeros_like(b)
    oldb, beta, dbar, epsln, phibar, cs, sn = 0.0, beta1, 0.0, 0.0, beta1, -1.0, 0.0
    it = 0
    for it in range(1, max_iter + 1):
        v = y / beta
        y = apply(v)
        if it >= 2:
            y = y - (beta / oldb) * r1
        alfa = float(torch.dot(v, y))
        y = y - (alfa / beta) * r2
        r1, r2 = r2, y
        y = minv(r2)
        oldb = beta
        beta = max(float(torch.dot(r2, y)), 0.0) ** 0.5
        oldeps = epsln
        delta = cs * dbar + sn * alfa
        gbar = sn * dbar - cs * alfa
        epsln = sn * beta
        dbar = -cs * beta
        gamma = max((gbar * gbar + beta * beta) ** 0.5, 1e-300)
        cs, sn = gbar / gamma, beta / gamma
        phi = cs * phibar
        phibar = sn * phibar
        w1, w2 = w2, w
        w = (v - oldeps * w1 - delta * w2) / gamma
        x = x + phi * w
        if phibar <= tol * beta1 or beta == 0.0:
            break
        if monitor is not None and it % every == 0 and monitor(x, it):
            break
    return x, it, phibar / beta1


def relaxed_coupling_gradients(sim, names=None, tol: float = 1e-8, max_iter: int = 20000, eps: float = 1e-6,
                               rtol: float = 1e-4, precondition: bool = True, shift: float = 1.0):
    """dE_min/dc at a relaxed field, with the discretisation correction of the adjoint.

    The flow relaxes to the zero of the reference's stencil gradient S (the 4th-order
    functional derivative, projected and with the chiral magnet's halo ring frozen),
    which is not the exact derivative X = dE_h/dphi / dA of the discrete energy sum E_h:
    r = X - S is O(h^4) in the interior and O(1/h) at the rows next to the frozen ring
    (the masked DMI term).  The relaxed energy E_min(c) = E_h(phi*(c), c) therefore has
        dE_min/dc = dE_h/dc (the envelope value) + dA <P r, dphi*/dc>,
    where P projects onto the flowed (tangent, non-ring) directions.  Linearising the
    stationarity condition P S(phi*(c), c) = 0 gives A dphi*/dc = -P dS/dc with A the
    Jacobian of P S (symmetric in the true rows of ss_energy_gradient), so the correction
    is -dA <w, P dS/dc> with A w = P r: one MINRES solve for all couplings (the adjoint
    method).  A is applied through central differences of the native stencil gradient
    along w (ss_energy_gradient, 2 evaluations per iteration, step eps relative to the
    largest entry of w), dS/dc by central differences in the coupling (solvers at
    c (1 +- 1e-4); S is linear in the reduced couplings but for the demag row's 1/coup_mu).
    With `precondition`, MINRES runs with the symmetric positive definite preconditioner
    P (shift - Laplacian)^-1 P (per component by FFT, periodic, second-order symbol; the
    demag row scaled by coup_mu, whose true-row block is Laplacian / coup_mu with the
    opposite sign): the spectrum of the preconditioned operator no longer spreads with
    1/h^2 and the saddle's indefinite block costs no more than the rest.  The solve stops
    at relative residual `tol`, after `max_iter` iterations, or when every correction has
    moved by less than `rtol` of itself over the last 1000 iterations.
    The field is the FP64 relaxed state (sim.Field64 after a mixed-precision minimize,
    else sim.Field).  Returns (grads, info) with info = the envelope values, the
    corrections, MINRES iterations and relative residual.  The Simulation is not
    modified."""
    import numpy as np
    import torch

    from soliton_solver_b200.core.solver import Solver

    src = getattr(sim, "Field64", None) if sim.precision == "fp32" else sim.Field
    if src is None:
        raise ValueError("an FP32 Simulation needs its FP64 relaxed state (sim.minimize with an FP64 phase)")
    rp = sim.rp
    nf, X, Y = rp.number_total_fields, rp.xlen, rp.ylen
    nmag = int(getattr(rp, "number_magnetization_fields", 0)) if getattr(sim.kernels, "CONSTRAINED", False) else 0
    ring = int(rp.halo) if sim.kernels.THEORY_ID == 0 else 0  # the chiral magnet freezes its halo ring
    F = src.detach().clone().to(torch.float64).reshape(-1)
    s64 = Solver(sim.kernels.THEORY_ID, sim.p_i_h, sim.p_f_h, "fp64", sim.device)
    s64.bind(F.clone(), torch.zeros_like(F))
    mhat = None
    if nmag:
        m = F.view(nf, X, Y)[:nmag]
        mhat = m / torch.linalg.vector_norm(m, dim=0, keepdim=True)

    def project(v):
        v = v.view(nf, X, Y).clone()
        if nmag:
            v[:nmag] -= (v[:nmag] * mhat).sum(0, keepdim=True) * mhat
        if ring:
            v[:, :ring] = 0
            v[:, -ring:] = 0
            v[:, :, :ring] = 0
            v[:, :, -ring:] = 0
        return v.reshape(-1)

    def flow_residual(field):
        """P S at `field` (projected with the field's own unit vectors)."""
        g = s64.energy_gradient(field).view(nf, X, Y).clone()
        if nmag:
            mm = field.view(nf, X, Y)[:nmag]
            mh = mm / torch.linalg.vector_norm(mm, dim=0, keepdim=True)
            g[:nmag] -= (g[:nmag] * mh).sum(0, keepdim=True) * mh
        return g.reshape(-1)

    def apply(v):
        step = eps / max(float(v.abs().max()), 1e-300)
        return project((flow_residual(F + step * v) - flow_residual(F - step * v)) / (2 * step))

    precond = None
    if precondition:
        fx = torch.fft.fftfreq(X, device=F.device, dtype=torch.float64)[:, None]
        fy = torch.fft.rfftfreq(Y, device=F.device, dtype=torch.float64)[None, :]
        symbol = (4.0 / rp.lsx ** 2) * torch.sin(torch.pi * fx) ** 2 + (4.0 / rp.lsy ** 2) * torch.sin(torch.pi * fy) ** 2
        inv_symbol = 1.0 / (symbol + shift)
        scale = torch.ones(nf, 1, 1, dtype=torch.float64, device=F.device)
        if sim.kernels.THEORY_ID == 0 and int(sim.p_i_h[15]):
            scale[3] = float(sim.p_f_h[8])  # demag row: (shift - Laplacian) / coup_mu

        def precond(v):
            v = project(v).view(nf, X, Y)
            z = torch.fft.irfft2(torch.fft.rfft2(v) * inv_symbol, s=(X, Y)) * scale
            return project(z)

    r = s64.energy_gradient_exact(F, minus_stencil=True)
    b = project(r)
    g0 = _partials(sim, s64, F, names)
    dA = float(sim.p_f_h[4])
    # dS/dc (true rows, projected) of every physical coupling by central differences
    dS = {}
    for name in g0:
        c = getattr(sim.p, name, None)
        if c is None or not c:
            continue
        h = 1e-4 * c
        S = []
        for sgn in (1, -1):
            ps = sim.p.with_(**{name: c + sgn * h}).resolved()
            p_i, p_f = sim.theory.params.pack_device_params(ps)
            sc = Solver(sim.kernels.THEORY_ID, p_i, p_f, "fp64", sim.device)
            sc.bind(F.clone(), torch.zeros_like(F))
            S.append(sc.energy_gradient(F))
            del sc
        dS[name] = project((S[0] - S[1]) / (2 * h))
    history = []

    def monitor(x, it):
        corr = {k: -dA * float(torch.dot(x, v)) for k, v in dS.items()}
        history.append((it, corr))
        if len(history) < 6:
            return False
        old = history[-6][1]  # the corrections 1000 iterations ago
        return all(abs(corr[k] - old[k]) <= rtol * max(abs(corr[k]), 1e-300) for k in corr)

    w, iters, rel = _minres(apply, b, tol, max_iter, monitor if dS else None, precond=precond)
    corr = {k: -dA * float(torch.dot(w, v)) for k, v in dS.items()}
    out = {k: g0[k] + corr.get(k, 0.0) for k in g0}
    info = {"uncorrected": g0, "correction": corr, "minres_iterations": iters, "minres_rel_residual": rel,
            "residual_max": float(r.abs().max()), "residual_projected_max": float(b.abs().max()),
            "history": history[-10:]}
    return out, info
