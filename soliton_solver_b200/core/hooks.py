"""Launch adapters with the reference's hook names and call signatures.

The reference's theories expose Numba kernels launched as
``kernel[grid2d, block2d](args...)`` and host helpers such as
``observables.compute_energy(...)``.  The objects built here accept exactly those
calls (the launch configuration is ignored: the native library picks its own) and
forward them to libsoliton_b200 through a cached ``Solver`` keyed by the packed
parameter arrays.  Derivative scratch arguments (``d1fd1x``, ``d2fd2x``) and the
reduction scratch (``entmp``, ``gridsum_partial``) are accepted and left
untouched: the fused kernels never materialise derivatives.
"""
from __future__ import annotations

import torch

from soliton_solver_b200.core.solver import solver_for


def as_tensor(x):
    """Torch view of a device buffer (torch tensor or __cuda_array_interface__ object)."""
    if isinstance(x, torch.Tensor):
        return x
    if hasattr(x, "__cuda_array_interface__"):
        return torch.as_tensor(x, device="cuda")
    raise TypeError(f"expected a CUDA buffer, got {type(x)!r}")


class Launch:
    """``obj[grid, block](*args)`` and ``obj(*args)`` both call ``fn(*args)``."""

    def __init__(self, fn, name):
        self.fn = fn
        self.__name__ = name

    def __getitem__(self, launch_config):
        return self.fn

    def __call__(self, *args, **kwargs):
        return self.fn(*args, **kwargs)


def _solver(theory_id, field, p_i, p_f):
    f = as_tensor(field)
    return solver_for(theory_id, p_i, p_f, f.dtype, f.device), f


def _geometry_solver(theory_id, field, p_i):
    """Solver for hooks that pass only p_i (pointwise densities): the float parameters
    are never read by those kernels, so unit placeholders stand in for them."""
    import numpy as np
    from soliton_solver_b200.core.solver import _to_host
    pf = np.ones(32)
    return _solver(theory_id, field, _to_host(p_i), pf)


def make_kernels(theory_id: int, charges=(), densities=()):
    """Hook adapters of one theory: returns a dict name -> Launch.  ``densities`` names
    the diagnostic densities the theory's kernels module provides ('higgs', 'higgs1',
    'higgs2', 'phase', 'supercurrent', 'magnetic')."""

    def do_gradient_step_kernel(l_out, Field, d1fd1x, d2fd2x, EnergyGradient, p_i, p_f):
        s, f = _solver(theory_id, Field, p_i, p_f)
        s.gradient(f, as_tensor(EnergyGradient) if EnergyGradient is not None else None,
                   as_tensor(l_out) if l_out is not None else None)

    def do_rk4_kernel(Velocity, Field, k1, k2, k3, k4, l1, l2, l3, l4, p_i, p_f):
        s, f = _solver(theory_id, Field, p_i, p_f)
        s.rk4_finalize(as_tensor(Velocity), f, *(as_tensor(t) for t in (k1, k2, k3, k4, l1, l2, l3, l4)))

    def do_rk4_step_kernel(k_out, Velocity, l_in, Temp, Field, k_prev, factor, p_i, p_f):
        s, f = _solver(theory_id, Field, p_i, p_f)
        s.rk4_stage(as_tensor(k_out), as_tensor(Velocity), as_tensor(l_in), as_tensor(Temp), f, as_tensor(k_prev),
                    factor)

    def compute_energy_kernel(en, Field, d1fd1x, p_i, p_f):
        s, f = _solver(theory_id, Field, p_i, p_f)
        s.energy_density(f, as_tensor(en))

    def create_grid_kernel(grid, p_i, p_f):
        g = as_tensor(grid)
        from soliton_solver_b200.core.solver import _to_host
        pi, pf = _to_host(p_i), _to_host(p_f)
        X, Y = int(pi[0]), int(pi[1])
        x = torch.arange(X, device=g.device, dtype=torch.float64)[:, None].expand(X, Y)
        y = torch.arange(Y, device=g.device, dtype=torch.float64)[None, :].expand(X, Y)
        g[: X * Y].copy_((float(pf[2]) * x).reshape(-1))
        g[X * Y: 2 * X * Y].copy_((float(pf[3]) * y).reshape(-1))

    out = {
        "do_gradient_step_kernel": Launch(do_gradient_step_kernel, "do_gradient_step_kernel"),
        "do_rk4_step_kernel": Launch(do_rk4_step_kernel, "do_rk4_step_kernel"),
        "compute_energy_kernel": Launch(compute_energy_kernel, "compute_energy_kernel"),
        "create_grid_kernel": Launch(create_grid_kernel, "create_grid_kernel"),
        "do_rk4_kernel": Launch(do_rk4_kernel, "do_rk4_kernel"),
    }
    if "skyrmion" in charges:
        def compute_skyrmion_number_kernel(en, Field, d1fd1x, p_i, p_f):
            s, f = _solver(theory_id, Field, p_i, p_f)
            s.charge_density(f, "skyrmion", as_tensor(en))
        out["compute_skyrmion_number_kernel"] = Launch(compute_skyrmion_number_kernel,
                                                       "compute_skyrmion_number_kernel")
    if "magnetic" in charges:
        def compute_magnetic_charge_kernel(Field, d1fd1x, en, p_i, p_f):
            s, f = _solver(theory_id, Field, p_i, p_f)
            s.charge_density(f, "magnetic", as_tensor(en))
        out["compute_magnetic_charge_kernel"] = Launch(compute_magnetic_charge_kernel,
                                                       "compute_magnetic_charge_kernel")
    if "vortex" in charges:
        def compute_vortex_number_kernel(en, Field, d1fd1x, which, p_i, p_f):
            s, f = _solver(theory_id, Field, p_i, p_f)
            s.charge_density(f, "vortex", as_tensor(en))
        out["compute_vortex_number_kernel"] = Launch(compute_vortex_number_kernel, "compute_vortex_number_kernel")
    pointwise = {"higgs": "compute_norm_higgs_kernel", "higgs1": "compute_norm_higgs1_kernel",
                 "higgs2": "compute_norm_higgs2_kernel", "phase": "compute_phase_difference_kernel"}
    for kind, name in pointwise.items():
        if kind in densities:
            def pointwise_kernel(en, Field, p_i, _kind=kind):
                s, f = _geometry_solver(theory_id, Field, p_i)
                s.field_density(f, _kind, as_tensor(en))
            out[name] = Launch(pointwise_kernel, name)
    if "supercurrent" in densities:
        def compute_supercurrent_kernel(Field, d2fd2x, Supercurrent, p_i, p_f):
            s, f = _solver(theory_id, Field, p_i, p_f)
            s.field_density(f, "supercurrent", as_tensor(Supercurrent))
        out["compute_supercurrent_kernel"] = Launch(compute_supercurrent_kernel, "compute_supercurrent_kernel")
    if "magnetic" in densities:
        def compute_magnetic_field_kernel(Field, d1fd1x, MagneticFluxDensity, p_i, p_f):
            s, f = _solver(theory_id, Field, p_i, p_f)
            s.field_density(f, "magnetic", as_tensor(MagneticFluxDensity))
        out["compute_magnetic_field_kernel"] = Launch(compute_magnetic_field_kernel, "compute_magnetic_field_kernel")
    return out


def make_observables(theory_id: int, charges=()):
    """Host observables with the reference's signatures (e.g. chiral_magnet/observables.py:15-141)."""

    def compute_energy(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h, p_f_h):
        s, f = _solver(theory_id, Field, p_i_h, p_f_h)
        return s.energy(f)

    out = {"compute_energy": compute_energy}
    if "skyrmion" in charges:
        def compute_skyrmion_number(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h):
            s, f = _solver(theory_id, Field, p_i_h, p_f_d)
            return s.charge(f, "skyrmion")
        out["compute_skyrmion_number"] = compute_skyrmion_number
    if "magnetic" in charges:
        def compute_magnetic_charge(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h):
            s, f = _solver(theory_id, Field, p_i_h, p_f_d)
            return s.charge(f, "magnetic")
        out["compute_magnetic_charge"] = compute_magnetic_charge
    if "vortex" in charges:
        def compute_vortex_number(Field, d1fd1x, en, entmp, gridsum_partial, which, p_i_d, p_f_d, p_i_h):
            s, f = _solver(theory_id, Field, p_i_h, p_f_d)
            return s.charge(f, "vortex")
        out["compute_vortex_number"] = compute_vortex_number
    return out
