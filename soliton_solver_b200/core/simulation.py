"""Simulation: the reference's driver object on the B200 backend.

Same constructor, attributes and methods as soliton_solver/core/simulation.py:24-533
for the flow hot path (``initialize``, ``set_params``, ``step``, ``observables`` and
the density helpers), with device buffers held as torch tensors that expose
``__cuda_array_interface__`` (so a viewer can keep reading ``sim.Field``).  Every
step runs the fused sm_100a kernels of libsoliton_b200; the energy and the arrest
decision stay on the device.

Extra keyword arguments: ``precision`` ("fp32": FP32 fields with FP64 reductions,
the default; "fp64": FP64 fields; "plain_fp64": the reference-structured FP64
form) and ``device``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from soliton_solver_b200.core.params import Params
from soliton_solver_b200.core.solver import Solver


class Simulation:
    def __init__(self, params, theory, precision: str = "fp32", device=None):
        self.theory = theory
        self.kernels = theory.kernels
        self.initial_config = theory.initial_config
        self.observables_mod = theory.observables
        self.threads2d = getattr(theory, "threads2d", (8, 8))
        if getattr(self.kernels, "do_gradient_step_kernel", None) is None:
            raise AttributeError("Theory kernels must provide do_gradient_step_kernel.")
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.solver = None
        self.set_params(params)
        rp = self.rp
        dtype = torch.float32 if precision == "fp32" else torch.float64
        z = lambda n, dt=dtype: torch.zeros(int(n), dtype=dt, device=self.device)  # noqa: E731
        self.Field = z(rp.dim_fields)
        self.Velocity = z(rp.dim_fields)
        self.EnergyGradient = z(rp.dim_fields)
        self.grid = z(rp.number_coordinates * rp.dim_grid, torch.float64)
        self.en = z(rp.dim_grid, torch.float64)
        self.entmp = z(rp.dim_grid, torch.float64)
        self._make_solver()
        self.last_energy = math.nan

    # ------------------------------------------------------------------ setup
    def _make_solver(self):
        self.solver = Solver(self.kernels.THEORY_ID, self.p_i_h, self.p_f_h, self.precision, self.device)
        self.solver.bind(self.Field, self.Velocity)

    def set_params(self, p):
        """Re-resolve and re-pack the parameters (soliton_solver/core/simulation.py:144-166)."""
        self.p = p
        self.rp = p.resolved() if isinstance(p, Params) else p
        self.p_i_h, self.p_f_h = self.theory.params.pack_device_params(self.rp)
        self.p_i_d = torch.from_numpy(self.p_i_h).to(self.device)
        self.p_f_d = torch.from_numpy(self.p_f_h).to(self.device)
        if self.solver is not None:
            if int(self.p_i_h[6]) != self.Field.numel():
                raise ValueError("set_params cannot change the lattice size of an existing Simulation")
            self._make_solver()

    def initialize(self, init_config: dict | None = None):
        """Grid coordinates, zeroed buffers and the theory's initial configuration."""
        cfg = init_config or {}
        self.kernels.create_grid_kernel[None, None](self.grid, self.p_i_h, self.p_f_h)
        self.Field.zero_()
        self.Velocity.zero_()
        self.initial_config.initialize(Velocity=self.Velocity, Field=self.Field, grid=self.grid, p_i_d=self.p_i_d,
                                       p_f_d=self.p_f_d, p_i_h=self.p_i_h, p_f_h=self.p_f_h, config=cfg, rp=self.rp)
        torch.cuda.synchronize(self.device)

    def load_field(self, field, velocity=None):
        """Copy a host or device field (reference flat layout or (nf, xlen, ylen)) into sim.Field."""
        f = torch.as_tensor(np.asarray(field) if not isinstance(field, torch.Tensor) else field)
        self.Field.copy_(f.reshape(-1).to(self.Field.dtype))
        if velocity is None:
            self.Velocity.zero_()
        else:
            v = torch.as_tensor(np.asarray(velocity) if not isinstance(velocity, torch.Tensor) else velocity)
            self.Velocity.copy_(v.reshape(-1).to(self.Velocity.dtype))

    # ------------------------------------------------------------------ flow
    def step(self, prev_energy: float) -> tuple[float, float]:
        """One arrested-Newton-flow RK4 step; returns (new_energy, err)
        (soliton_solver/core/simulation.py:388-409)."""
        E, err = self.solver.step(1, prev_energy)
        self.last_energy = float(E[0])
        return float(E[0]), float(err[0])

    def relax(self, n_steps: int, prev_energy: float = math.nan):
        """``n_steps`` steps in one native call; returns (energy_traj, err_traj).

        With ``prev_energy`` NaN the first arrest test compares against the energy
        the previous call left on the device (or nothing, on the first call)."""
        E, err = self.solver.step(int(n_steps), prev_energy)
        if len(E):
            self.last_energy = float(E[-1])
        return E, err

    # ------------------------------------------------------------------ observables
    def observables(self):
        """Energy plus every charge the theory's observables module provides
        (soliton_solver/core/simulation.py:168-192)."""
        obs = {"energy": self.solver.energy(self.Field)}
        om = self.observables_mod
        if hasattr(om, "compute_skyrmion_number"):
            obs["skyrmion_number"] = self.solver.charge(self.Field, "skyrmion")
        if hasattr(om, "compute_vortex_number"):
            obs["vortex_number"] = self.solver.charge(self.Field, "vortex")
        if hasattr(om, "compute_magnetic_charge"):
            obs["magnetic_charge"] = self.solver.charge(self.Field, "magnetic")
        return obs

    def projected_energy(self) -> float:
        """FP64 energy of sim.Field with every site's magnetisation divided by its FP64
        norm.  For an FP32 relaxation this is the energy of the relaxed state on the
        constraint manifold: the stored FP32 m3 rounds to 1 wherever |m_perp| < 2.4e-4,
        which drops the |m_perp|^2 / 2 that the Zeeman and anisotropy terms should see
        there and biases the plain energy of a large vacuum downwards.  Equal to
        observables()["energy"] to FP64 rounding for FP64 fields and for theories
        without a unit-vector constraint."""
        return self.solver.energy_projected(self.Field)

    def save_output(self, output_dir: str | None = None, precision: int = 32):
        """The theory's .dat output bundle (soliton_solver/core/simulation.py save_output):
        lattice sizes and vectors, the field dump and the component grids of the field,
        the energy density and the theory's charge densities, formatted on the GPU.
        Arrays this backend does not compute (supercurrent, magnetic flux density) are
        passed as None and their files skipped, as the reference skips missing arrays.
        The default directory is the theory package's ``results``."""
        import inspect
        import os
        if output_dir is None:
            output_dir = os.path.join(os.path.dirname(os.path.abspath(self.theory.io.__file__)), "results")
        os.makedirs(output_dir, exist_ok=True)
        self.kernels.create_grid_kernel[None, None](self.grid, self.p_i_h, self.p_f_h)
        om = self.observables_mod
        dens = {"h_EnergyDensity": self.solver.energy_density(self.Field).clone()}
        if hasattr(om, "compute_skyrmion_number"):
            dens["h_BaryonDensity"] = self.solver.charge_density(self.Field, "skyrmion").clone()
        if hasattr(om, "compute_magnetic_charge"):
            dens["h_MagneticChargeDensity"] = self.solver.charge_density(self.Field, "magnetic").clone()
        if hasattr(om, "compute_vortex_number"):
            dens["h_VortexDensity"] = self.solver.charge_density(self.Field, "vortex").clone()
        kwargs = dict(output_dir=output_dir, h_Field=self.Field, h_grid=self.grid, h_Supercurrent=None,
                      h_MagneticFluxDensity=None, xlen=int(self.p_i_h[0]), ylen=int(self.p_i_h[1]),
                      number_coordinates=int(self.p_i_h[3]), number_total_fields=int(self.p_i_h[4]),
                      precision=precision, **dens)
        accepted = set(inspect.signature(self.theory.io.output_data_bundle).parameters)
        self.theory.io.output_data_bundle(**{k: v for k, v in kwargs.items() if k in accepted})

    def compute_energy_density(self):
        self.solver.energy_density(self.Field, self.en)
        torch.cuda.synchronize(self.device)

    def compute_magnetic_flux_density(self, which=2):
        self.solver.charge_density(self.Field, "vortex", self.en)
        torch.cuda.synchronize(self.device)

    def compute_magnetic_charge_density(self):
        self.solver.charge_density(self.Field, "magnetic", self.en)
        torch.cuda.synchronize(self.device)

    def compute_skyrmion_density(self):
        self.solver.charge_density(self.Field, "skyrmion", self.en)
        torch.cuda.synchronize(self.device)

    def gradient(self):
        """Projected energy gradient of the current field into sim.EnergyGradient."""
        self.solver.gradient(self.Field, self.EnergyGradient, None)
        return self.EnergyGradient

    def print_instructions(self):
        if hasattr(self.theory, "describe"):
            self.theory.describe()
        else:
            print("No specific instructions available for this theory.")
