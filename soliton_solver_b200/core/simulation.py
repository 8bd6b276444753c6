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


def fp32_stalled(E_prev: float, energies, plateau: float) -> bool:
    """One chunk of an arrested FP32 flow at FP32's resolution: no two consecutive steps
    lower the energy (each free step is followed by an arrest, so no velocity builds
    up), fewer than 60% of the steps raise it (a saddle flow raises E on nearly every
    step while it converges), and the energy moved by less than 10 x ``plateau`` x |E|
    over the chunk.  ``E_prev``: the energy before the chunk."""
    Eh = np.asarray(energies, dtype=np.float64)
    if Eh.size < 2:
        return False
    up = np.diff(np.concatenate([[E_prev], Eh])) > 0
    E = float(Eh[-1])
    return (not np.any(~up[1:] & ~up[:-1])) and float(up.mean()) < 0.6 and abs(E_prev - E) < 10 * plateau * abs(E)


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

    # The reference's Simulation allocates the derivative, RK4 and reduction scratch that
    # its hooks pass around (soliton_solver/core/simulation.py:91-115).  The fused kernels
    # never read them, so they are allocated only when a caller touches them, with the
    # reference's sizes: reference-style code such as
    # observables.compute_energy(sim.Field, sim.d1fd1x, sim.en, ...) runs unchanged.
    def __getattr__(self, name):
        sizes = self._scratch_sizes()
        if name not in sizes:
            raise AttributeError(f"{type(self).__name__!s} has no attribute {name!r}")
        n, dtype = sizes[name]
        t = torch.zeros(int(n), dtype=dtype, device=self.__dict__["device"])
        self.__dict__[name] = t
        return t

    def _scratch_sizes(self):
        rp = self.__dict__.get("rp")
        if rp is None:
            return {}
        field_dtype = torch.float32 if self.__dict__.get("precision") == "fp32" else torch.float64
        nc, nf, N = rp.number_coordinates, rp.number_total_fields, rp.dim_grid
        ng = int(getattr(rp, "number_gauge_fields", 0))
        out = {f"{k}{i}": (rp.dim_fields, field_dtype) for k in ("k", "l") for i in range(1, 5)}
        out.update(Temp=(rp.dim_fields, field_dtype), d1fd1x=(nc * nf * N, torch.float64),
                   d2fd2x=(nc * nc * nf * N, torch.float64), gridsum_partial=((N + 1023) // 1024, torch.float64),
                   max_partial=((rp.dim_fields + 1023) // 1024, torch.float64),
                   MagneticFluxDensity=(ng * N if ng > 0 else 1, torch.float64),
                   Supercurrent=(ng * N if ng > 0 else 1, torch.float64))
        return out

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

    def minimize(self, tol: float = 1e-6, max_steps: int = 1_000_000, schedule: str | None = None,
                 chunk: int | None = None, plateau: float = 1e-9, record: bool = False) -> dict:
        """Relax sim.Field by arrested Newton flow until the stage-4 gradient max
        |dE/dphi| (the reference's err) drops below ``tol``.

        The reference documents ``sim.minimize(tol=...)`` (soliton_solver/core/
        simulation.py:8,39) but relaxes by calling ``E, err = sim.step(E)`` until err <
        tol (core/integrator.py:217-348); this runs that loop on the device in chunks of
        ``chunk`` steps (one host synchronisation per chunk, CUDA-graph replays).

        schedule
          "fp64"       FP64 fields throughout (an FP64 copy of an FP32 Simulation's field).
          "fp32"       FP32 fields with FP64 energy sums; stops at tol or at the FP32
                       energy plateau (see below), whichever comes first.
          "fp32+fp64"  (default for FP32 Simulations) the FP32 flow until tol or its
                       plateau, then the same flow on an FP64 copy of the state, each
                       site's unit vector renormalised in FP64, until tol.  FP32 steps
                       run at about a third of the FP64 cost; FP32 rounding bounds how far
                       they get (the gradient stalls at ~eps/h^2), and the FP64 steps
                       finish from there.
        An FP32 phase reaches its plateau when, for two chunks in a row, its energy moves
        by less than ``plateau`` x |E| (in either direction: the flow of a saddle field
        such as the chiral magnet's demag potential raises E while it converges), or the
        flow has stalled at FP32's resolution: no two consecutive steps of the chunk lower
        the energy (every free step is followed by an arrest, so no velocity builds up),
        fewer than 60% of them raise it (a saddle flow raises E on nearly every step) and
        the energy moved by less than 10 x ``plateau`` x |E|.  (C2, the 320^2 chiral
        anti-skyrmion: the stall sets in after ~39 000 FP32 steps; the FP64 phase then
        needs 1 100 steps, against 106 000 from the state 9 000 steps earlier and 3 700
        from the state 30 000 steps later.)  ``max_steps`` bounds the total.  Needs the
        arrested flow (killkinen on).

        Returns a dict: energy (FP64 observable of the final field), err, converged,
        steps, and per phase its precision, steps, wall seconds, start/end energy, end
        err and stop reason.  The final field is written to sim.Field (rounded to its
        element type) and kept in FP64 as sim.Field64 after an FP64 phase.  With
        ``record`` the result also holds the per-step energy / err trajectories and, for
        FP32 phases, the FP64 projected energy at every chunk end."""
        import time

        if not int(self.p_i_h[7]):
            raise ValueError("minimize needs the arrested flow: set killkinen=True in the parameters")
        if schedule is None:
            schedule = "fp32+fp64" if self.precision == "fp32" else "fp64"
        if schedule not in ("fp64", "fp32", "fp32+fp64"):
            raise ValueError("schedule must be 'fp64', 'fp32' or 'fp32+fp64'")
        if schedule != "fp64" and self.precision != "fp32":
            raise ValueError(f"schedule {schedule!r} needs an FP32 Simulation")
        N = self.rp.dim_grid
        chunk = int(chunk) if chunk else 1000
        out = {"schedule": schedule, "tol": tol, "phases": [], "steps": 0}
        traj = {"energy": [], "err": [], "precision": [], "projected": []}
        budget = int(max_steps)
        E_start = self.observables()["energy"] if math.isnan(self.last_energy) else self.last_energy

        def phase(solver, field, vel, prec, E0, budget, project_chunks):
            t0 = time.perf_counter()
            Et = torch.empty(chunk, dtype=torch.float64, device=self.device)
            rt = torch.empty(chunk, dtype=torch.float64, device=self.device)
            steps, hits, stalls, stop = 0, 0, 0, "max_steps"
            E_prev, E, err = E0, E0, math.inf
            graph = False
            while steps < budget:
                n = min(chunk, budget - steps)
                if n == chunk and steps > 0:
                    if not graph:
                        solver.capture(chunk, Et, rt)
                        graph = True
                    solver.replay()
                else:
                    solver.step_async(n, E0 if steps == 0 else math.nan, Et, rt)
                Eh = Et[:n].cpu().numpy()
                rh = rt[:n].cpu().numpy()
                solver.check_status()
                if record:
                    traj["energy"].append(Eh.copy())
                    traj["err"].append(rh.copy())
                    traj["precision"].append(np.full(n, 32 if prec == "fp32" else 64, np.int8))
                    if project_chunks:
                        traj["projected"].append((out["steps"] + steps + n, solver.energy_projected(field)))
                below = np.nonzero(np.abs(rh) < tol)[0]
                if below.size:
                    steps += int(below[0]) + 1
                    E, err, stop = float(Eh[below[0]]), float(rh[below[0]]), "tol"
                    break
                steps += n
                E, err = float(Eh[-1]), float(rh[-1])
                hits = hits + 1 if abs(E_prev - E) < plateau * abs(E) else 0
                stalls = stalls + 1 if fp32_stalled(E_prev, Eh, plateau) else 0
                E_prev = E
                if (hits >= 2 or stalls >= 2) and prec == "fp32":
                    stop = "plateau"
                    break
            torch.cuda.synchronize(self.device)
            rec = {"precision": prec, "steps": steps, "wall_s": time.perf_counter() - t0, "energy_start": E0,
                   "energy_end": E, "err_end": err, "stop": stop}
            out["phases"].append(rec)
            out["steps"] += steps
            return rec

        if schedule in ("fp32", "fp32+fp64"):
            rec = phase(self.solver, self.Field, self.Velocity, "fp32", E_start, budget, record)
            budget -= rec["steps"]
            E_start = rec["energy_end"]
            if schedule == "fp32" or rec["stop"] == "tol" or budget <= 0:
                out.update(energy=self.solver.energy(self.Field), err=rec["err_end"], converged=rec["stop"] == "tol")
                self.last_energy = rec["energy_end"]
                return self._finish_minimize(out, traj, record)
        # FP64 phase: on the Simulation's own buffers, or on a projected FP64 copy
        if self.precision == "fp32":
            F64 = torch.empty(self.Field.numel(), dtype=torch.float64, device=self.device)
            V64 = torch.empty_like(F64)
            self.solver.convert(self.Field, F64, project=True)
            self.solver.convert(self.Velocity, V64, project=False)
            s64 = Solver(self.kernels.THEORY_ID, self.p_i_h, self.p_f_h, "fp64", self.device)
            s64.bind(F64, V64)
            E_start = s64.energy(F64)
        else:
            F64, V64, s64 = self.Field, self.Velocity, self.solver
        rec = phase(s64, F64, V64, "fp64", E_start, budget, False)
        out.update(energy=s64.energy(F64), err=rec["err_end"], converged=rec["stop"] == "tol")
        if F64 is not self.Field:
            s64.convert(F64, self.Field, project=False)
            s64.convert(V64, self.Velocity, project=False)
            self.Field64 = F64
            self.solver.rebind()  # the FP32 flow restarts its arrest history from the new state
        self.last_energy = out["energy"]
        torch.cuda.synchronize(self.device)
        return self._finish_minimize(out, traj, record)

    @staticmethod
    def _finish_minimize(out, traj, record):
        if record:
            out["trajectory"] = {"energy": np.concatenate(traj["energy"]) if traj["energy"] else np.empty(0),
                                 "err": np.concatenate(traj["err"]) if traj["err"] else np.empty(0),
                                 "precision": np.concatenate(traj["precision"]) if traj["precision"] else
                                 np.empty(0, np.int8),
                                 "projected": np.array(traj["projected"], dtype=np.float64).reshape(-1, 2)}
        return out

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
        """The theory's .dat output bundle (soliton_solver/core/simulation.py:411-516):
        lattice sizes and vectors, the field dump and the component grids of the field,
        the energy density, the charge densities and, for the gauge theories, the Higgs
        densities, supercurrent and magnetic flux density, formatted on the GPU.  The
        default directory is the theory package's ``results``."""
        import inspect
        import os
        if output_dir is None:
            output_dir = os.path.join(os.path.dirname(os.path.abspath(self.theory.io.__file__)), "results")
        os.makedirs(output_dir, exist_ok=True)
        self.kernels.create_grid_kernel[None, None](self.grid, self.p_i_h, self.p_f_h)
        om = self.observables_mod
        dens = {"h_EnergyDensity": self.solver.energy_density(self.Field).clone()}
        for name, method in (("h_MagneticFluxDensity", self.magnetic_field), ("h_Supercurrent", self.supercurrent)):
            try:
                dens[name] = method().clone()
            except AttributeError:  # the theory has no such kernel: the reference skips it too
                pass
        if hasattr(om, "compute_skyrmion_number"):
            dens["h_BaryonDensity"] = self.solver.charge_density(self.Field, "skyrmion").clone()
        if hasattr(om, "compute_magnetic_charge"):
            dens["h_MagneticChargeDensity"] = self.solver.charge_density(self.Field, "magnetic").clone()
        if hasattr(om, "compute_vortex_number"):
            dens["h_VortexDensity"] = self.solver.charge_density(self.Field, "vortex").clone()
        if hasattr(self.kernels, "compute_norm_higgs_kernel"):
            dens["h_HiggsDensity"] = self.solver.field_density(self.Field, "higgs").clone()
        if hasattr(self.kernels, "compute_norm_higgs1_kernel"):
            dens["h_Higgs1Density"] = self.solver.field_density(self.Field, "higgs1").clone()
            dens["h_Higgs2Density"] = self.solver.field_density(self.Field, "higgs2").clone()
        dens.setdefault("h_Supercurrent", None)
        dens.setdefault("h_MagneticFluxDensity", None)
        kwargs = dict(output_dir=output_dir, h_Field=self.Field, h_grid=self.grid, xlen=int(self.p_i_h[0]),
                      ylen=int(self.p_i_h[1]),
                      number_coordinates=int(self.p_i_h[3]), number_total_fields=int(self.p_i_h[4]),
                      precision=precision, **dens)
        accepted = set(inspect.signature(self.theory.io.output_data_bundle).parameters)
        self.theory.io.output_data_bundle(**{k: v for k, v in kwargs.items() if k in accepted})

    def compute_energy_density(self):
        self.solver.energy_density(self.Field, self.en)
        torch.cuda.synchronize(self.device)

    # diagnostic densities of the gauge theories (soliton_solver/core/simulation.py:211-386)
    def _kernel_density(self, kernel_name, kind, out):
        if not hasattr(self.kernels, kernel_name):
            raise AttributeError(f"theory kernels have no {kernel_name}")
        self.solver.field_density(self.Field, kind, out)
        torch.cuda.synchronize(self.device)
        return out

    def compute_higgs_density(self):
        """|psi|^2 per site into ``en`` (compute_norm_higgs_kernel)."""
        self._kernel_density("compute_norm_higgs_kernel", "higgs", self.en)

    def compute_higgs1_density(self):
        """|psi1|^2 per site into ``en`` (compute_norm_higgs1_kernel)."""
        self._kernel_density("compute_norm_higgs1_kernel", "higgs1", self.en)

    def compute_higgs2_density(self):
        """|psi2|^2 per site into ``en`` (compute_norm_higgs2_kernel)."""
        self._kernel_density("compute_norm_higgs2_kernel", "higgs2", self.en)

    def compute_phase_difference_density(self):
        """cos(arg psi1 - arg psi2) per site into ``en`` (compute_phase_difference_kernel)."""
        self._kernel_density("compute_phase_difference_kernel", "phase", self.en)

    def magnetic_field(self):
        """Magnetic flux density (dx A2 - dy A1) dA/(2 pi Q) into the first N entries of
        ``MagneticFluxDensity`` and returned (compute_magnetic_field_kernel; the
        Ginzburg-Landau theory has none, as in the reference)."""
        return self._kernel_density("compute_magnetic_field_kernel", "magnetic", self.MagneticFluxDensity)

    def supercurrent(self):
        """Supercurrent (dxy A2 - dyy A1, dxy A1 - dxx A2) into ``Supercurrent`` (x plane,
        then y plane) and returned (compute_supercurrent_kernel)."""
        return self._kernel_density("compute_supercurrent_kernel", "supercurrent", self.Supercurrent)

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
