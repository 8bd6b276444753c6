"""Generate golden vectors from the reference soliton_solver itself.

Run in a container that has the reference checkout (it is NOT needed at test time):

    python tests/golden/make_golden.py --ref <reference checkout> --out tests/golden

It imports the reference package with Numba's CUDA simulator enabled
(``NUMBA_ENABLE_CUDASIM=1``; no GPU is used) and with empty stand-in modules for
the viewer's window/GL imports (``glfw``, ``OpenGL*``, ``moderngl``) so that the
theory packages register; no GL code is ever executed.  It then calls the
reference's own hooks on seeded random fields and writes their outputs:

* per-hook cases: ``do_gradient_step_kernel`` (l_out and EnergyGradient),
  ``compute_energy_kernel`` (energy density), the charge-density kernels, the
  ``observables.compute_*`` scalar reductions, ``do_rk4_step_kernel`` and the
  theory's RK4 finalize kernel;
* trajectory cases: several ``Simulation.step`` calls (energy and err per step,
  final Field and Velocity), including one case where arrest fires.

Each case is one ``.npz`` file holding the theory name, the packed ``p_i``/``p_f``
arrays the reference built, the inputs and the outputs.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
import types

import numpy as np


def _import_reference(ref_root):
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    for name in ["glfw", "OpenGL", "OpenGL.GL", "OpenGL.GL.shaders", "OpenGL.GLUT", "moderngl"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, ref_root)
    from numba import cuda  # noqa: F401
    from soliton_solver.theories import load_theory
    from soliton_solver.core.simulation import Simulation
    from soliton_solver.core import integrator
    return load_theory, Simulation, integrator


THEORY_NAMES = {
    "chiral_magnet": "Chiral magnet",
    "baby_skyrme": "Baby Skyrme model",
    "ginzburg_landau_superconductor": "Ginzburg-Landau superconductor",
    "anisotropic_superconductor": "Anisotropic superconductor",
}


def _random_field(theory, rp, rng, amp=0.3):
    nf, X, Y = rp.number_total_fields, rp.xlen, rp.ylen
    x = np.linspace(-1, 1, X)[:, None]
    y = np.linspace(-1, 1, Y)[None, :]
    F = np.zeros((nf, X, Y))
    if theory in ("chiral_magnet", "baby_skyrme"):
        r = np.sqrt(x * x + y * y)
        th = np.arctan2(y, x)
        f = np.pi * np.exp(-r / 0.5)
        F[0] = np.sin(f) * np.cos(th)
        F[1] = np.sin(f) * np.sin(th)
        F[2] = np.cos(f)
        F[:3] += amp * rng.standard_normal((3, X, Y))
        n = np.sqrt((F[:3] ** 2).sum(0))
        F[:3] /= n
        if nf > 3:
            F[3:] = amp * rng.standard_normal((nf - 3, X, Y))
    else:
        F[:] = amp * rng.standard_normal((nf, X, Y))
        F[2] += 0.8
        if nf > 4:
            F[4] += 0.5
    return F


def _cases():
    common = dict(xlen=13, ylen=10, xsize=2.4, ysize=1.8)
    out = []
    for dmi in ("Dresselhaus", "Rashba", "Heusler", "Hybrid"):
        for demag in (False, True):
            out.append((f"chiral_{dmi.lower()}_demag{int(demag)}", "chiral_magnet",
                        dict(common, dmi_term=dmi, demag=demag, B=0.15, unit_magnetization=True)))
    out.append(("chiral_halo3", "chiral_magnet",
                dict(common, xlen=15, ylen=12, halo=3, dmi_term="Heusler", demag=True, unit_magnetization=True)))
    pots = ["Standard", "Holomorphic", "Easy plane", "Dihedral2", "Aloof", "Dihedral3", "Broken", "DoubleVacua"]
    for pot in pots:
        out.append((f"bs_{pot.replace(' ', '').lower()}", "baby_skyrme",
                    dict(common, potential=pot, kappa=0.8, mpi=1.3, unit_magnetization=True, N=2)))
    out.append(("bs_broken_n3", "baby_skyrme",
                dict(common, potential="Broken", kappa=1.1, mpi=0.7, unit_magnetization=True, N=3)))
    out.append(("bs_mixed", "baby_skyrme",
                dict(common, potential=["Standard", "Easy plane"], kappa=1.0, mpi=1.0, unit_magnetization=True)))
    out.append(("ah_default", "ginzburg_landau_superconductor", dict(common, q=1.0, Lambda=1.0, u1=1.0)))
    out.append(("ah_quirk", "ginzburg_landau_superconductor",
                dict(common, q=0.7, Lambda=2.0, u1=1.2, vortex_number=1.5)))
    out.append(("sid_default", "anisotropic_superconductor", dict(common)))
    out.append(("sid_neg_beta4", "anisotropic_superconductor",
                dict(common, beta4=-0.3, Q=0.8, kappa=0.9, gamma12=0.3)))
    return out


def _traj_cases():
    common = dict(xlen=12, ylen=9, xsize=2.2, ysize=1.6)
    return [
        ("traj_chiral", "chiral_magnet",
         dict(common, dmi_term="Heusler", demag=True, B=0.1, unit_magnetization=True), 1e300, 3),
        ("traj_chiral_arrest", "chiral_magnet",
         dict(common, dmi_term="Rashba", demag=False, unit_magnetization=True), -1e300, 3),
        ("traj_bs", "baby_skyrme",
         dict(common, potential="Standard", kappa=1.0, mpi=1.0, time_step=0.01, unit_magnetization=True), 1e300, 3),
        ("traj_ah", "ginzburg_landau_superconductor", dict(common, q=1.0, Lambda=1.0, u1=1.0), 1e300, 3),
        ("traj_sid", "anisotropic_superconductor", dict(common), 1e300, 2),
    ]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SOLITON_SOLVER_REF"), required="SOLITON_SOLVER_REF" not in os.environ,
                    help="root of the reference soliton_solver checkout (or set SOLITON_SOLVER_REF)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    load_theory, Simulation, integrator = _import_reference(args.ref)
    from numba import cuda

    os.makedirs(args.out, exist_ok=True)
    for seed, (name, theory, kw) in enumerate(_cases()):
        if args.only and args.only not in name:
            continue
        t0 = time.time()
        th = load_theory(THEORY_NAMES[theory])
        sim = Simulation(th.params.default_params(**kw), th)
        rp = sim.rp
        rng = np.random.default_rng(1000 + seed)
        F = _random_field(theory, rp, rng)
        V = 0.2 * rng.standard_normal(F.shape)
        sim.Field.copy_to_device(F.reshape(-1))
        sim.Velocity.copy_to_device(V.reshape(-1))
        grid2d, block2d = ((rp.xlen + 7) // 8, (rp.ylen + 7) // 8), (8, 8)
        rec = dict(theory=theory, p_i=sim.p_i_h, p_f=sim.p_f_h, field=F.reshape(-1), velocity=V.reshape(-1))
        # gradient hook
        th.kernels.do_gradient_step_kernel[grid2d, block2d](sim.l1, sim.Field, sim.d1fd1x, sim.d2fd2x,
                                                           sim.EnergyGradient, sim.p_i_d, sim.p_f_d)
        cuda.synchronize()
        rec["l_out"] = sim.l1.copy_to_host()
        rec["energy_gradient"] = sim.EnergyGradient.copy_to_host()
        # energy density + reduction
        th.kernels.compute_energy_kernel[grid2d, block2d](sim.en, sim.Field, sim.d1fd1x, sim.p_i_d, sim.p_f_d)
        cuda.synchronize()
        rec["energy_density"] = sim.en.copy_to_host()
        rec["energy"] = np.float64(th.observables.compute_energy(sim.Field, sim.d1fd1x, sim.en, sim.entmp,
                                                                 sim.gridsum_partial, sim.p_i_d, sim.p_f_d,
                                                                 sim.p_i_h, sim.p_f_h))
        obs = sim.observables()
        for k, v in obs.items():
            rec["obs_" + k] = np.float64(v)
        # densities
        if hasattr(th.kernels, "compute_skyrmion_number_kernel"):
            th.kernels.compute_skyrmion_number_kernel[grid2d, block2d](sim.en, sim.Field, sim.d1fd1x,
                                                                       sim.p_i_d, sim.p_f_d)
            cuda.synchronize()
            rec["skyrmion_density"] = sim.en.copy_to_host()
        if hasattr(th.kernels, "compute_magnetic_charge_kernel"):
            th.kernels.compute_magnetic_charge_kernel[grid2d, block2d](sim.Field, sim.d1fd1x, sim.en,
                                                                       sim.p_i_d, sim.p_f_d)
            cuda.synchronize()
            rec["magnetic_charge_density"] = sim.en.copy_to_host()
        if hasattr(th.kernels, "compute_vortex_number_kernel"):
            th.kernels.compute_vortex_number_kernel[grid2d, block2d](sim.en, sim.Field, sim.d1fd1x, 2,
                                                                     sim.p_i_d, sim.p_f_d)
            cuda.synchronize()
            rec["vortex_density"] = sim.en.copy_to_host()
        # RK4 stage and finalize hooks on random slopes
        ks = [0.1 * rng.standard_normal(F.size) for _ in range(4)]
        ls = [0.1 * rng.standard_normal(F.size) for _ in range(4)]
        for buf, val in zip((sim.k1, sim.k2, sim.k3, sim.k4, sim.l1, sim.l2, sim.l3, sim.l4), ks + ls):
            buf.copy_to_device(val)
        integrator.do_rk4_step_kernel[grid2d, block2d](sim.k2, sim.Velocity, sim.l1, sim.Temp, sim.Field, sim.k1,
                                                       0.5, sim.p_i_d, sim.p_f_d)
        cuda.synchronize()
        rec["rk4_stage_k_out"] = sim.k2.copy_to_host()
        rec["rk4_stage_temp"] = sim.Temp.copy_to_host()
        sim.k2.copy_to_device(ks[1])
        rec["rk4_k"] = np.stack(ks)
        rec["rk4_l"] = np.stack(ls)
        sim.rk4_kernel[grid2d, block2d](sim.Velocity, sim.Field, sim.k1, sim.k2, sim.k3, sim.k4,
                                        sim.l1, sim.l2, sim.l3, sim.l4, sim.p_i_d, sim.p_f_d)
        cuda.synchronize()
        rec["rk4_final_velocity"] = sim.Velocity.copy_to_host()
        rec["rk4_final_field"] = sim.Field.copy_to_host()
        np.savez_compressed(os.path.join(args.out, f"hook_{name}.npz"), **rec)
        print(f"hook_{name}: {time.time() - t0:.1f}s", flush=True)

    # diagnostic densities of the gauge theories through the reference's Simulation helpers
    for seed, (name, theory, kw) in enumerate(_cases()):
        if theory not in ("ginzburg_landau_superconductor", "anisotropic_superconductor"):
            continue
        if args.only and args.only not in "density_" + name:
            continue
        th = load_theory(THEORY_NAMES[theory])
        sim = Simulation(th.params.default_params(**kw), th)
        rp = sim.rp
        F = _random_field(theory, rp, np.random.default_rng(3000 + seed))
        sim.Field.copy_to_device(F.reshape(-1))
        rec = dict(theory=theory, p_i=sim.p_i_h, p_f=sim.p_f_h, field=F.reshape(-1))
        N = rp.xlen * rp.ylen
        if theory == "ginzburg_landau_superconductor":
            sim.compute_higgs_density()
            rec["higgs"] = sim.en.copy_to_host()
        else:
            sim.compute_higgs1_density()
            rec["higgs1"] = sim.en.copy_to_host()
            sim.compute_higgs2_density()
            rec["higgs2"] = sim.en.copy_to_host()
            sim.compute_phase_difference_density()
            rec["phase"] = sim.en.copy_to_host()
            rec["magnetic"] = sim.magnetic_field().copy_to_host()[:N]
        rec["supercurrent"] = sim.supercurrent().copy_to_host()[:2 * N]
        np.savez_compressed(os.path.join(args.out, f"density_{name}.npz"), **rec)
        print(f"density_{name}", flush=True)

    for seed, (name, theory, kw, prev_e, nsteps) in enumerate(_traj_cases()):
        if args.only and args.only not in name:
            continue
        t0 = time.time()
        th = load_theory(THEORY_NAMES[theory])
        sim = Simulation(th.params.default_params(**kw), th)
        sim.initialize({"mode": "ground"})
        rp = sim.rp
        rng = np.random.default_rng(2000 + seed)
        F = _random_field(theory, rp, rng, amp=0.05)
        V = 0.05 * rng.standard_normal(F.shape)
        sim.Field.copy_to_device(F.reshape(-1))
        sim.Velocity.copy_to_device(V.reshape(-1))
        E_traj, err_traj = [], []
        E = prev_e
        for _ in range(nsteps):
            E, err = sim.step(E)
            E_traj.append(E)
            err_traj.append(err)
        rec = dict(theory=theory, p_i=sim.p_i_h, p_f=sim.p_f_h, field=F.reshape(-1), velocity=V.reshape(-1),
                   prev_energy=np.float64(prev_e), n_steps=np.int64(nsteps),
                   energy_traj=np.array(E_traj), err_traj=np.array(err_traj),
                   final_field=sim.Field.copy_to_host(), final_velocity=sim.Velocity.copy_to_host())
        np.savez_compressed(os.path.join(args.out, f"{name}.npz"), **rec)
        print(f"{name}: {time.time() - t0:.1f}s E={E_traj}", flush=True)


if __name__ == "__main__":
    main()
