"""Golden initial conditions from the reference's own initial-condition kernels.

Run in a container that has the reference checkout (it is NOT needed at test time):

    python tests/golden/make_golden_init.py --ref <reference checkout> --out tests/golden

With Numba's CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``; no GPU, no GL) it builds
each theory's coordinate grid with the theory's ``create_grid_kernel`` and runs, per
theory, ``create_ground_state_kernel``, ``create_initial_configuration_kernel``
(called directly with its full argument list: the chiral magnet's and baby Skyrme's
``initialize(mode="initial")`` passes one argument too few and cannot run; the
Abelian Higgs kernel reads ``ainf`` one slot past the packed ``p_f``, so it is given
``p_f`` with ``ainf`` appended) and the
soliton-insertion kernel (``create_skyrmion_kernel`` / ``create_vortex_kernel``)
applied on top of the ground state and of the ansatz.  Each case is one
``init_*.npz`` with the packed parameters, the arguments and the resulting Field
(and Velocity where the kernel writes it).
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys
import types

import numpy as np

THEORIES = {
    "chiral_magnet": ("Chiral magnet", dict(xlen=23, ylen=17, xsize=4.4, ysize=3.2, demag=True, skyrmion_number=1.0)),
    "baby_skyrme": ("Baby Skyrme model", dict(xlen=19, ylen=24, xsize=3.6, ysize=4.6, skyrmion_number=2.0)),
    "ginzburg_landau_superconductor": ("Ginzburg-Landau superconductor",
                                       dict(xlen=21, ylen=18, xsize=6.0, ysize=5.1, u1=1.3, vortex_number=2.0)),
    "anisotropic_superconductor": ("Anisotropic superconductor", dict(xlen=20, ylen=22, xsize=5.7, ysize=6.3)),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SOLITON_SOLVER_REF"), required="SOLITON_SOLVER_REF" not in os.environ,
                    help="root of the reference soliton_solver checkout (or set SOLITON_SOLVER_REF)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    for name in ["glfw", "OpenGL", "OpenGL.GL", "OpenGL.GL.shaders", "OpenGL.GLUT", "moderngl"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, args.ref)
    from soliton_solver.theories import load_theory

    for key, (name, kw) in THEORIES.items():
        th = load_theory(name)
        ic = importlib.import_module(f"soliton_solver.theories.{key}.initial_config")
        rp = th.params.default_params(**kw).resolved()
        p_i, p_f = th.params.pack_device_params(rp)
        X, Y, nf = rp.xlen, rp.ylen, rp.number_total_fields
        N = X * Y
        launch = ((X + 7) // 8, (Y + 7) // 8), (8, 8)
        grid = np.zeros(2 * N)
        th.kernels.create_grid_kernel[launch](grid, p_i, p_f)
        z = lambda: np.zeros(nf * N)  # noqa: E731
        scratch = [z() for _ in range(9)]  # k1..k4, l1..l4, Temp

        def save(case, F, V=None, **extra):
            np.savez_compressed(os.path.join(args.out, f"init_{key}_{case}.npz"), theory=key, p_i=p_i, p_f=p_f,
                                field=F, velocity=V if V is not None else np.zeros(0), **extra)

        V = np.full(nf * N, 0.7)
        F = np.full(nf * N, 0.3)
        ic.create_ground_state_kernel[launch](V, F, grid, *scratch, p_i, p_f)
        save("ground", F.copy(), V.copy(), mode=0)
        ground = F.copy()
        if key in ("chiral_magnet", "baby_skyrme"):
            ansatz_cases = [("bloch", (1, 0, 0), 0.0), ("neel", (0, 1, 0), 0.4), ("anti", (0, 0, 1), -1.1),
                            ("none", (0, 0, 0), 0.0)]
            for tag, (b, n, a), rot in ansatz_cases:
                V = np.full(nf * N, 0.7)
                F = np.full(nf * N, 0.3)
                ic.create_initial_configuration_kernel[launch](V, F, grid, *scratch, bool(b), bool(n), bool(a), rot,
                                                               1.0, p_i, p_f)
                save(f"initial_{tag}", F.copy(), V.copy(), mode=1, ansatz=[b, n, a], rotation=rot)
            base = ground.copy()
            for tag, (b, n, a), rot, (pxi, pxj) in (("bloch", (1, 0, 0), 0.3, (7, 5)), ("anti", (0, 0, 1), 0.0,
                                                                                        (X - 4, Y - 3))):
                F = base.copy()
                ic.create_skyrmion_kernel[launch](F, grid, pxi, pxj, rot, bool(b), bool(n), bool(a), p_i, p_f)
                save(f"insert_{tag}", F.copy(), None, mode=2, ansatz=[b, n, a], rotation=rot, pxi=pxi, pxj=pxj,
                     before=base.copy())
                base = F.copy()
        else:
            if key == "ginzburg_landau_superconductor":
                # the kernel reads ainf from p_f[11], one past the packed array (ainf is
                # p_f[10]); append ainf so that the reference kernel can run
                p_f_ext = np.append(p_f, p_f[10])
                V = np.full(nf * N, 0.7)
                F = np.full(nf * N, 0.3)
                ic.create_initial_configuration_kernel[launch](V, F, grid, *scratch, 2.0, p_i, p_f_ext)
                save("initial", F.copy(), V.copy(), mode=1, vortex_number=2.0)
            else:
                V = np.full(nf * N, 0.7)
                F = np.full(nf * N, 0.3)
                ic.create_initial_configuration_kernel[launch](V, F, grid, *scratch, p_i, p_f)
                save("initial", F.copy(), V.copy(), mode=1)
            base = F.copy()
            for tag, vortex, (pxi, pxj) in (("vortex", True, (6, 8)), ("antivortex", False, (X - 5, 4))):
                F = base.copy()
                ic.create_vortex_kernel[launch](F, grid, pxi, pxj, vortex, p_i, p_f)
                save(f"insert_{tag}", F.copy(), None, mode=2, vortex=vortex, pxi=pxi, pxj=pxj, before=base.copy())
                base = F.copy()
        print("wrote", key)


if __name__ == "__main__":
    main()
