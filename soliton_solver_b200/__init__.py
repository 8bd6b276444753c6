"""soliton_solver_b200: B200-native (sm_100a) backend for soliton_solver's flow hot path.

Public surface mirrors the reference package:

    from soliton_solver_b200.theories import load_theory
    from soliton_solver_b200.core.simulation import Simulation

    theory = load_theory("Chiral magnet")
    params = theory.params.default_params(xlen=320, ylen=320, xsize=10.0, ysize=10.0, dmi_term="Heusler",
                                          unit_magnetization=True)
    sim = Simulation(params, theory)          # precision="fp32" | "fp64" | "plain_fp64"
    sim.initialize({"mode": "ground"})
    E, err = sim.step(prev_energy)

All compute runs in libsoliton_b200.so (built by ``python -m soliton_solver_b200.build``).
"""
__version__ = "0.1.0"
