"""Observables of the Ginzburg-Landau superconductor theory with the reference's signatures
(soliton_solver/theories/ginzburg_landau_superconductor/observables.py), reduced on the GPU in FP64 with a
fixed-order compensated sum."""
from soliton_solver_b200.core.hooks import make_observables
from soliton_solver_b200.theories.ginzburg_landau_superconductor.kernels import CHARGES, THEORY_ID

globals().update(make_observables(THEORY_ID, CHARGES))
