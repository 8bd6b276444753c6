"""Observables of the Anisotropic superconductor theory with the reference's signatures
(soliton_solver/theories/anisotropic_superconductor/observables.py), reduced on the GPU in FP64 with a
fixed-order compensated sum."""
from soliton_solver_b200.core.hooks import make_observables
from soliton_solver_b200.theories.anisotropic_superconductor.kernels import CHARGES, THEORY_ID

globals().update(make_observables(THEORY_ID, CHARGES))
