"""Observables of the Chiral magnet theory with the reference's signatures
(soliton_solver/theories/chiral_magnet/observables.py), reduced on the GPU in FP64 with a
fixed-order compensated sum."""
from soliton_solver_b200.core.hooks import make_observables
from soliton_solver_b200.theories.chiral_magnet.kernels import CHARGES, THEORY_ID

globals().update(make_observables(THEORY_ID, CHARGES))
