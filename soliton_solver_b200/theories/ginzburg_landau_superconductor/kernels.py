"""Hook adapters of the Ginzburg-Landau superconductor theory.

Same hook names and call signatures as soliton_solver/theories/ginzburg_landau_superconductor/kernels.py;
every call runs the hand-written sm_100a kernels of libsoliton_b200.
"""
from soliton_solver_b200 import _native as _nat
from soliton_solver_b200.core.hooks import make_kernels

THEORY_ID = _nat.SS_THEORY_GINZBURG_LANDAU
CHARGES = ('vortex',)
DENSITIES = ('higgs', 'supercurrent')
CONSTRAINED = False

globals().update(make_kernels(THEORY_ID, CHARGES, DENSITIES))

del do_rk4_kernel  # unconstrained: Simulation uses the core no-constraint finalize
