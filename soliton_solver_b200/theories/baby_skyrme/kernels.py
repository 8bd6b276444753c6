"""Hook adapters of the Baby Skyrme model theory.

Same hook names and call signatures as soliton_solver/theories/baby_skyrme/kernels.py;
every call runs the hand-written sm_100a kernels of libsoliton_b200.
"""
from soliton_solver_b200 import _native as _nat
from soliton_solver_b200.core.hooks import make_kernels

THEORY_ID = _nat.SS_THEORY_BABY_SKYRME
CHARGES = ('skyrmion',)
CONSTRAINED = True

globals().update(make_kernels(THEORY_ID, CHARGES))
