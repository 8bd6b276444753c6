"""Initial configurations of the Baby Skyrme theory.

``initialize``, ``create_ground_state_kernel``, ``create_initial_configuration_kernel`` and
``create_skyrmion_kernel`` keep the reference's names and signatures
(soliton_solver/theories/baby_skyrme/initial_config.py) and run the native initial-condition
kernels (``ss_initialize``, ``ss_insert_soliton``).

The reference's ``initialize(mode="initial")`` (its default mode) passes one argument
too few to create_initial_configuration_kernel and cannot run; this one runs the ansatz.
"""
from __future__ import annotations

from soliton_solver_b200 import _native as _nat
from soliton_solver_b200.core.initial import make_initial_config


def vacuum(rp):
    """Per-component vacuum values."""
    return [0.0, 0.0, 1.0]


globals().update(make_initial_config(_nat.SS_THEORY_BABY_SKYRME, "baby_skyrme"))
