"""Initial configurations of the s+id superconductor theory.

``initialize``, ``create_ground_state_kernel``, ``create_initial_configuration_kernel`` and
``create_vortex_kernel`` keep the reference's names and signatures
(soliton_solver/theories/anisotropic_superconductor/initial_config.py) and run the native initial-condition
kernels (``ss_initialize``, ``ss_insert_soliton``).

The ground state of ``initialize(mode="ground")`` follows the reference's
create_ground_state_kernel, which reads u1, u2 from p_f[11], p_f[12] (beta2, beta3 in
the packed parameters); ``vacuum`` returns the physical vacuum (u1, u2).
"""
from __future__ import annotations

import math

from soliton_solver_b200 import _native as _nat
from soliton_solver_b200.core.initial import make_initial_config


def vacuum(rp):
    """Per-component vacuum values."""
    return [0.0, 0.0, rp.u1, 0.0, rp.u2 * math.cos(rp.theta_diff), rp.u2 * math.sin(rp.theta_diff)]


globals().update(make_initial_config(_nat.SS_THEORY_ANISOTROPIC, "anisotropic_superconductor"))
