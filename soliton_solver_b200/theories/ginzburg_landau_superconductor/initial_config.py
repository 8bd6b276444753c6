"""Initial configurations of the Abelian Higgs (Ginzburg-Landau) theory.

``initialize``, ``create_ground_state_kernel``, ``create_initial_configuration_kernel`` and
``create_vortex_kernel`` keep the reference's names and signatures
(soliton_solver/theories/ginzburg_landau_superconductor/initial_config.py) and run the native initial-condition
kernels (``ss_initialize``, ``ss_insert_soliton``).

The reference's create_initial_configuration_kernel reads ainf from p_f[11], one past
the packed array; the native kernel reads the packed ainf, p_f[10].
"""
from __future__ import annotations

from soliton_solver_b200 import _native as _nat
from soliton_solver_b200.core.initial import make_initial_config


def vacuum(rp):
    """Per-component vacuum values."""
    return [0.0, 0.0, rp.u1, 0.0]


globals().update(make_initial_config(_nat.SS_THEORY_GINZBURG_LANDAU, "ginzburg_landau_superconductor"))
