"""Initial configurations of the Anisotropic superconductor theory.

``initialize`` keeps the reference's keyword signature
(soliton_solver/theories/anisotropic_superconductor/initial_config.py) and its ``mode="ground"``
vacuum.  Seeded soliton ansätze for benchmarks and tests live in
``soliton_solver_b200.initial_conditions`` and are written into ``sim.Field``.
"""
from __future__ import annotations

import math

import torch

from soliton_solver_b200.core.hooks import as_tensor
from soliton_solver_b200.core.solver import _to_host


def vacuum(rp):
    """Per-component vacuum values."""
    return [0.0, 0.0, rp.u1, 0.0, rp.u2 * math.cos(rp.theta_diff), rp.u2 * math.sin(rp.theta_diff)]


def initialize(*, Velocity, Field, grid=None, k1=None, k2=None, k3=None, k4=None, l1=None, l2=None, l3=None,
               l4=None, Temp=None, p_i_d=None, p_f_d=None, p_i_h=None, p_f_h=None, grid2d=None, block2d=None,
               config: dict | None = None, rp=None):
    cfg = config or {}
    mode = str(cfg.get("mode", "initial")).lower()
    if mode not in ("ground", "uniform", "vacuum", "gs"):
        raise NotImplementedError(
            f"initial mode {mode!r}: only the ground state is built in; write an ansatz from "
            "soliton_solver_b200.initial_conditions into sim.Field")
    F = as_tensor(Field)
    V = as_tensor(Velocity)
    if rp is None:
        raise ValueError("initialize needs the resolved parameters (rp=...)")
    N = int(rp.dim_grid)
    for a, v in enumerate(vacuum(rp)):
        F[a * N:(a + 1) * N].fill_(float(v))
    V.zero_()
    for buf in (k1, k2, k3, k4, l1, l2, l3, l4, Temp):
        if buf is not None:
            as_tensor(buf).zero_()
