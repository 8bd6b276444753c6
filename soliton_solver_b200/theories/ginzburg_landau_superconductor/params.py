"""Ginzburg-Landau (Abelian Higgs) parameters.

Same fields and packed layout as the reference
(soliton_solver/theories/ginzburg_landau_superconductor/params.py:18-194):
``p_i = core + [number_higgs_fields, number_gauge_fields]``;
``p_f = core + [q, Lambda, u1, vortex_number, ainf]`` with ``ainf = vortex_number/q``
unless given.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from soliton_solver_b200.core.params import Params as CoreParams
from soliton_solver_b200.core.params import ResolvedParams as CoreResolvedParams
from soliton_solver_b200.core.params import pack_device_params as pack_core_device_params


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 4
    number_higgs_fields: int = 2
    number_gauge_fields: int = 2
    q: float = 1.0
    Lambda: float = 1.0
    u1: float = 1.0
    vortex_number: float = 1.0
    ainf: float | None = None

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    number_higgs_fields: int
    number_gauge_fields: int
    q: float
    Lambda: float
    u1: float
    vortex_number: float
    ainf: float

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        core = CoreResolvedParams.core_fields(p)
        ainf = p.ainf if p.ainf is not None else p.vortex_number / p.q
        return ResolvedParams(**core, number_higgs_fields=int(p.number_higgs_fields),
                              number_gauge_fields=int(p.number_gauge_fields), q=float(p.q), Lambda=float(p.Lambda),
                              u1=float(p.u1), vortex_number=float(p.vortex_number), ainf=float(ainf))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    p_i, p_f = pack_core_device_params(rp)
    p_i_t = np.array([rp.number_higgs_fields, rp.number_gauge_fields], dtype=np.int32)
    p_f_t = np.array([rp.q, rp.Lambda, rp.u1, rp.vortex_number, rp.ainf], dtype=np.float64)
    return np.concatenate((p_i, p_i_t)), np.concatenate((p_f, p_f_t))


def describe() -> None:
    print("Field content: gauge field (A1, A2) and complex order parameter (Re psi, Im psi).")
    print("Couplings: q (charge), Lambda (potential), u1 (vacuum value).")
    print("Note: the energy density reads u from the vortex_number slot, as the reference does;")
    print("keep vortex_number == u1 for a consistent energy.")
