"""Chiral magnet parameters.

Same fields, derived couplings and packed layout as the reference
(soliton_solver/theories/chiral_magnet/params.py:22-378):
``coup_K = K J / D^2``, ``coup_h = M B J / D^2``, ``coup_mu = mu0 M^2 J / D^2``
(all 1.0 when D == 0 and not given); ``p_i = core + [nmag, dresselhaus, rashba,
heusler, hybrid, demag]``; ``p_f = core + [coup_K, coup_h, coup_mu,
skyrmion_number, skyrmion_rotation, bloch, neel, anti, uniform]``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable

import numpy as np

from soliton_solver_b200.core.params import Params as CoreParams
from soliton_solver_b200.core.params import ResolvedParams as CoreResolvedParams
from soliton_solver_b200.core.params import pack_device_params as pack_core_device_params

_DMI_NAMES = {"dresselhaus": "dresselhaus", "bulk": "dresselhaus", "rashba": "rashba", "interfacial": "rashba",
              "heusler": "heusler", "b20": "heusler", "hybrid": "hybrid"}


def _norm(s) -> str:
    return (str(s) or "").strip().lower().replace("_", " ").replace("-", " ")


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 4
    number_magnetization_fields: int = 3
    J: float = 40e-12
    K: float = 0.8e6
    D: float = 4e-3
    M: float = 580e3
    B: float = 0.0
    mu0: float = 1.25663706127e-6
    coup_K: float | None = None
    coup_h: float | None = None
    coup_mu: float | None = None
    dmi_dresselhaus: bool = True
    dmi_rashba: bool = False
    dmi_heusler: bool = False
    dmi_hybrid: bool = False
    demag: bool = False
    dmi_term: str | Iterable[str] | None = None
    skyrmion_number: float = 1.0
    skyrmion_rotation: float = 0.0
    ansatz: str = "bloch"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    number_magnetization_fields: int
    J: float
    K: float
    D: float
    M: float
    B: float
    mu0: float
    coup_K: float
    coup_h: float
    coup_mu: float
    skyrmion_number: float
    skyrmion_rotation: float
    ansatz_bloch: bool
    ansatz_neel: bool
    ansatz_anti: bool
    ansatz_uniform: bool
    dmi_dresselhaus: bool
    dmi_rashba: bool
    dmi_heusler: bool
    dmi_hybrid: bool
    demag: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        core = CoreResolvedParams.core_fields(p)
        ans = (p.ansatz or "bloch").lower()
        denom = p.D * p.D
        if p.coup_K is None or p.coup_h is None or p.coup_mu is None:
            if denom != 0.0:
                coup_K = p.K * p.J / denom
                coup_h = p.M * p.B * p.J / denom
                coup_mu = p.mu0 * p.M * p.M * p.J / denom
            else:
                coup_K = coup_h = coup_mu = 1.0
        else:
            coup_K, coup_h, coup_mu = float(p.coup_K), float(p.coup_h), float(p.coup_mu)
        flags = {"dresselhaus": bool(p.dmi_dresselhaus), "rashba": bool(p.dmi_rashba),
                 "heusler": bool(p.dmi_heusler), "hybrid": bool(p.dmi_hybrid)}
        if p.dmi_term is not None:
            flags = dict.fromkeys(flags, False)
            items = [p.dmi_term] if isinstance(p.dmi_term, str) else list(p.dmi_term)
            for item in items:
                key = _DMI_NAMES.get(_norm(item))
                if key is None:
                    raise ValueError(f"Unknown DMI '{item}'. Valid: Dresselhaus (bulk), Rashba (interfacial), "
                                     "Heusler (B20), Hybrid")
                flags[key] = True
            if not any(flags.values()):
                raise ValueError("p.dmi_term was provided but no valid DMIs were selected.")
        return ResolvedParams(
            **core, number_magnetization_fields=int(p.number_magnetization_fields), J=float(p.J), K=float(p.K),
            D=float(p.D), M=float(p.M), B=float(p.B), mu0=float(p.mu0), coup_K=float(coup_K), coup_h=float(coup_h),
            coup_mu=float(coup_mu), skyrmion_number=float(p.skyrmion_number),
            skyrmion_rotation=float(p.skyrmion_rotation), ansatz_bloch=ans == "bloch", ansatz_neel=ans == "neel",
            ansatz_anti=ans == "anti", ansatz_uniform=ans == "uniform", dmi_dresselhaus=flags["dresselhaus"],
            dmi_rashba=flags["rashba"], dmi_heusler=flags["heusler"], dmi_hybrid=flags["hybrid"],
            demag=bool(p.demag))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    p_i, p_f = pack_core_device_params(rp)
    p_i_t = np.array([rp.number_magnetization_fields, rp.dmi_dresselhaus, rp.dmi_rashba, rp.dmi_heusler,
                      rp.dmi_hybrid, rp.demag], dtype=np.int32)
    p_f_t = np.array([rp.coup_K, rp.coup_h, rp.coup_mu, rp.skyrmion_number, rp.skyrmion_rotation,
                      float(rp.ansatz_bloch), float(rp.ansatz_neel), float(rp.ansatz_anti), float(rp.ansatz_uniform)],
                     dtype=np.float64)
    return np.concatenate((p_i, p_i_t)), np.concatenate((p_f, p_f_t))


def coupling_chain(rp: ResolvedParams) -> dict:
    """d(coup_*)/d(physical constant) at fixed reduced lattice, for coupling gradients.

    coup_K = K J/D^2, coup_h = M B J/D^2, coup_mu = mu0 M^2 J/D^2, so
    dcoup_h/dB = M J/D^2 and dcoup/dD = -2 coup/D for all three.  The reduced
    lattice (xsize in units of J/D) is held fixed, which is the convention of the
    reference's parameterisation.
    """
    D2 = rp.D * rp.D
    return {
        "B": {"coup_h": rp.M * rp.J / D2 if D2 else 0.0},
        "K": {"coup_K": rp.J / D2 if D2 else 0.0},
        "D": {"coup_K": -2.0 * rp.coup_K / rp.D, "coup_h": -2.0 * rp.coup_h / rp.D,
              "coup_mu": -2.0 * rp.coup_mu / rp.D} if rp.D else {},
    }


def describe() -> None:
    print("Field content: 3 magnetization components m1..m3 and the magnetostatic potential psi.")
    print("Couplings: J, K, D, M, B, mu0 -> coup_K, coup_h, coup_mu (override directly if given).")
    print("DMI: dmi_term in Dresselhaus (bulk), Rashba (interfacial), Heusler (B20), Hybrid.")
    print("demag: relax psi as a fourth flowed (saddle) field.")
