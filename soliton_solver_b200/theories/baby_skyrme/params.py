"""Baby Skyrme model parameters.

Same fields, potential selection and packed layout as the reference
(soliton_solver/theories/baby_skyrme/params.py:25-378): ``p_i = core + [nmag,
Standard, Holomorphic, EasyPlane, Dihedral2, Aloof, Dihedral3, Broken,
DoubleVacua, N]``; ``p_f = core + [mpi, kappa, skyrmion_number,
skyrmion_rotation, bloch, neel, anti, uniform]``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable

import numpy as np

from soliton_solver_b200.core.params import Params as CoreParams
from soliton_solver_b200.core.params import ResolvedParams as CoreResolvedParams
from soliton_solver_b200.core.params import pack_device_params as pack_core_device_params

POTENTIALS = ("Standard", "Holomorphic", "EasyPlane", "Dihedral2", "Aloof", "Dihedral3", "Broken", "DoubleVacua")
_ALIASES = {
    "standard": "Standard", "holomorphic": "Holomorphic", "holomorhpic": "Holomorphic",
    "easy plane": "EasyPlane", "easyplane": "EasyPlane", "dihedral2": "Dihedral2", "dihedral 2": "Dihedral2",
    "aloof": "Aloof", "dihedral3": "Dihedral3", "dihedral 3": "Dihedral3", "broken": "Broken",
    "double vacua": "DoubleVacua", "doublevacua": "DoubleVacua", "2 vacua": "DoubleVacua", "two vacua": "DoubleVacua",
}


def _norm(s) -> str:
    return (str(s) or "").strip().lower().replace("_", " ").replace("-", " ")


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 3
    number_magnetization_fields: int = 3
    mpi: float = 1.0
    kappa: float = 1.0
    N: int = 1
    Potential_Standard: bool = True
    Potential_Holomorphic: bool = False
    Potential_EasyPlane: bool = False
    Potential_Dihedral2: bool = False
    Potential_Aloof: bool = False
    Potential_Dihedral3: bool = False
    Potential_Broken: bool = False
    Potential_DoubleVacua: bool = False
    potential: str | Iterable[str] | None = None
    skyrmion_number: float = 1.0
    skyrmion_rotation: float = 0.0
    ansatz: str = "bloch"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    number_magnetization_fields: int
    N: int
    mpi: float
    kappa: float
    skyrmion_number: float
    skyrmion_rotation: float
    ansatz_bloch: bool
    ansatz_neel: bool
    ansatz_anti: bool
    ansatz_uniform: bool
    Potential_Standard: bool
    Potential_Holomorphic: bool
    Potential_EasyPlane: bool
    Potential_Dihedral2: bool
    Potential_Aloof: bool
    Potential_Dihedral3: bool
    Potential_Broken: bool
    Potential_DoubleVacua: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        core = CoreResolvedParams.core_fields(p)
        ans = (p.ansatz or "bloch").lower()
        flags = {name: bool(getattr(p, "Potential_" + name)) for name in POTENTIALS}
        if p.potential is not None:
            flags = dict.fromkeys(flags, False)
            items = [p.potential] if isinstance(p.potential, str) else list(p.potential)
            for item in items:
                key = _ALIASES.get(_norm(item))
                if key is None:
                    raise ValueError(f"Unknown potential '{item}'. Valid: Standard, Holomorphic, Easy plane, "
                                     "Dihedral2, Aloof, Dihedral3, Broken, DoubleVacua")
                flags[key] = True
            if not any(flags.values()):
                raise ValueError("p.potential was provided but no valid potentials were selected.")
        return ResolvedParams(
            **core, number_magnetization_fields=int(p.number_magnetization_fields), N=int(p.N), mpi=float(p.mpi),
            kappa=float(p.kappa), skyrmion_number=float(p.skyrmion_number),
            skyrmion_rotation=float(p.skyrmion_rotation), ansatz_bloch=ans == "bloch", ansatz_neel=ans == "neel",
            ansatz_anti=ans == "anti", ansatz_uniform=ans == "uniform",
            **{"Potential_" + k: v for k, v in flags.items()})


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    p_i, p_f = pack_core_device_params(rp)
    p_i_t = np.array([rp.number_magnetization_fields] + [int(getattr(rp, "Potential_" + k)) for k in POTENTIALS]
                     + [int(rp.N)], dtype=np.int32)
    p_f_t = np.array([rp.mpi, rp.kappa, rp.skyrmion_number, rp.skyrmion_rotation, float(rp.ansatz_bloch),
                      float(rp.ansatz_neel), float(rp.ansatz_anti), float(rp.ansatz_uniform)], dtype=np.float64)
    return np.concatenate((p_i, p_i_t)), np.concatenate((p_f, p_f_t))


def describe() -> None:
    print("Field content: 3 components of the unit vector m.")
    print("Couplings: mpi (potential strength), kappa (Skyrme term), N (broken potential).")
    print("Potentials: " + ", ".join(POTENTIALS) + " (select with potential=...).")
