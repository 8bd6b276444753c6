"""Anisotropic s+id superconductor parameters.

Same fields, derived ground-state quantities and packed layout as the reference
(soliton_solver/theories/anisotropic_superconductor/params.py:23-310):
``beta4 = beta3/4`` unless given; ``theta_diff = pi/2`` if beta4 >= 0 else 0;
``beta3tilde = beta3 + 2 cos(2 theta_diff) beta4``; u1, u2 from the quadratic
minimisation; ``p_i = core + [nmag, nhiggs, ngauge, vortex_type]``;
``p_f = core + [kappa, Q, alpha1, alpha2, beta1..beta4, gamma1, gamma2, gamma12,
u1, u2, theta_diff, beta3tilde, vortex_number, ainf, N1, N2]``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from soliton_solver_b200.core.params import Params as CoreParams
from soliton_solver_b200.core.params import ResolvedParams as CoreResolvedParams
from soliton_solver_b200.core.params import pack_device_params as pack_core_device_params


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 6
    number_magnetization_fields: int = 0
    number_higgs_fields: int = 4
    number_gauge_fields: int = 2
    vortex_type: int = 0
    N1: float = 1.0
    N2: float = 1.0
    alpha1: float = -1.0
    alpha2: float = -1.24503
    beta1: float = 1.0
    beta2: float = 1.4959
    beta3: float = 4.02498
    beta4: float | None = None
    Q: float = 1.0
    kappa: float = 0.673274
    gamma1: float = 1.0
    gamma2: float = 0.877868
    gamma12: float = 0.534484
    theta_diff: float = math.pi / 2.0
    beta3tilde: float | None = None
    u1: float | None = None
    u2: float | None = None
    vortex_number: float | None = None
    ainf: float | None = None

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    number_magnetization_fields: int
    number_higgs_fields: int
    number_gauge_fields: int
    vortex_type: int
    N1: float
    N2: float
    alpha1: float
    alpha2: float
    beta1: float
    beta2: float
    beta3: float
    beta4: float
    Q: float
    kappa: float
    gamma1: float
    gamma2: float
    gamma12: float
    theta_diff: float
    beta3tilde: float
    u1: float
    u2: float
    vortex_number: float
    ainf: float

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        core = CoreResolvedParams.core_fields(p)
        beta4 = float(p.beta4) if p.beta4 is not None else float(p.beta3) / 4.0
        theta_diff = math.pi / 2.0 if beta4 >= 0.0 else 0.0
        beta3tilde = (float(p.beta3tilde) if p.beta3tilde is not None
                      else float(p.beta3 + 2.0 * math.cos(2.0 * theta_diff) * beta4))
        if p.u1 is None or p.u2 is None:
            denom = beta3tilde * beta3tilde - 4.0 * p.beta1 * p.beta2
            num1 = 2.0 * p.beta2 * p.alpha1 - beta3tilde * p.alpha2
            num2 = 2.0 * p.beta1 * p.alpha2 - beta3tilde * p.alpha1
            u1 = math.sqrt(num1 / denom) if denom != 0.0 and num1 / denom > 0.0 else 0.0
            u2 = math.sqrt(num2 / denom) if denom != 0.0 and num2 / denom > 0.0 else 0.0
        else:
            u1, u2 = float(p.u1), float(p.u2)
        if p.vortex_number is None:
            dv = u1 * u1 + u2 * u2
            vortex_number = (u1 * u1 * p.N1 + u2 * u2 * p.N2) / dv if dv != 0.0 else 0.0
        else:
            vortex_number = float(p.vortex_number)
        if p.ainf is None:
            ainf = -vortex_number / p.Q if p.Q != 0.0 else 0.0
        else:
            ainf = float(p.ainf)
        return ResolvedParams(
            **core, number_magnetization_fields=int(p.number_magnetization_fields),
            number_higgs_fields=int(p.number_higgs_fields), number_gauge_fields=int(p.number_gauge_fields),
            vortex_type=int(p.vortex_type), N1=float(p.N1), N2=float(p.N2), alpha1=float(p.alpha1),
            alpha2=float(p.alpha2), beta1=float(p.beta1), beta2=float(p.beta2), beta3=float(p.beta3),
            beta4=float(beta4), Q=float(p.Q), kappa=float(p.kappa), gamma1=float(p.gamma1), gamma2=float(p.gamma2),
            gamma12=float(p.gamma12), theta_diff=float(theta_diff), beta3tilde=float(beta3tilde), u1=float(u1),
            u2=float(u2), vortex_number=float(vortex_number), ainf=float(ainf))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    p_i, p_f = pack_core_device_params(rp)
    p_i_t = np.array([rp.number_magnetization_fields, rp.number_higgs_fields, rp.number_gauge_fields,
                      rp.vortex_type], dtype=np.int32)
    p_f_t = np.array([rp.kappa, rp.Q, rp.alpha1, rp.alpha2, rp.beta1, rp.beta2, rp.beta3, rp.beta4, rp.gamma1,
                      rp.gamma2, rp.gamma12, rp.u1, rp.u2, rp.theta_diff, rp.beta3tilde, rp.vortex_number, rp.ainf,
                      rp.N1, rp.N2], dtype=np.float64)
    return np.concatenate((p_i, p_i_t)), np.concatenate((p_f, p_f_t))


def describe() -> None:
    print("Field content: gauge field (A1, A2), condensates psi1 = (2, 3) and psi2 = (4, 5).")
    print("Couplings: alpha1/2, beta1..beta4, Q, kappa, anisotropy gamma1, gamma2, gamma12.")
