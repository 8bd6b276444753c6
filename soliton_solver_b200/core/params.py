"""Theory-agnostic lattice parameters.

Mirrors the reference's parameter interface (soliton_solver/core/params.py:16-249):
the same dataclass fields, the same derived quantities (``lsx = xsize/(xlen-1)``
unless given, ``time_step = courant*lsx`` unless given) and the same packed
``p_i`` (int32) / ``p_f`` (float64) arrays, which are the C ABI's parameter format.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

# slots of the packed core arrays (soliton_solver/core/params.py:229-249)
CORE_P_I = ("xlen", "ylen", "halo", "number_coordinates", "number_total_fields", "dim_grid", "dim_fields",
            "killkinen", "newtonflow", "unit_magnetization")
CORE_P_F = ("xsize", "ysize", "lsx", "lsy", "grid_volume", "time_step")


@dataclass(frozen=True)
class Params:
    """User-facing lattice parameters shared by all theories."""

    xlen: int = 256
    ylen: int = 256
    halo: int = 2
    number_coordinates: int = 2
    number_total_fields: int = 0
    xsize: float = 80.0
    ysize: float = 80.0
    lsx: float | None = None
    lsy: float | None = None
    courant: float = 0.5
    time_step: float | None = None
    killkinen: bool = True
    newtonflow: bool = True
    unit_magnetization: bool = False

    def with_(self, **kwargs) -> "Params":
        """Copy with some fields replaced."""
        return replace(self, **kwargs)

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams:
    """Parameters with every derived quantity filled in."""

    xlen: int
    ylen: int
    halo: int
    number_coordinates: int
    number_total_fields: int
    dim_grid: int
    dim_fields: int
    killkinen: int
    newtonflow: int
    unit_magnetization: int
    xsize: float
    ysize: float
    lsx: float
    lsy: float
    grid_volume: float
    time_step: float

    @staticmethod
    def core_fields(p: Params) -> dict:
        lsx = p.lsx if p.lsx is not None else p.xsize / (p.xlen - 1)
        lsy = p.lsy if p.lsy is not None else p.ysize / (p.ylen - 1)
        time_step = p.time_step if p.time_step is not None else p.courant * lsx
        dim_grid = int(p.xlen) * int(p.ylen)
        return dict(xlen=int(p.xlen), ylen=int(p.ylen), halo=int(p.halo), number_coordinates=int(p.number_coordinates),
                    number_total_fields=int(p.number_total_fields), dim_grid=dim_grid,
                    dim_fields=int(p.number_total_fields) * dim_grid, killkinen=int(bool(p.killkinen)),
                    newtonflow=int(bool(p.newtonflow)), unit_magnetization=int(bool(p.unit_magnetization)),
                    xsize=float(p.xsize), ysize=float(p.ysize), lsx=float(lsx), lsy=float(lsy),
                    grid_volume=float(lsx) * float(lsy), time_step=float(time_step))

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        return ResolvedParams(**ResolvedParams.core_fields(p))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    """The core slots of the packed arrays: ``p_i`` int32[10] and ``p_f`` float64[6]."""
    p_i = np.array([getattr(rp, k) for k in CORE_P_I], dtype=np.int32)
    p_f = np.array([getattr(rp, k) for k in CORE_P_F], dtype=np.float64)
    return p_i, p_f
