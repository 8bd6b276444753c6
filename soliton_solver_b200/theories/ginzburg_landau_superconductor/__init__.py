"""Ginzburg-Landau superconductor theory package of the B200 backend (reference package:
soliton_solver/theories/ginzburg_landau_superconductor)."""
from __future__ import annotations

from soliton_solver_b200.theories.registry import TheorySpec

from . import params
from . import kernels
from . import initial_config
from . import observables
from . import io

THEORY_SPEC = TheorySpec(
    name='Ginzburg-Landau superconductor',
    aliases=('Abelian Higgs', 'Ginzburg-Landau', 'Abelian Higgs model', 'Ginzburg-Landau model'),
    import_path="soliton_solver_b200.theories.ginzburg_landau_superconductor",
    description='Superconducting vortices in the Ginzburg-Landau or Abelian Higgs model.',
    version='1.0',
)


def describe() -> None:
    print("=" * 72)
    print(f"{THEORY_SPEC.name} (version {THEORY_SPEC.version})")
    print("=" * 72)
    print(THEORY_SPEC.description)
    print("Aliases:", ", ".join(THEORY_SPEC.aliases))
    params.describe()
