"""Anisotropic superconductor theory package of the B200 backend (reference package:
soliton_solver/theories/anisotropic_superconductor)."""
from __future__ import annotations

from soliton_solver_b200.theories.registry import TheorySpec

from . import params
from . import kernels
from . import initial_config
from . import observables
from . import io

THEORY_SPEC = TheorySpec(
    name='Anisotropic superconductor',
    aliases=('s+id superconductor', 'Multicomponent superconductor', 'Multi-component superconductor', 'Multicomponent GL', 'Multi-component GL', 'Multicomponent Ginzburg-Landau', 'Multi-component Ginzburg-Landau'),
    import_path="soliton_solver_b200.theories.anisotropic_superconductor",
    description='Multi-component anisotropic s+id superconductor, simulating multi-component vortices.',
    version='1.0',
)


def describe() -> None:
    print("=" * 72)
    print(f"{THEORY_SPEC.name} (version {THEORY_SPEC.version})")
    print("=" * 72)
    print(THEORY_SPEC.description)
    print("Aliases:", ", ".join(THEORY_SPEC.aliases))
    params.describe()
