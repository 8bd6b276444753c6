"""Chiral magnet theory package of the B200 backend (reference package:
soliton_solver/theories/chiral_magnet)."""
from __future__ import annotations

from soliton_solver_b200.theories.registry import TheorySpec

from . import params
from . import kernels
from . import initial_config
from . import observables
from . import io

THEORY_SPEC = TheorySpec(
    name='Chiral magnet',
    aliases=('Chiral ferromagnet', 'Chiral magnetic skyrmion', 'Magnetic skyrmion'),
    import_path="soliton_solver_b200.theories.chiral_magnet",
    description='Skyrmions in chiral ferromagnetic systems, with various DMI choices and optional demagnetization.',
    version='1.1',
)


def describe() -> None:
    print("=" * 72)
    print(f"{THEORY_SPEC.name} (version {THEORY_SPEC.version})")
    print("=" * 72)
    print(THEORY_SPEC.description)
    print("Aliases:", ", ".join(THEORY_SPEC.aliases))
    params.describe()
