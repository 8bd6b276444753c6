"""Baby Skyrme model theory package of the B200 backend (reference package:
soliton_solver/theories/baby_skyrme)."""
from __future__ import annotations

from soliton_solver_b200.theories.registry import TheorySpec

from . import params
from . import kernels
from . import initial_config
from . import observables
from . import io

THEORY_SPEC = TheorySpec(
    name='Baby Skyrme model',
    aliases=('Baby Skyrme', 'Baby skyrmion', 'Planar skyrmion'),
    import_path="soliton_solver_b200.theories.baby_skyrme",
    description='Skyrmions in a 2D planar Skyrme model, with numerous choices of potentials.',
    version='1.1',
)


def describe() -> None:
    print("=" * 72)
    print(f"{THEORY_SPEC.name} (version {THEORY_SPEC.version})")
    print("=" * 72)
    print(THEORY_SPEC.description)
    print("Aliases:", ", ".join(THEORY_SPEC.aliases))
    params.describe()
