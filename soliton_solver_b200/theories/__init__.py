"""Theory plugins of the B200 backend and the public registry surface
(same names as soliton_solver/theories/__init__.py)."""
from __future__ import annotations

from .registry import (TheorySpec, describe_theory, discover_theories, get_theory_spec, list_theories,
                       load_theory, print_theory_table, register_theory)

__all__ = ["TheorySpec", "register_theory", "discover_theories", "load_theory", "list_theories",
           "get_theory_spec", "describe_theory", "print_theory_table", "list", "print_description",
           "print_table"]

discover_theories()


def list() -> tuple[str, ...]:  # noqa: A001 - same name as the reference's helper
    return list_theories()


def print_description(name: str) -> None:
    describe_theory(name)


def print_table() -> None:
    print_theory_table()
