"""Theory registry: names, aliases, discovery and loading.

Same public surface as the reference's registry
(soliton_solver/theories/registry.py:21-329): ``TheorySpec``, ``register_theory``,
``list_theories``, ``get_theory_spec``, ``load_theory``, ``describe_theory``,
``print_theory_table``, ``discover_theories``.  Keys are case-insensitive.
"""
from __future__ import annotations

import importlib
import pkgutil
import warnings
from dataclasses import dataclass
from types import ModuleType
from typing import Dict


@dataclass(frozen=True)
class TheorySpec:
    name: str
    import_path: str
    description: str = ""
    version: str = "0.0"
    aliases: tuple[str, ...] = ()
    required_submodules: tuple[str, ...] = ("kernels", "initial_config", "observables")


_REGISTRY: Dict[str, TheorySpec] = {}


def _key(name) -> str:
    return (name or "").strip().lower()


def register_theory(spec: TheorySpec) -> None:
    """Register a spec under its name and aliases; duplicates raise ValueError."""
    for k in (spec.name, *spec.aliases):
        key = _key(k)
        if not key:
            raise ValueError("TheorySpec names must be non-empty")
        if key in _REGISTRY:
            raise ValueError(f"Theory '{key}' is already registered")
        _REGISTRY[key] = spec


def list_theories() -> tuple[str, ...]:
    return tuple(sorted({s.name for s in _REGISTRY.values()}))


def get_theory_spec(name: str) -> TheorySpec:
    key = _key(name)
    if key not in _REGISTRY:
        raise KeyError(f"Unknown theory '{name}'. Available: {list_theories()}")
    return _REGISTRY[key]


def load_theory(name: str) -> ModuleType:
    """Import and return the theory package registered under ``name`` (or an alias)."""
    spec = get_theory_spec(name)
    mod = importlib.import_module(spec.import_path)
    for sub in spec.required_submodules:
        importlib.import_module(f"{spec.import_path}.{sub}")
    return mod


def describe_theory(name: str) -> None:
    spec = get_theory_spec(name)
    print(f"Theory: {spec.name}")
    print(f"Import path: {spec.import_path}")
    print(f"Version: {spec.version}")
    if spec.aliases:
        print("Aliases:", ", ".join(spec.aliases))
    if spec.description:
        print(f"Description: {spec.description}")


def print_theory_table() -> None:
    specs = sorted(set(_REGISTRY.values()), key=lambda s: s.name.lower())
    if not specs:
        print("No theories registered.")
        return
    w1 = max(len("Theory"), *(len(s.name) for s in specs))
    w2 = max(len("Version"), *(len(s.version) for s in specs))
    print(f"{'Theory':<{w1}}  {'Version':<{w2}}  Description")
    print("-" * (w1 + w2 + 16))
    for s in specs:
        print(f"{s.name:<{w1}}  {s.version:<{w2}}  {s.description}")


def discover_theories(package: str = "soliton_solver_b200.theories") -> None:
    """Import every theory subpackage and register its THEORY_SPEC.

    A subpackage that fails to import is skipped with a warning (the reference
    skips silently, registry.py:313-316)."""
    pkg = importlib.import_module(package)
    for m in pkgutil.iter_modules(pkg.__path__):
        if not m.ispkg or m.name == "__pycache__":
            continue
        path = f"{package}.{m.name}"
        try:
            sub = importlib.import_module(path)
        except Exception as exc:  # pragma: no cover - only on a broken install
            warnings.warn(f"theory package {path} failed to import: {exc}")
            continue
        spec = getattr(sub, "THEORY_SPEC", None)
        if isinstance(spec, TheorySpec):
            for k in (spec.name, *spec.aliases):
                key = _key(k)
                if key and key not in _REGISTRY:
                    _REGISTRY[key] = spec
