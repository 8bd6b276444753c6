"""Host-side parity: parameter resolution/packing and the theory registry.

The golden fixtures hold the packed p_i/p_f arrays the reference built for the
keyword arguments listed in tests/golden/make_golden.py; our params modules must
produce the identical arrays for the same arguments.
"""
import importlib.util
import os

import numpy as np
import pytest

from soliton_solver_b200.theories import get_theory_spec, list_theories, load_theory

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)

CASES = [(f"hook_{n}", t, kw) for n, t, kw in make_golden._cases()] + \
        [(n, t, kw) for n, t, kw, _, _ in make_golden._traj_cases()]


@pytest.mark.parametrize("name,theory,kw", CASES, ids=[c[0] for c in CASES])
def test_packing_matches_reference(name, theory, kw):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    th = load_theory(make_golden.THEORY_NAMES[theory])
    rp = th.params.default_params(**kw).resolved()
    p_i, p_f = th.params.pack_device_params(rp)
    assert p_i.dtype == np.int32 and p_f.dtype == np.float64
    np.testing.assert_array_equal(p_i, g["p_i"])
    np.testing.assert_array_equal(p_f, g["p_f"])


def test_registry_names_and_aliases():
    assert set(list_theories()) == {"Chiral magnet", "Baby Skyrme model", "Ginzburg-Landau superconductor",
                                    "Anisotropic superconductor"}
    for alias, canon in [("abelian higgs", "Ginzburg-Landau superconductor"), ("  Baby Skyrme ", "Baby Skyrme model"),
                         ("s+id superconductor", "Anisotropic superconductor"), ("MAGNETIC SKYRMION", "Chiral magnet")]:
        assert get_theory_spec(alias).name == canon
    with pytest.raises(KeyError):
        get_theory_spec("no such theory")


def test_bad_selectors_raise():
    cm = load_theory("Chiral magnet")
    with pytest.raises(ValueError):
        cm.params.default_params(dmi_term="nope").resolved()
    bs = load_theory("Baby Skyrme")
    with pytest.raises(ValueError):
        bs.params.default_params(potential=["nope"]).resolved()


def test_derived_quantities():
    cm = load_theory("Chiral magnet")
    rp = cm.params.default_params(xlen=320, ylen=320, xsize=10.0, ysize=10.0, dmi_term="Heusler").resolved()
    assert rp.lsx == 10.0 / 319 and rp.time_step == 0.5 * rp.lsx
    assert rp.coup_K == 0.8e6 * 40e-12 / (4e-3) ** 2
    assert rp.dmi_heusler and not rp.dmi_dresselhaus
