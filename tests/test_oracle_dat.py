"""Pin the .dat restatement to files the reference's writers produced
(``tests/golden/make_golden_dat.py``): byte-identical."""
import os

import numpy as np
import pytest

from oracle import io as oio

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("p", [32, 16, 8])
def test_oracle_matches_reference_files(p):
    g = np.load(os.path.join(GOLDEN, "dat_values.npz"))
    X, Y, nf = int(g["xlen"]), int(g["ylen"]), int(g["nf"])
    read = lambda name: open(os.path.join(GOLDEN, "dat", name), "rb").read()  # noqa: E731
    assert oio.field_text(g["field"], X, Y, nf, p) == read(f"field_p{p}.dat")
    assert oio.density_text(g["density"], 1, X, Y, p) == read(f"density1_p{p}.dat")
    assert oio.iteration_text(g["iters"], p) == read(f"iters_p{p}.dat")
