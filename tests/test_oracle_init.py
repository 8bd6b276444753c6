"""Pin the initial-condition restatement (oracle/init.py) to the outputs of the
reference's own initial-condition kernels (``tests/golden/make_golden_init.py``):
1e-13 relative to the largest magnitude (libm ulps of sin/cos/exp/atan2/tanh)."""
import glob
import os

import numpy as np
import pytest

from oracle import init as oi

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "init_*.npz")))


def ansatz_of(g):
    if "ansatz" not in g:
        return oi.ANSATZ_NONE
    b, n, a = (int(v) for v in g["ansatz"])
    return oi.ANSATZ_BLOCH if b else oi.ANSATZ_NEEL if n else oi.ANSATZ_ANTI if a else oi.ANSATZ_NONE


def oracle_field(g):
    th, p_i, p_f = str(g["theory"]), g["p_i"], g["p_f"]
    X, Y, nf = int(p_i[0]), int(p_i[1]), int(p_i[4])
    mode = int(g["mode"])
    rot = float(g["rotation"]) if "rotation" in g else 0.0
    if mode == 0:
        return oi.ground(th, p_i, p_f)
    if mode == 1:
        return oi.initial(th, p_i, p_f, ansatz_of(g), rot, float(g["vortex_number"]) if "vortex_number" in g else 1.0)
    return oi.insert(th, g["before"].reshape(nf, X, Y), p_i, p_f, int(g["pxi"]), int(g["pxj"]), ansatz_of(g), rot,
                     bool(g["vortex"]) if "vortex" in g else True)


def test_fixtures_present():
    assert len(GOLDEN) == 22


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[5:-4] for p in GOLDEN])
def test_oracle_matches_reference_kernels(path):
    g = np.load(path)
    F = oracle_field(g).reshape(-1)
    want = g["field"]
    assert np.max(np.abs(F - want)) <= 1e-13 * max(1.0, np.max(np.abs(want)))
    if g["velocity"].size:
        assert np.all(g["velocity"] == 0.0)
