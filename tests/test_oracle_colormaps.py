"""Pin the colormap restatement to RGBA images the reference itself produced
(``tests/golden/make_golden_colormaps.py``): byte-exact."""
import glob
import os

import numpy as np
import pytest

from oracle import colormaps as oc

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "colormap_*.npz")))


def test_fixtures_present():
    assert len(GOLDEN) == 10


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[9:-4] for p in GOLDEN])
def test_oracle_matches_reference_images(path):
    g = np.load(path)
    kind, X, Y = str(g["kind"]), int(g["xlen"]), int(g["ylen"])
    if kind == "magnetization":
        img = oc.render_magnetization(g["field"], X, Y)
    else:
        img = oc.render_density(kind, g["density"], X, Y, float(g["vmin"]), float(g["vmax"]))
    np.testing.assert_array_equal(img, g["rgba"])
