import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "kaust-hierarchical-matrices_b200")
for p in (PKG, os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def golden_cases():
    import glob

    import numpy as np

    out = {}
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        g = np.load(f)
        out[os.path.basename(f)[:-4]] = {k: g[k] for k in g.files}
    return out


def ref_lists(g):
    """Split a golden case's concatenated Morton lists per level."""
    depth = int(g["depth"])
    nt = g["num_tiles"]
    tiles = g["tiles"]
    out, o = [], 0
    for lv in range(depth):
        out.append(tiles[o : o + nt[lv]])
        o += nt[lv]
    return out
