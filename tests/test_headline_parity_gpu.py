"""Bit-exact parity of the device KD tree and block structure at the
benchmark's sizes.

tests/golden/headline_hashes.json holds SHA-256 digests of the reference's own
compiled pipeline (generateDataset -> constructKDTree ->
constructHMatrixStructure, run by tests/golden/make_headline_hashes.py) on the
precision workload's 2^20 points, the scale workload's 2^21 mixture points and
a non-power-of-two cloud.  The device tree's permutation, leaf offsets and
boxes, and every level's Morton block list, must hash to the same digests.
The scale workload itself uses eta = 1.5, which the reference cannot express
(it fixes 1.0, src/HMatrixStructure.cu:7); its block lists are compared with
the CPU oracle's (pinned to the reference's outputs on the golden cases).
"""
import json
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

HASHES = os.path.join(GOLDEN, "headline_hashes.json")


@pytest.fixture(scope="module")
def hm():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(HASHES):
        pytest.skip("headline digests not generated")
    import hmatrix

    return hmatrix


def _cases():
    if not os.path.exists(HASHES):
        return []
    return sorted(json.load(open(HASHES)).items())


def _points(hm, c):
    n, d = c["N"], c["d"]
    if c["points_source"] == "gen":
        return hm.generate_dataset(n, d, seed=1234)
    return hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=1234)


@pytest.mark.parametrize("name,case", _cases())
def test_tree_and_structure_digests(hm, name, case):
    if GOLDEN not in sys.path:
        sys.path.insert(0, GOLDEN)
    from make_headline_hashes import digests

    n, d, b = case["N"], case["d"], case["bucket"]
    pts = _points(hm, case)
    tree = hm.construct_kdtree(pts, n, d, b)
    assert tree.depth == case["depth"]
    st = hm.construct_hmatrix_structure(tree, case["admiss"], 1.0)
    t = tree.copy_out()
    nb = ((1 << tree.depth) - 1) * d  # levels 0..depth-1
    mine = digests(pts.cpu().numpy(), t["perm"], t["offsets"], t["bmin"][:nb], t["bmax"][:nb], st.all_tiles())
    for key in ("points", "perm", "offsets", "bmin", "bmax", "counts", "tiles"):
        assert mine[key] == case[key], "%s: %s differs from the reference's" % (name, key)


def test_scale_workload_structure_at_eta_1_5(hm):
    """The scale workload's eta = 1.5 block lists against the CPU oracle, on
    the oracle's own tree of the same 2^21 points."""
    import oracle

    n, d, b = 1 << 21, 3, 64
    pts = hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=1234)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.5)
    ref = oracle.kdtree(pts.cpu().numpy(), n, d, b)
    t = tree.copy_out()
    assert np.array_equal(t["perm"], ref["perm"])
    lists = oracle.structure(d, ref["depth"], 1, 1.5, ref["bmin"], ref["bmax"], cap=int(st.counts.max()) + 1)
    for lv, r in enumerate(lists, start=1):
        assert np.array_equal(st.tiles(lv), r), "level %d" % lv
