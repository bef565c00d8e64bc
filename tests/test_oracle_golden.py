"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's compiled KD-tree and structure
code).  Runs on CPU."""
import numpy as np
import pytest

import oracle
from conftest import ref_lists

CASES = ["c1_box", "c1_weak", "n1000_d3", "n5000_d3_b64", "n20_single_leaf", "d1_n777",
         "lattice_ties", "mixture_d3"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_kdtree_matches_reference(golden_cases, name):
    g = golden_cases[name]
    n, d, b = int(g["N"]), int(g["d"]), int(g["bucket"])
    t = oracle.kdtree(g["points"], n, d, b)
    assert t["depth"] == int(g["depth"])
    np.testing.assert_array_equal(t["perm"], g["perm"])
    np.testing.assert_array_equal(t["offsets"], g["offsets"])
    nb = ((1 << t["depth"]) - 1) * d
    np.testing.assert_array_equal(t["bmin"][:nb], g["bmin"])
    np.testing.assert_array_equal(t["bmax"][:nb], g["bmax"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_structure_matches_reference(golden_cases, name):
    g = golden_cases[name]
    d, depth = int(g["d"]), int(g["depth"])
    # the structure from the reference's own boxes
    nodes = (1 << depth) - 1
    bmin = np.concatenate([g["bmin"], np.zeros((nodes + 1) * d)])
    bmax = np.concatenate([g["bmax"], np.zeros((nodes + 1) * d)])
    lists = oracle.structure(d, depth, int(g["admiss"]), 1.0, bmin, bmax)
    ref = ref_lists(g)
    assert len(lists) == len(ref)
    for lv, (a, r) in enumerate(zip(lists, ref)):
        np.testing.assert_array_equal(a, r, err_msg="level %d" % (lv + 1))


def test_golden_points_are_reference_uniforms(golden_cases):
    g = golden_cases["c1_box"]
    p = g["points"]
    assert p.shape == (8192 * 2,)
    assert (p > 0).all() and (p <= 1).all()
    # curand_uniform returns floats: every value is exactly representable in FP32
    assert np.array_equal(p, p.astype(np.float32).astype(np.float64))


def test_weak_structure_is_the_off_diagonal_pairs(golden_cases):
    # weak admissibility: at each level l the two off-diagonal children of every
    # diagonal block of level l-1 (src/admissibilityCondition.cu:54-68)
    g = golden_cases["c1_weak"]
    for lv, lst in enumerate(ref_lists(g), start=1):
        exp = []
        for p in range(1 << (lv - 1)):
            exp.append(oracle.morton(2 * p + 1, 2 * p))
            exp.append(oracle.morton(2 * p, 2 * p + 1))
        np.testing.assert_array_equal(np.sort(lst), np.array(sorted(exp), np.int32))


def test_structure_partitions_the_matrix(golden_cases):
    """Blocks of all levels plus the dense diagonal leaves tile the matrix."""
    g = golden_cases["n5000_d3_b64"]
    depth = int(g["depth"])
    nleaf = 1 << depth
    cover = np.zeros((nleaf, nleaf), np.int32)
    for lv, lst in enumerate(ref_lists(g), start=1):
        span = 1 << (depth - lv)
        for z in lst:
            u = sum(((int(z) >> (2 * b)) & 1) << b for b in range(16))
            v = sum(((int(z) >> (2 * b + 1)) & 1) << b for b in range(16))
            cover[v * span:(v + 1) * span, u * span:(u + 1) * span] += 1
    cover[np.arange(nleaf), np.arange(nleaf)] += 1
    assert (cover == 1).all()


def test_tree_depth_and_offsets_are_ceil_halvings():
    for n, b in [(8192, 32), (1000, 32), (777, 16), (20, 32), (2 ** 20, 64), (3 * 2 ** 19 + 5, 64)]:
        depth = oracle.tree_depth(n, b)
        sizes = [n]
        for _ in range(depth):
            sizes = [x for s in sizes for x in ((s + 1) // 2, s // 2)]
        assert max(sizes) <= b
        assert len(sizes) == 1 << depth
