"""Point generation, KD tree and block structure on the GPU, through the C ABI,
bit for bit against the reference's own outputs (golden fixtures) and against
the pinned CPU oracle at larger sizes."""
import numpy as np
import pytest

import oracle
from conftest import ref_lists

pytestmark = pytest.mark.gpu

GOLDEN = ["c1_box", "c1_weak", "n1000_d3", "n5000_d3_b64", "n20_single_leaf", "d1_n777",
          "lattice_ties", "mixture_d3"]


@pytest.fixture(scope="module")
def hm():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hmatrix

    return hmatrix


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("name", [c for c in GOLDEN])
def test_generate_dataset_matches_reference(hm, golden_cases, name):
    g = golden_cases[name]
    if str(g["source"]) != "gen":
        pytest.skip("points not from generateDataset")
    n, d = int(g["N"]), int(g["d"])
    pts = hm.generate_dataset(n, d, seed=1234).cpu().numpy()
    np.testing.assert_array_equal(pts, g["points"])


@pytest.mark.parametrize("name", GOLDEN)
def test_kdtree_and_structure_match_reference(hm, golden_cases, name):
    g = golden_cases[name]
    n, d, b = int(g["N"]), int(g["d"]), int(g["bucket"])
    pts = to_dev(g["points"])
    tree = hm.construct_kdtree(pts, n, d, b)
    assert tree.depth == int(g["depth"])
    t = tree.copy_out()
    np.testing.assert_array_equal(t["perm"], g["perm"])
    np.testing.assert_array_equal(t["offsets"], g["offsets"])
    nb = ((1 << tree.depth) - 1) * d
    np.testing.assert_array_equal(t["bmin"][:nb], g["bmin"])
    np.testing.assert_array_equal(t["bmax"][:nb], g["bmax"])
    st = hm.construct_hmatrix_structure(tree, int(g["admiss"]), 1.0)
    for lv, r in enumerate(ref_lists(g), start=1):
        np.testing.assert_array_equal(st.tiles(lv), r, err_msg="level %d" % lv)


def lattice(n, d, seed, levels=8):
    rng = np.random.default_rng(seed)
    return rng.integers(0, levels, size=(d, n)).astype(np.float64) / levels


def mixture(n, d, seed, k=16):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (k, d))
    s = np.exp(rng.uniform(np.log(0.01), np.log(0.1), k))
    w = rng.dirichlet(np.ones(k))
    comp = rng.choice(k, size=n, p=w)
    return np.ascontiguousarray((c[comp] + s[comp, None] * rng.standard_normal((n, d))).T)


# sizes that use the wide (radix-select) levels as well as the local levels
CASES = [
    ("uniform", 65536, 3, 64, 1),
    ("uniform", 100003, 3, 32, 1),
    ("uniform", 70000, 2, 16, 0),
    ("lattice", 50000, 3, 16, 1),
    ("lattice", 6000, 2, 8, 1),
    ("lattice_fine", 40000, 2, 8, 1),
    ("mixture", 131072, 3, 64, 1),
    ("uniform", 30000, 5, 32, 1),
    ("uniform", 9000, 1, 8, 1),
]


@pytest.mark.parametrize("kind,n,d,b,adm", CASES)
def test_kdtree_and_structure_match_oracle_large(hm, kind, n, d, b, adm):
    if kind == "uniform":
        pts = hm.generate_dataset(n, d, seed=99).cpu().numpy()
    elif kind == "lattice":
        pts = lattice(n, d, seed=n).reshape(-1)
    elif kind == "lattice_fine":
        pts = lattice(n, d, seed=n, levels=1024).reshape(-1)
    else:
        pts = mixture(n, d, seed=n).reshape(-1)
    ref = oracle.kdtree(pts, n, d, b)
    tree = hm.construct_kdtree(to_dev(pts), n, d, b)
    t = tree.copy_out()
    np.testing.assert_array_equal(t["perm"], ref["perm"])
    np.testing.assert_array_equal(t["offsets"], ref["offsets"])
    np.testing.assert_array_equal(t["bmin"], ref["bmin"])
    np.testing.assert_array_equal(t["bmax"], ref["bmax"])
    np.testing.assert_array_equal(t["split_dim"], ref["split_dim"])
    st = hm.construct_hmatrix_structure(tree, adm, 1.0)
    lists = oracle.structure(d, ref["depth"], adm, 1.0, ref["bmin"], ref["bmax"], cap=4_000_000)
    for lv, r in enumerate(lists, start=1):
        np.testing.assert_array_equal(st.tiles(lv), r, err_msg="level %d" % lv)


def test_structure_eta_parameter(hm):
    n, d, b = 20000, 3, 32
    pts = hm.generate_dataset(n, d, seed=5).cpu().numpy()
    ref = oracle.kdtree(pts, n, d, b)
    tree = hm.construct_kdtree(to_dev(pts), n, d, b)
    for eta in (0.5, 1.5, 2.0):
        st = hm.construct_hmatrix_structure(tree, 1, eta)
        lists = oracle.structure(d, ref["depth"], 1, eta, ref["bmin"], ref["bmax"], cap=4_000_000)
        for lv, r in enumerate(lists, start=1):
            np.testing.assert_array_equal(st.tiles(lv), r)


def test_jds_layout_consistent(hm):
    n, d, b = 40000, 3, 32
    pts = hm.generate_dataset(n, d, seed=3)
    tree = hm.construct_kdtree(pts, n, d, b)
    st = hm.construct_hmatrix_structure(tree, 1, 1.0)
    for lv in range(1, st.depth + 1):
        tiles = st.tiles(lv)
        j = st.jds(lv)
        nrows = 1 << lv
        u = np.array([oracle_compact(z) for z in tiles], np.int64)
        v = np.array([oracle_compact(z >> 1) for z in tiles], np.int64)
        cnt = np.bincount(v, minlength=nrows)
        np.testing.assert_array_equal(np.diff(j["row_ptr"]), cnt)
        # CSR: grouped by row, increasing column inside a row
        order = np.lexsort((u, v))
        np.testing.assert_array_equal(j["csr_blk"], order)
        # JDS: rows by decreasing count (stable), diagonals
        jr = j["jds_rows"]
        np.testing.assert_array_equal(jr, np.argsort(-cnt, kind="stable"))
        if len(tiles):
            for dg in range(j["max_row_blocks"]):
                seg = j["jds_blk"][j["jds_ptr"][dg]:j["jds_ptr"][dg + 1]]
                rows = jr[: len(seg)]
                assert (cnt[rows] > dg).all()
                np.testing.assert_array_equal(seg, j["csr_blk"][j["row_ptr"][rows] + dg])


def oracle_compact(z):
    z = int(z)
    return sum(((z >> (2 * k)) & 1) << k for k in range(16))


def test_kdtree_rejects_bad_arguments(hm):
    import ctypes

    out = ctypes.c_void_p()
    assert hm.lib().hm_kdtree_build(None, 100, 3, 16, None, ctypes.byref(out)) == 1
    pts = hm.generate_dataset(100, 3)
    assert hm.lib().hm_kdtree_build(ctypes.c_void_p(pts.data_ptr()), 100, 17, 16, None,
                                    ctypes.byref(out)) == 1
