"""Generate the golden fixtures that pin the CPU oracle.

Runs the reference's own compiled pipeline stages (oracle/_ref/ref_pipeline,
built by `make -C oracle ref` from the unmodified reference sources) on a GPU
and stores each output as a compressed .npz next to this script:

    python tests/golden/make_golden.py [outdir]

Each case records the inputs (points, N, d, bucket, admissibility) and the
reference's outputs: the KD-tree permutation and leaf offsets, the per-level
bounding boxes and the per-level Morton block lists of the H-matrix structure.
Point sets that the reference's generateDataset does not produce (lattice
points with many exact ties, a Gaussian mixture) are written by this script
from fixed numpy seeds and fed to the reference through its point-file input.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_pipeline")

# name, N, d, bucket, admissibility (0 weak, 1 box-center), point source
CASES = [
    ("c1_box", 8192, 2, 32, 1, "gen"),
    ("c1_weak", 8192, 2, 32, 0, "gen"),
    ("n1000_d3", 1000, 3, 32, 1, "gen"),
    ("n5000_d3_b64", 5000, 3, 64, 1, "gen"),
    ("n20_single_leaf", 20, 2, 32, 1, "gen"),
    ("d1_n777", 777, 1, 16, 1, "gen"),
    ("lattice_ties", 4096, 3, 16, 1, "lattice"),
    ("mixture_d3", 20000, 3, 64, 1, "mixture"),
]


def lattice_points(n, d, seed=7):
    """Points on an 8-level lattice per axis: every coordinate ties with ~n/8
    others and many points coincide exactly."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 8, size=(d, n)).astype(np.float64) / 8.0).copy()


def mixture_points(n, d, seed=11, k=16):
    """Isotropic Gaussian mixture: centres U[0,1]^d, sigma log-uniform in
    [0.01, 0.1], weights Dirichlet(1)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(k, d))
    sigma = np.exp(rng.uniform(np.log(0.01), np.log(0.1), size=k))
    w = rng.dirichlet(np.ones(k))
    comp = rng.choice(k, size=n, p=w)
    pts = centres[comp] + sigma[comp, None] * rng.standard_normal((n, d))
    return np.ascontiguousarray(pts.T)


def parse(path):
    with open(path, "rb") as f:
        buf = f.read()
    assert buf[:8] == b"HMREF01\x00", "bad magic"
    off = 8
    hdr = np.frombuffer(buf, np.int32, 6, off)
    off += 24
    n, d, b, adm, depth, nlev = (int(x) for x in hdr)

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(buf, dtype, count, off).copy()
        off += a.nbytes
        return a

    out = dict(N=n, d=d, bucket=b, admiss=adm, depth=depth, num_levels=nlev)
    out["points"] = take(np.float64, n * d)
    out["perm"] = take(np.int32, n)
    out["offsets"] = take(np.int32, (1 << depth) + 1)
    bmin, bmax = [], []
    for lv in range(depth):
        bmin.append(take(np.float64, (1 << lv) * d))
        bmax.append(take(np.float64, (1 << lv) * d))
    out["bmin"] = np.concatenate(bmin) if bmin else np.zeros(0)
    out["bmax"] = np.concatenate(bmax) if bmax else np.zeros(0)
    counts = take(np.int32, nlev)
    out["num_tiles"] = counts
    tiles = [take(np.int32, int(counts[lv])) for lv in range(nlev - 1)]
    out["tiles"] = np.concatenate(tiles) if tiles else np.zeros(0, np.int32)
    assert off == len(buf), "trailing bytes"
    return out


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name, n, d, b, adm, src in CASES:
            args = [REF, str(n), str(d), str(b), str(adm), os.path.join(tmp, name + ".bin")]
            if src != "gen":
                pts = lattice_points(n, d) if src == "lattice" else mixture_points(n, d)
                pf = os.path.join(tmp, name + ".pts")
                pts.astype(np.float64).tofile(pf)
                args.append(pf)
            subprocess.run(args, check=True)
            res = parse(os.path.join(tmp, name + ".bin"))
            res["source"] = np.array(src)
            np.savez_compressed(os.path.join(outdir, name + ".npz"), **res)
            print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
