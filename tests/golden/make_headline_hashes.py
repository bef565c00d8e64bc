"""Generate tests/golden/headline_hashes.json: digests of the reference's own
KD tree and block structure at the benchmark's sizes.

Runs oracle/_ref/ref_pipeline (the reference's generateDataset,
allocateKDTree/constructKDTree and constructHMatrixStructure, compiled from
the unmodified sources by `make -C oracle ref`) on a GPU for each case below
and records SHA-256 digests of its outputs (the outputs themselves are tens of
MB per case):

  points   float64 SoA p[dim*N + i]
  perm     int32, tree position -> original index (segmentIndices)
  offsets  int32 leaf offsets (segmentOffsets)
  bmin/bmax float64, levels 0..depth-1 concatenated, [node*d + dim]
  tiles    int32 Morton list of each level 1..depth (counts stored too)

Cases: the precision workload's points (N = 2^20, 3-D, the reference's
generateDataset with seed 1234, bucket 64) under box-center and weak
admissibility; the scale workload's points (N = 2^21 Gaussian mixture drawn by
this engine's hm_generate_mixture, seed 1234, fed to the reference through its
point-file input) under box-center admissibility with the reference's eta = 1
(it has no other); and one batch-sized cloud of a non-power-of-two size.

    python tests/golden/make_headline_hashes.py   (on a GPU box, after `make -C oracle ref`)
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "kaust-hierarchical-matrices_b200"))

from make_golden import REF, parse  # noqa: E402

# name, N, d, bucket, admissibility (0 weak, 1 box-center), points
CASES = [
    ("precision_box", 1 << 20, 3, 64, 1, "gen"),
    ("precision_weak", 1 << 20, 3, 64, 0, "gen"),
    ("scale_mixture_box", 1 << 21, 3, 64, 1, "mixture"),
    ("cloud_n50016_box", 50016, 3, 64, 1, "gen"),
]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def digests(points, perm, offsets, bmin, bmax, tiles_per_level):
    return dict(points=sha(points.astype(np.float64)), perm=sha(perm.astype(np.int32)),
                offsets=sha(offsets.astype(np.int32)), bmin=sha(bmin.astype(np.float64)),
                bmax=sha(bmax.astype(np.float64)),
                tiles=[sha(t.astype(np.int32)) for t in tiles_per_level],
                counts=[int(len(t)) for t in tiles_per_level])


def mixture_points(n, d, seed):
    """The scale workload's points: this engine's device mixture generator."""
    import hmatrix as hm

    return hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=seed).cpu().numpy()


def main(out):
    res = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, n, d, b, adm, src in CASES:
            args = [REF, str(n), str(d), str(b), str(adm), os.path.join(tmp, name + ".bin")]
            if src == "mixture":
                pf = os.path.join(tmp, name + ".pts")
                mixture_points(n, d, 1234).astype(np.float64).tofile(pf)
                args.append(pf)
            p = subprocess.run(args, check=True, capture_output=True, text=True)
            g = parse(os.path.join(tmp, name + ".bin"))
            depth = int(g["depth"])
            nt = g["num_tiles"]
            lists, o = [], 0
            for lv in range(depth):
                lists.append(g["tiles"][o:o + nt[lv]])
                o += nt[lv]
            res[name] = dict(N=n, d=d, bucket=b, admiss=adm, points_source=src, depth=depth,
                             **digests(g["points"], g["perm"], g["offsets"], g["bmin"], g["bmax"], lists))
            print(name, p.stdout.strip(), flush=True)
    with open(out, "w") as f:
        json.dump(res, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "headline_hashes.json"))
