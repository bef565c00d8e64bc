"""Times the KD tree and the block structure: the reference's own compiled
code (oracle/_ref/ref_pipeline, built by `make -C oracle ref`) against this
engine's, on the same points (the reference's generateDataset, seed 1234).

Baseline measurement only (test infrastructure; never part of the product).
Usage on a GPU box: python oracle/time_front.py [N ...]
"""
import os
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "kaust-hierarchical-matrices_b200"))


def ref_times(n, d, b, admiss):
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run([os.path.join(HERE, "_ref", "ref_pipeline"), str(n), str(d), str(b), str(admiss),
                              os.path.join(td, "o.bin")], capture_output=True, text=True, check=True).stdout
    m = re.search(r"kdtree_ms=([0-9.]+) structure_ms=([0-9.]+)", out)
    return float(m.group(1)), float(m.group(2))


def our_times(n, d, b, admiss, reps=3):
    import torch

    import hmatrix as hm

    pts = hm.generate_dataset(n, d, seed=1234)
    best = (1e30, 1e30)
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tree = hm.construct_kdtree(pts, n, d, b)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        st = hm.construct_hmatrix_structure(tree, admiss, 1.0)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        best = (min(best[0], (t1 - t0) * 1e3), min(best[1], (t2 - t1) * 1e3))
        del st, tree
    return best


def main():
    sizes = [int(x) for x in sys.argv[1:]] or [8192, 1 << 17, 1 << 20]
    print("| N | d | bucket | admissibility | reference KD tree ms | ours | reference structure ms | ours |")
    print("|---|---|---|---|---|---|---|---|")
    for n in sizes:
        d, b = (2, 32) if n == 8192 else (3, 64)
        for admiss in (1, 0):
            rk, rs = ref_times(n, d, b, admiss)
            ok, os_ = our_times(n, d, b, admiss)
            print("| %d | %d | %d | %s | %.1f | %.2f | %.1f | %.2f |" % (n, d, b, "box-center" if admiss else "weak",
                                                                       rk, ok, rs, os_), flush=True)


if __name__ == "__main__":
    main()
