"""Benchmark of the H-matrix engine on the precision-form workload.

Workload (default): N = 2^20 points uniform in [0,1]^3 from the engine's
generateDataset-equivalent generator, Matern-3/2 kernel with l = 0.2 plus 1e-3
on the diagonal, bucket 64, box-center admissibility eta = 1, ARA tolerance
1e-4, rank cap 128, 16 right-hand sides ~ N(0,1).

Both forms are built on the same tree and structure: the mixed-precision form
(BF16 hi + lo factor panels, the headline) and the plain FP32 form (timed
beside it).  A step is one H-matvec Y = H X (16 columns) with X already
resident on the GPU.  value = algorithmic GB/s of that product: the stored
factor and dense-block bytes read once per phase plus X read and Y written
(the H-matrix is GBs, far larger than the 126 MB L2, so every step streams it
from HBM; no flush needed).  Build seconds (points + KD tree + structure +
compression) are reported beside it.  The roofline object is the dominant
kernel of the headline form, timed with CUDA events on the launching stream.
`--impl reference` times the reference's CPU path for the same product (dense
FP64 kernel generation + OpenBLAS dgemm, extrapolated from a bounded sample of
row panels) and reports it in the same unit: the bytes of the dense FP64
matrix it forms divided by its time.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--n N] [--precision both|mixed|fp32]
Multi-GPU (torchrun): every rank builds and multiplies its own independent
cloud (seed offset by rank): weak scaling with no data-path collective.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "kaust-hierarchical-matrices_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "H-build s & H-matvec GB/s (%HBM peak): mixed vs FP32 at 1e-4 rel err"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def workload_config(args):
    return {
        "workload": "precision form: N=%d uniform 3-D, Matern-3/2 l=0.2 + 1e-3 diag, bucket 64, "
                    "box-center eta=1, tol 1e-4, rank cap 128, %d RHS" % (args.n, args.nrhs),
        "n": args.n, "d": 3, "bucket": 64, "eta": 1.0, "kernel": "matern32", "ell": 0.2, "nugget": 1e-3,
        "tol": 1e-4, "max_rank": 128, "sample_block": 16, "nrhs": args.nrhs,
        "l2": "no flush: the streamed H-matrix (GBs) exceeds the 126 MB L2",
    }


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, device_index):
        try:
            rows = [r.split(", ") for r in open(self.path).read().strip().splitlines()]
            rows = [r for r in rows if len(r) >= 8 and r[0].strip() == str(device_index)]
            sm = [float(r[1]) for r in rows]
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].strip() == "Active"})
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": float(rows[0][2]) if rows else None, "reasons": reasons,
                    "samples": len(rows)}
        except Exception as e:  # clocks are advisory
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)}


def cpu_reference(args, n, nrhs, budget_s, threads):
    """The reference's CPU path on a bounded sample of row panels; returns
    (seconds for the full product, extrapolated, sample description)."""
    import oracle

    rng = np.random.default_rng(1234)
    pts = rng.uniform(0.0, 1.0, size=(3, n))  # same distribution; the CPU path needs no tree
    perm = np.arange(n, dtype=np.int32)
    X = rng.standard_normal((nrhs, n))
    rows_per_panel = 64
    work = np.empty(rows_per_panel * n)
    done_rows, t_gen, t_blas = 0, 0.0, 0.0
    t0 = time.time()
    while time.time() - t0 < budget_s and done_rows < n:
        r0 = int(rng.integers(0, n - rows_per_panel))
        _, tg, tb = oracle.cpu_panel_matvec(pts, n, 3, perm, oracle.K_MATERN32, 0.2, 1e-3, r0, rows_per_panel, X,
                                            threads, work)
        t_gen += tg
        t_blas += tb
        done_rows += rows_per_panel
    per_row = (t_gen + t_blas) / done_rows
    return per_row * n, "%d rows x %d cols (%d panels of %d rows), extrapolated linearly to %d rows" % (
        done_rows, n, done_rows // rows_per_panel, rows_per_panel, n), t_gen, t_blas, done_rows


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n, nrhs = args.n, args.nrhs
    dense_bytes = 8.0 * n * n + 8.0 * n * nrhs * 2
    vals = []
    # each step is a bounded sample of the product, sized so that the whole
    # run stays within about two minutes whatever --steps is
    per_step = max(0.2, min(args.ref_budget, 120.0 / (args.warmup + args.steps)))
    for _ in range(args.warmup + args.steps):
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, per_step, threads)
        vals.append(t_full)
    t = float(np.mean(vals[args.warmup:]))
    value = dense_bytes / t / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(args), bytes_per_step=dense_bytes,
                       path="dense FP64 kernel generation + OpenBLAS dgemm (the reference has no CPU "
                            "H-matrix path)"),
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def kernel_times(hm, lib, H, X, Y, n, nrhs, stream, reps=6):
    """Per-kernel device times (CUDA events on `stream`) and algorithmic bytes of
    one product, averaged over reps after one warm call."""
    import ctypes

    cap = 8
    names = (ctypes.c_char_p * cap)()
    ms = (ctypes.c_float * cap)()
    by = (ctypes.c_longlong * cap)()
    cnt = ctypes.c_int()
    acc = {}
    order = []
    for r in range(reps + 1):
        hm._check(lib.hm_hmatvec_kernels(H.h, nrhs, hm._ptr(X), n, hm._ptr(Y), n, hm._stream(stream), cap, names,
                                         ms, by, ctypes.byref(cnt)))
        if r == 0:
            continue
        for i in range(cnt.value):
            k = names[i].decode()
            if k not in acc:
                acc[k] = [0.0, by[i]]
                order.append(k)
            acc[k][0] += ms[i] / reps
    return [(k, acc[k][0], acc[k][1]) for k in order]


def traffic_for(kernel, n, nrhs):
    """DRAM bytes per launch of `kernel` from the committed ncu summary of this
    workload (profiles/*.json), or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_c2.json")
    try:
        with open(path) as f:
            t = json.load(f)
        if t.get("n") == n and t.get("nrhs") == nrhs:
            return t["kernels"].get(kernel)
    except Exception:
        pass
    return None


def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist

    import hmatrix as hm

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    n, d, b, nrhs = args.n, 3, 64, args.nrhs
    lib = hm.lib()

    def barrier():
        if world > 1:
            dist.barrier()

    def ev_time(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    # ---- build: points, KD tree, structure, then each form's H-matrix ---------
    def front():
        pts = hm.generate_dataset(n, d, seed=1234 + rank, stream=stream)
        tree = hm.construct_kdtree(pts, n, d, b, stream=stream)
        st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0, stream=stream)
        return pts, tree, st

    (pts, tree, st), front_s = ev_time(front)
    forms = ["mixed", "fp32"] if args.precision == "both" else [args.precision]
    Hs, build_s = {}, {}
    for f in forms:
        prec = hm.PREC_MIXED if f == "mixed" else hm.PREC_FP32
        Hs[f], t = ev_time(lambda: hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3,
                                                    tol=1e-4, max_rank=128, sample_block=16, precision=prec,
                                                    seed=7, stream=stream))
        build_s[f] = front_s + t
    head = forms[0]

    gen = torch.Generator(device=dev)
    gen.manual_seed(99 + rank)
    X = torch.randn((nrhs, n), generator=gen, device=dev, dtype=torch.float32)  # column-major n x nrhs
    Y = torch.empty((nrhs, n), device=dev, dtype=torch.float32)

    def step_of(H):
        def step():
            hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(X), n, hm._ptr(Y), n, 0, hm._stream(stream)))
        return step

    def timed(step, sampler=None):
        if sampler is not None:
            sampler.__enter__()
            time.sleep(0.5)  # nvidia-smi is sampling before the timed region starts
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.__exit__()
        barrier()
        ms = t0.elapsed_time(t1) / args.steps
        if world > 1:
            tt = torch.tensor([ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms

    clocks = ClockSampler(os.path.join(ROOT, "gpurun_out", "bench_clocks_%d.csv" % rank)
                          if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "/tmp/bench_clocks_%d.csv" % rank)
    res = {}
    for f in forms:
        ms = timed(step_of(Hs[f]), clocks if f == head else None)
        kt = kernel_times(hm, lib, Hs[f], X, Y, n, nrhs, stream)
        bp, be = ctypes.c_longlong(), ctypes.c_longlong()
        mp, me = ctypes.c_float(), ctypes.c_float()
        hm._check(lib.hm_hmatvec_profile(Hs[f].h, nrhs, hm._ptr(X), n, hm._ptr(Y), n, hm._stream(stream),
                                         ctypes.byref(mp), ctypes.byref(me), ctypes.byref(bp), ctypes.byref(be)))
        res[f] = {"ms": ms, "bytes": bp.value + be.value, "kernels": kt, "launches_per_step": len(kt)}

    # ---- roofline of the headline form's dominant kernel --------------------
    hbm, peak_kind = peaks()
    kt = res[head]["kernels"]
    dom = max(kt, key=lambda x: x[1])
    ach = dom[2] / (dom[1] * 1e-3) / 1e9
    traffic = traffic_for(dom[0], n, nrhs)
    roof = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "peak_kind": peak_kind + " (STREAM-style copy)", "traffic": traffic,
            "kernels": {k: {"ms": t, "bytes": by, "gbs": by / (t * 1e-3) / 1e9, "frac": by / (t * 1e-3) / 1e9 / hbm}
                        for k, t, by in kt}}

    # ---- end to end through the C ABI with host buffers ---------------------
    H = Hs[head]
    Xh = torch.empty((nrhs, n), dtype=torch.float32, pin_memory=True)
    Xh.copy_(X.cpu())
    Yh = torch.empty((nrhs, n), dtype=torch.float32, pin_memory=True)
    Xd = torch.empty_like(X)

    def e2e_step():
        Xd.copy_(Xh, non_blocking=True)
        hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(Xd), n, hm._ptr(Y), n, 0, hm._stream(stream)))
        Yh.copy_(Y, non_blocking=True)

    e2e_ms = timed(e2e_step)

    # ---- accuracy against the FP64 oracle on sampled rows -------------------
    errs = {}
    if rank == 0 and not args.skip_check:
        import oracle

        perm = tree.copy_out()["perm"]
        p_h = pts.cpu().numpy()
        rows = np.random.default_rng(5).choice(n, args.check_rows, replace=False)
        Xn = X.cpu().numpy().astype(np.float64)
        Yref = oracle.dense_rows_matvec(p_h, n, d, perm, oracle.K_MATERN32, 0.2, 1e-3, rows, Xn)
        for f in forms:
            step_of(Hs[f])()
            torch.cuda.synchronize()
            Yn = Y.cpu().numpy()[:, rows]
            errs[f] = float(np.linalg.norm(Yn - Yref) / np.linalg.norm(Yref))

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, args.cpu_budget, threads)
        dense_bytes = 8.0 * n * n + 8.0 * n * nrhs * 2
        cpu = {"value": dense_bytes / t_full / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": sample, "seconds_per_product_extrapolated": t_full}

    if rank == 0:
        r = res[head]
        value = world * r["bytes"] / (r["ms"] * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 hi+lo, f32 acc" if head == "mixed" else "f32",
            "data": "synthetic",
            "config": dict(workload_config(args), precision=head, bytes_per_step=r["bytes"],
                           parallelism="independent cloud per rank" if world > 1 else "single GPU"),
            "hbm_frac": value / world / hbm,
            "build_s": build_s[head], "rel_err_vs_fp64": errs.get(head), "rel_err_rows": args.check_rows,
            "hbuild": Hs[head].stats(),
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": world * r["bytes"] / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": 4 * n * nrhs, "d2h_bytes_per_step": 4 * n * nrhs},
            "gpu_launches": r["launches_per_step"] * args.steps * ((nrhs + 15) // 16),
            "clocks": clocks.summary(local),
        }
        if "fp32" in res and head != "fp32":
            f = res["fp32"]
            line["fp32_form"] = {
                "ms_per_step": f["ms"], "gbs": f["bytes"] / (f["ms"] * 1e-3) / 1e9,
                "hbm_frac": f["bytes"] / (f["ms"] * 1e-3) / 1e9 / hbm, "bytes_per_step": f["bytes"],
                "build_s": build_s["fp32"], "rel_err_vs_fp64": errs.get("fp32"),
                "kernels": {k: {"ms": t, "bytes": by} for k, t, by in f["kernels"]}}
            line["speedup_vs_fp32"] = f["ms"] / r["ms"]
            line["fp32_equivalent_gbs"] = f["bytes"] / (r["ms"] * 1e-3) / 1e9
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "mixed"],
                    help="both: the mixed form is the headline, the FP32 form is timed beside it")
    ap.add_argument("--check-rows", type=int, default=256)
    ap.add_argument("--skip-check", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=5.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
