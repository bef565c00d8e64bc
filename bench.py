"""Benchmark of the H-matrix engine on the precision-form workload.

Workload (default): N = 2^20 points uniform in [0,1]^3 from the engine's
generateDataset-equivalent generator, Matern-3/2 kernel with l = 0.2 plus 1e-3
on the diagonal, bucket 64, box-center admissibility eta = 1, ARA tolerance
1e-4, rank cap 128, 16 right-hand sides ~ N(0,1).

A step is one H-matvec Y = H X (16 columns) on the built H-matrix with X
already resident on the GPU.  value = algorithmic GB/s of that product: bytes
of the stored factors and dense blocks read once plus X read and Y written
(the H-matrix is GBs, far larger than the 126 MB L2, so every step streams it
from HBM).  The H-build time (KD tree + structure + compression) is reported
beside it.  `--impl reference` times the reference's CPU path for the same
product (dense FP64 kernel generation + OpenBLAS dgemm, extrapolated from a
bounded sample of row panels) and reports it in the same unit: the bytes of
the dense FP64 matrix it forms divided by its time.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--n N] [--precision fp32|mixed]
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
    for _ in range(args.warmup + args.steps):
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, args.ref_budget, threads)
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


def run_ours(args):
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

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- build (timed once) -------------------------------------------------
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    pts = hm.generate_dataset(n, d, seed=1234 + rank, stream=stream)
    tree = hm.construct_kdtree(pts, n, d, b, stream=stream)
    st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, 1.0, stream=stream)
    prec = hm.PREC_MIXED if args.precision == "mixed" else hm.PREC_FP32
    H = hm.build_hmatrix(tree, st, pts, kernel=hm.K_MATERN32, ell=0.2, nugget=1e-3, tol=1e-4, max_rank=128,
                         sample_block=16, precision=prec, seed=7, stream=stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    build_s = ev0.elapsed_time(ev1) / 1e3
    hstats = H.stats()

    gen = torch.Generator(device=dev)
    gen.manual_seed(99 + rank)
    X = torch.randn((nrhs, n), generator=gen, device=dev, dtype=torch.float32)  # column-major n x nrhs
    Y = torch.empty((nrhs, n), device=dev, dtype=torch.float32)
    lib = hm.lib()
    import ctypes

    def step():
        hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(X), n, hm._ptr(Y), n, 0, hm._stream(stream)))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region ---------------------------------------------------------
    clocks = ClockSampler(os.path.join(ROOT, "gpurun_out", "bench_clocks_%d.csv" % rank)
                          if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "/tmp/bench_clocks_%d.csv" % rank)
    with clocks:
        barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = t0.elapsed_time(t1) / args.steps
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())

    # ---- per-kernel device times for the roofline ---------------------------
    mp, me = ctypes.c_float(), ctypes.c_float()
    bp, be = ctypes.c_longlong(), ctypes.c_longlong()
    prof = []
    for _ in range(5):
        hm._check(lib.hm_hmatvec_profile(H.h, nrhs, hm._ptr(X), n, hm._ptr(Y), n, hm._stream(stream),
                                         ctypes.byref(mp), ctypes.byref(me), ctypes.byref(bp), ctypes.byref(be)))
        prof.append((mp.value, me.value))
    mp_avg = float(np.mean([p[0] for p in prof[1:]]))
    me_avg = float(np.mean([p[1] for p in prof[1:]]))
    bytes_step = bp.value + be.value
    hbm, peak_kind = peaks()
    dom = ("k_mv_expand", be.value, me_avg) if me_avg >= mp_avg else ("k_mv_project", bp.value, mp_avg)
    ach = dom[1] / (dom[2] * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": hbm, "unit": "GB/s",
            "frac": ach / hbm, "peak_kind": peak_kind, "traffic": None,
            "other": {"k_mv_project" if dom[0] == "k_mv_expand" else "k_mv_expand": {
                "bytes": bp.value if dom[0] == "k_mv_expand" else be.value,
                "ms": mp_avg if dom[0] == "k_mv_expand" else me_avg}},
            "matvec_frac": bytes_step / ((mp_avg + me_avg) * 1e-3) / 1e9 / hbm}

    # ---- end to end through the C ABI with host buffers ---------------------
    Xh = torch.empty((nrhs, n), dtype=torch.float32, pin_memory=True)
    Xh.copy_(X.cpu())
    Yh = torch.empty((nrhs, n), dtype=torch.float32, pin_memory=True)
    Xd = torch.empty_like(X)
    for _ in range(2):
        Xd.copy_(Xh, non_blocking=True)
        step()
        Yh.copy_(Y, non_blocking=True)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        Xd.copy_(Xh, non_blocking=True)
        hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(Xd), n, hm._ptr(Y), n, 0, hm._stream(stream)))
        Yh.copy_(Y, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        tt = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())

    # ---- accuracy against the FP64 oracle on sampled rows -------------------
    rel_err = None
    if rank == 0 and not args.skip_check:
        import oracle

        perm = tree.copy_out()["perm"]
        p_h = pts.cpu().numpy()
        rows = np.random.default_rng(5).choice(n, args.check_rows, replace=False)
        Xn = X.cpu().numpy().astype(np.float64)
        Yref = oracle.dense_rows_matvec(p_h, n, d, perm, oracle.K_MATERN32, 0.2, 1e-3, rows, Xn)
        Yn = Y.cpu().numpy()[:, rows]
        hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(X), n, hm._ptr(Y), n, 0, hm._stream(stream)))
        torch.cuda.synchronize()
        Yn = Y.cpu().numpy()[:, rows]
        rel_err = float(np.linalg.norm(Yn - Yref) / np.linalg.norm(Yref))

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, args.cpu_budget, threads)
        dense_bytes = 8.0 * n * n + 8.0 * n * nrhs * 2
        cpu = {"value": dense_bytes / t_full / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": sample, "seconds_per_product_extrapolated": t_full}

    if rank == 0:
        value = world * bytes_step / (ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == hm.PREC_FP32 else "bf16+f32acc", "data": "synthetic",
            "config": dict(workload_config(args), precision=args.precision, bytes_per_step=bytes_step,
                           parallelism="independent cloud per rank" if world > 1 else "single GPU"),
            "build_s": build_s, "hbuild": {k: hstats[k] for k in hstats},
            "rel_err_vs_fp64": rel_err, "rel_err_rows": args.check_rows,
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": world * bytes_step / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                    "ms_per_step": e2e_ms, "h2d_bytes_per_step": 4 * n * nrhs, "d2h_bytes_per_step": 4 * n * nrhs},
            "gpu_launches": 2 * args.steps * ((nrhs + 15) // 16),
            "clocks": clocks.summary(local),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "mixed"])
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
