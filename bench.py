"""Benchmark of the H-matrix engine on the precision-form workload.

Workload (default): N = 2^20 points uniform in [0,1]^3 from the engine's
generateDataset-equivalent generator, Matern-3/2 kernel with l = 0.2 plus 1e-3
on the diagonal, bucket 64, box-center admissibility eta = 1, ARA tolerance
1e-4, rank cap 128, 16 right-hand sides ~ N(0,1).

Both forms are built on the same tree and structure: the mixed-precision form
(BF16 hi + lo factor panels, the headline) and the plain FP32 form (timed
beside it).  A step is one H-matvec Y = H X (16 columns) with X already
resident on the GPU.  value = products per second (whole job), the unit both
arms share; the metric's GB/s and fraction of the HBM peak are reported beside
it ("gbs", "hbm_frac"): the algorithmic bytes of the product (stored factor
and dense-block bytes read once per phase plus X read and Y written) over its
time.  The H-matrix is GBs, far larger than the 126 MB L2, so every step
streams it from HBM; no flush is needed.  Build seconds (points + KD tree +
structure + compression) are reported beside it.  The roofline object is the
dominant kernel of the headline form, timed with CUDA events on the launching
stream.  `--impl reference` times the reference's CPU path for the same
product (dense FP64 kernel generation + OpenBLAS dgemm) on a bounded sample of
row panels per step and extrapolates it to the whole product
("extrapolated": true); its value is products per second of that
extrapolated time.

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
import tempfile
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


# The workloads: "precision" is the headline (the bench line of a plain
# `python bench.py`); "scale" and "batch" measure the other two forms.
WORKLOADS = {
    "precision": dict(desc="precision form: N=%(n)d uniform 3-D, Matern-3/2 l=0.2 + 1e-3 diag, bucket 64, "
                           "box-center eta=1, tol 1e-4, rank cap 128, %(nrhs)d RHS",
                      n=1 << 20, nrhs=16, points="uniform", kernel="matern32", ell=0.2, nugget=1e-3, eta=1.0,
                      tol=1e-4, max_rank=128),
    "scale": dict(desc="scale stress: N=%(n)d points of a 16-component Gaussian mixture (sigma log-uniform "
                       "[0.01, 0.1], Dirichlet(1) weights), exp(-r/0.05), bucket 64, box-center eta=1.5, tol 1e-4, "
                       "rank cap 256, %(nrhs)d RHS",
                  n=1 << 21, nrhs=128, points="mixture", kernel="exp", ell=0.05, nugget=0.0, eta=1.5, tol=1e-4,
                  max_rank=256),
    "batch": dict(desc="batching form: %(clouds)d clouds of log-uniform [2048, 65536] points (multiples of 32), "
                       "uniform 3-D, exp(-r/0.1), bucket 64, box-center eta=1, tol 1e-5, rank cap 256, %(nrhs)d RHS "
                       "per cloud, one graph launch per product",
                  n=0, nrhs=32, clouds=64, points="uniform", kernel="exp", ell=0.1, nugget=0.0, eta=1.0, tol=1e-5,
                  max_rank=256),
}
KERNEL_IDS = {"exp": 0, "matern32": 1, "gauss": 2}


def workload(args):
    w = dict(WORKLOADS[args.workload])
    if args.n:
        w["n"] = args.n
    if args.nrhs:
        w["nrhs"] = args.nrhs
    return w


def workload_config(args):
    """The workload's description: identical keys and values in both arms."""
    w = workload(args)
    cfg = {"workload": w["desc"] % w, "name": args.workload}
    cfg.update({k: v for k, v in w.items() if k != "desc"})
    cfg.update({"d": 3, "bucket": 64, "sample_block": 16,
                "l2": "no flush: the streamed H-matrix (GBs) exceeds the 126 MB L2"})
    return cfg


PRODUCTS = "products/s"  # the unit of `value` in both arms


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
        w = workload(args)
        _, tg, tb = oracle.cpu_panel_matvec(pts, n, 3, perm, KERNEL_IDS[w["kernel"]], w["ell"], w["nugget"], r0,
                                            rows_per_panel, X, threads, work)
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
    w = workload(args)
    nrhs = w["nrhs"]
    if args.workload == "batch":
        # every cloud's dense product; the cost per entry is sampled on the
        # largest cloud and scaled by sum n_c^2
        sizes = batch_sizes(w, 2024)
        n = max(sizes)
        scale = float(sum(x * x for x in sizes)) / (n * n)
        dense_bytes = float(sum(8.0 * x * x + 16.0 * x * nrhs for x in sizes))
    else:
        n = w["n"]
        scale = 1.0
        dense_bytes = 8.0 * n * n + 8.0 * n * nrhs * 2
    vals, walls = [], []
    # each step is a bounded sample of the product (a few row panels), sized
    # so that the whole run stays within about two minutes whatever --steps
    # is; the sample's time is extrapolated linearly to the whole product
    per_step = max(0.2, min(args.ref_budget, 120.0 / (args.warmup + args.steps)))
    for _ in range(args.warmup + args.steps):
        w0 = time.time()
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, per_step, threads)
        walls.append(time.time() - w0)
        vals.append(t_full * scale)
    t = float(np.mean(vals[args.warmup:]))
    wall = float(np.mean(walls[args.warmup:]))
    value = 1.0 / t  # products per second, of the extrapolated whole product
    line = {
        "metric": METRIC, "value": value, "unit": PRODUCTS, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "extrapolated": True,
        "value_note": "each step times a sample of row panels of the dense product (ms_per_step is that "
                      "sample's wall time) and extrapolates it linearly to the whole product; value = 1 / "
                      "extrapolated_s_per_product",
        "extrapolated_s_per_product": t,
        "path": "dense FP64 kernel generation + OpenBLAS dgemm (the reference has no CPU H-matrix path)",
        "dense_bytes_per_product": dense_bytes, "dense_gbs": dense_bytes / t / 1e9,
        "cpu_baseline": {"value": value, "unit": PRODUCTS, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": PRODUCTS, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class CopyPipeline:
    """End-to-end steps with host buffers.  Every step copies its input from
    pinned host memory to the device, runs the product and copies the result
    back to pinned host memory.  Uploads run on one copy stream and downloads
    on another, each into one of two device buffers, so that step i + 1's
    upload and step i - 1's download overlap step i's product; the products
    stay in order on the compute stream (a matrix has one workspace).  Every
    step's two copies lie inside the timed region.  product(xd, yd) issues one
    product on the compute stream (the current stream when it is called)."""

    def __init__(self, torch, compute, Xh, y_shape, product):
        self.t, self.s, self.Xh, self.product = torch, compute, Xh, product
        dev = compute.device
        self.up, self.down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        self.Xd = [torch.empty(Xh.shape, dtype=Xh.dtype, device=dev) for _ in range(2)]
        self.Yd = [torch.empty(y_shape, dtype=torch.float32, device=dev) for _ in range(2)]
        self.Yh = [torch.empty(y_shape, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        self.read_done = [None, None]  # the product that last read Xd[b]
        self.down_done = [None, None]  # the download that last read Yd[b]
        self.i = 0

    def start(self):
        """Copy streams wait for all work issued so far on the compute stream."""
        e = self.t.cuda.Event()
        e.record(self.s)
        self.up.wait_event(e)
        self.down.wait_event(e)

    def step(self):
        T, b = self.t, self.i & 1
        self.i += 1
        if self.read_done[b] is not None:
            self.up.wait_event(self.read_done[b])
        with T.cuda.stream(self.up):
            self.Xd[b].copy_(self.Xh, non_blocking=True)
        e_up = T.cuda.Event()
        e_up.record(self.up)
        self.s.wait_event(e_up)
        if self.down_done[b] is not None:
            self.s.wait_event(self.down_done[b])
        with T.cuda.stream(self.s):
            self.product(self.Xd[b], self.Yd[b])
        e_p = T.cuda.Event()
        e_p.record(self.s)
        self.read_done[b] = e_p
        self.down.wait_event(e_p)
        with T.cuda.stream(self.down):
            self.Yh[b].copy_(self.Yd[b], non_blocking=True)
        e_d = T.cuda.Event()
        e_d.record(self.down)
        self.down_done[b] = e_d

    def finish(self):
        """The compute stream waits for the last downloads (an event recorded
        on it afterwards marks the end of every step)."""
        for e in self.down_done:
            if e is not None:
                self.s.wait_event(e)

    def time(self, warmup, steps, barrier, world):
        import ranks as _ranks

        self.start()
        for _ in range(warmup):
            self.step()
        self.finish()
        self.t.cuda.synchronize()
        barrier()
        self.t.cuda.synchronize()
        t0, t1 = self.t.cuda.Event(enable_timing=True), self.t.cuda.Event(enable_timing=True)
        t0.record(self.s)
        self.start()
        for _ in range(steps):
            self.step()
        self.finish()
        t1.record(self.s)
        self.t.cuda.synchronize()
        barrier()
        return _ranks.max_over_ranks(t0.elapsed_time(t1) / steps, world)


def out_dir():
    """Where the clock log and the autotuner's cache go: $HM_BENCH_OUT, else
    the temporary directory."""
    d = os.environ.get("HM_BENCH_OUT") or tempfile.gettempdir()
    os.makedirs(d, exist_ok=True)
    return d


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


TRAFFIC_SOURCES = ["csrc/hm_mixed.cu", "csrc/hm_mixed.h", "csrc/hm_fp32.cu", "csrc/hm_mma.cuh", "csrc/hm_matvec.cu",
                   "csrc/hm_mixed_tc.cu", "csrc/hm_tc.cuh"]


def kernel_source_digest():
    """SHA-256 over the product kernels' sources, code only (// comments and
    blank lines removed): a DRAM-traffic capture is used only while the
    kernels it measured are unchanged."""
    import hashlib
    import re

    h = hashlib.sha256()
    for f in TRAFFIC_SOURCES:
        with open(os.path.join(PKG, f), encoding="utf-8") as fh:
            for line in fh:
                code = re.sub(r"//.*$", "", line).strip()
                if code:
                    h.update(code.encode() + b"\n")
    return h.hexdigest()


def traffic_for(kernel, workload_name, alg_bytes):
    """DRAM bytes per launch of `kernel` on this workload: the committed ncu
    capture of a small case of the same workload (profiles/dram_traffic.json,
    one kernel, few launches) scaled by algorithmic bytes to the full launch,
    or None when there is no capture of the current kernel sources."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        if t.get("source_sha256") != kernel_source_digest():
            return None
        k = t["workloads"][workload_name]["kernels"][kernel]
        return float(k["dram_bytes_per_launch"]) * float(alg_bytes) / float(k["algorithmic_bytes_per_launch"])
    except Exception:
        return None


def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist

    import hmatrix as hm
    import ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    w = workload(args)
    n, d, b, nrhs = w["n"], 3, 64, w["nrhs"]
    kid = KERNEL_IDS[w["kernel"]]
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

    # One cloud split by block rows (--shard rows): every rank builds the same
    # cloud's tree and structure and its own row shard of the H-matrix; a step
    # all-gathers X (rows spread over the ranks like Y's) and multiplies.
    # Otherwise every rank has its own independent cloud.
    sharded = args.shard == "rows"
    seed = 1234 if sharded else ranks.cloud_seed(1234, rank)

    # ---- build: points, KD tree, structure, then each form's H-matrix ---------
    def front():
        if w["points"] == "mixture":
            pts = hm.generate_mixture(n, d, ncomp=16, sigma_min=0.01, sigma_max=0.1, seed=seed, stream=stream)
        else:
            pts = hm.generate_dataset(n, d, seed=seed, stream=stream)
        tree = hm.construct_kdtree(pts, n, d, b, stream=stream)
        st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, w["eta"], stream=stream)
        return pts, tree, st

    (pts, tree, st), front_s = ev_time(front)
    shards = ranks.subtree_shards(list(tree.copy_out()["offsets"]), world if sharded else 1)
    own = shards[rank if sharded else 0]
    forms = ["mixed", "fp32"] if args.precision == "both" else [args.precision]
    Hs, build_s = {}, {}
    for f in forms:
        prec = hm.PREC_MIXED if f == "mixed" else hm.PREC_FP32
        Hs[f], t = ev_time(lambda: hm.build_hmatrix(tree, st, pts, kernel=kid, ell=w["ell"], nugget=w["nugget"],
                                                    tol=w["tol"], max_rank=w["max_rank"], sample_block=16,
                                                    precision=prec, seed=7, stream=stream,
                                                    leaves=own[:2] if sharded else None))
        build_s[f] = front_s + t
        if f == "mixed" and args.schedule:
            hm.schedule_set(Hs[f], args.schedule, stream=stream)
    head = forms[0]

    gen = torch.Generator(device=dev)
    gen.manual_seed(99 if sharded else 99 + rank)
    X = torch.randn((nrhs, n), generator=gen, device=dev, dtype=torch.float32)  # column-major n x nrhs
    Y = torch.empty((nrhs, n), device=dev, dtype=torch.float32)
    r0, r1 = own[2], own[3]
    X_own = X[:, r0:r1].contiguous()  # this rank's rows of X (all of them unless sharded)
    gather = ranks.RowGather(shards, nrhs, torch.float32, dev) if sharded and world > 1 else None

    def step_of(H):
        def step():
            xs = gather.gather(X_own, rank) if gather is not None else X
            hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(xs), n, hm._ptr(Y), n, 0, hm._stream(stream)))
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
        return ranks.max_over_ranks(t0.elapsed_time(t1) / args.steps, world)

    clocks = ClockSampler(os.path.join(out_dir(), "bench_clocks_%d.csv" % rank))
    res = {}
    for f in forms:
        # the product runs in passes of 128 right-hand sides (mixed form) or 16 (FP32)
        width = 128 if f == "mixed" else 16
        nr = min(width, nrhs)
        panels = (nrhs + width - 1) // width
        ms = timed(step_of(Hs[f]), clocks if f == head else None)
        Hs[f].check()  # no bounded device-side wait gave up in the timed products
        kt = kernel_times(hm, lib, Hs[f], X, Y, n, nr, stream)
        bp, be = ctypes.c_longlong(), ctypes.c_longlong()
        mp, me = ctypes.c_float(), ctypes.c_float()
        hm._check(lib.hm_hmatvec_profile(Hs[f].h, nr, hm._ptr(X), n, hm._ptr(Y), n, hm._stream(stream),
                                         ctypes.byref(mp), ctypes.byref(me), ctypes.byref(bp), ctypes.byref(be)))
        # algorithmic bytes of the whole product: factors and dense blocks once
        # per phase, X and Y for every right-hand side (12 bytes per row each)
        by = bp.value + be.value + 12 * n * (nrhs - nr)
        res[f] = {"ms": ms, "bytes": by, "kernels": kt, "launches_per_step": len(kt) * panels,
                  "panels": panels}

    # ---- roofline of the headline form's dominant kernel --------------------
    hbm, peak_kind = peaks()
    kt = res[head]["kernels"]
    dom = max(kt, key=lambda x: x[1])
    ach = dom[2] / (dom[1] * 1e-3) / 1e9
    traffic = traffic_for(dom[0], args.workload, dom[2])
    roof = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "peak_kind": peak_kind + " (STREAM-style copy)", "traffic": traffic,
            "kernels": {k: {"ms": t, "bytes": by, "gbs": by / (t * 1e-3) / 1e9, "frac": by / (t * 1e-3) / 1e9 / hbm}
                        for k, t, by in kt}}

    # ---- end to end through the C ABI with host buffers ---------------------
    # (copies of step i +- 1 overlap step i's product; see CopyPipeline)
    H = Hs[head]
    Xh = torch.empty((nrhs, r1 - r0), dtype=torch.float32, pin_memory=True)  # this rank's rows
    Xh.copy_(X_own.cpu())
    Yfull = torch.empty((nrhs, n), device=dev, dtype=torch.float32)

    def e2e_product(xd, yd):
        if sharded:
            xs = gather.gather(xd, rank) if gather is not None else xd
            hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(xs), n, hm._ptr(Yfull), n, 0, hm._stream(stream)))
            yd.copy_(Yfull[:, r0:r1])
        else:
            hm._check(lib.hm_hmatvec(H.h, 0, nrhs, hm._ptr(xd), n, hm._ptr(yd), n, 0, hm._stream(stream)))

    e2e_ms = CopyPipeline(torch, stream, Xh, (nrhs, r1 - r0), e2e_product).time(args.warmup, args.steps, barrier,
                                                                               world)

    # ---- optional: conjugate-gradient iterations on the same matrix ----------
    # (a tolerance no residual meets, so exactly cg_iters iterations run and
    # the call reports HM_ERR_NOT_CONVERGED, or HM_ERR_UNSUPPORTED if the
    # compressed operator shows itself indefinite first; device time with CUDA
    # events on the solve's stream)
    cg = None
    if args.cg_iters > 0:
        cs = torch.cuda.Stream(device=dev)
        Xs = torch.empty_like(X)
        it, res_c = ctypes.c_int(), ctypes.c_double()

        def cg_run(k):
            st_ = lib.hm_cg_solve(Hs[head].h, nrhs, hm._ptr(X), n, hm._ptr(Xs), n, 1e-300, k, 8, hm._stream(cs),
                                  ctypes.byref(it), ctypes.byref(res_c))
            if st_ not in (0, 4, 6):
                hm._check(st_)

        torch.cuda.synchronize()
        cg_run(16)  # warm-up (records its graph, allocates the workspace from the pool)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(cs)
        cg_run(args.cg_iters)
        c1.record(cs)
        torch.cuda.synchronize()
        cg_ms = c0.elapsed_time(c1)
        cg = {"iterations": it.value, "ms": cg_ms, "ms_per_iteration": cg_ms / max(it.value, 1),
              "product_ms": res[head]["ms"], "check_every": 8}

    # ---- accuracy against the FP64 oracle on sampled rows -------------------
    errs = {}
    if rank == 0 and not args.skip_check and not sharded:
        import oracle

        perm = tree.copy_out()["perm"]
        p_h = pts.cpu().numpy()
        rows = np.random.default_rng(5).choice(n, args.check_rows, replace=False)
        # all columns up to 32; beyond that the first and the last 16 (they lie
        # in different passes of the product)
        cols = np.arange(nrhs) if nrhs <= 32 else np.r_[0:16, nrhs - 16:nrhs]
        Xn = X.cpu().numpy()[cols].astype(np.float64)
        Yref = oracle.dense_rows_matvec(p_h, n, d, perm, kid, w["ell"], w["nugget"], rows, Xn)
        for f in forms:
            step_of(Hs[f])()
            torch.cuda.synchronize()
            Yn = Y.cpu().numpy()[cols][:, rows]
            errs[f] = float(np.linalg.norm(Yn - Yref) / np.linalg.norm(Yref))

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        t_full, sample, tg, tb, rows = cpu_reference(args, n, nrhs, args.cpu_budget, threads)
        dense_bytes = 8.0 * n * n + 8.0 * n * nrhs * 2
        cpu = {"value": 1.0 / t_full, "unit": PRODUCTS, "cores": threads, "kind": "port",
               "sample": sample, "seconds_per_product_extrapolated": t_full, "dense_gbs": dense_bytes / t_full / 1e9}

    # products per step over the whole job: one per rank (independent clouds)
    # or one in all (row shards of one cloud)
    jobs = 1 if sharded else world
    all_bytes = res[head]["bytes"]
    if world > 1:
        bt = torch.tensor([float(all_bytes)], dtype=torch.float64, device=dev)
        dist.all_reduce(bt)
        all_bytes = float(bt.item())
    if rank == 0:
        r = res[head]
        gbs = all_bytes / (r["ms"] * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": jobs * 1e3 / r["ms"], "unit": PRODUCTS, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "bf16 hi+lo, f32 acc" if head == "mixed" else "f32",
            "data": "synthetic",
            "config": workload_config(args),
            "precision": head, "bytes_per_step": r["bytes"],
            "parallelism": ("one cloud in %d block-row shards (subtrees), NCCL all-gather of X per product" % world
                            if sharded else ("independent cloud per rank" if world > 1 else "single GPU")),
            "gbs": gbs, "hbm_frac": gbs / world / hbm,
            "build_s": build_s[head], "rel_err_vs_fp64": errs.get(head), "rel_err_rows": args.check_rows,
            "rel_err_cols": min(nrhs, 32),
            "hbuild": Hs[head].stats(),
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": jobs * 1e3 / e2e_ms, "unit": PRODUCTS, "ms_per_step": e2e_ms,
                    "gbs": all_bytes / (e2e_ms * 1e-3) / 1e9,
                    "h2d_bytes_per_step": 4 * (r1 - r0) * nrhs, "d2h_bytes_per_step": 4 * (r1 - r0) * nrhs},
            "gpu_launches": r["launches_per_step"] * args.steps,
            "clocks": clocks.summary(local),
        }
        if cg is not None:
            line["cg"] = cg
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


def batch_sizes(w, seed):
    """Cloud sizes log-uniform in [2048, 65536], rounded to multiples of 32."""
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(2048), np.log(65536), w["clouds"]))
    return [int(max(32, round(v / 32) * 32)) for v in x]


def run_batch(args):
    """Batching form: all clouds in one forest, one graph launch per product."""
    import ctypes

    import torch
    import torch.distributed as dist

    import hmatrix as hm
    import ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    s = torch.cuda.Stream(dev)  # a created stream: the product is a recorded graph
    w = workload(args)
    nrhs, kid = w["nrhs"], KERNEL_IDS[w["kernel"]]
    # --shard clouds: one job's clouds spread over the ranks by a size-balanced
    # assignment; otherwise every rank has a job of its own
    split = args.shard == "clouds" and world > 1
    if split:
        every = batch_sizes(w, 2024)
        mine = ranks.assign_clouds(every, world)[rank]
        sizes = [every[i] for i in mine]
        seeds = [5000 + i for i in mine]
    else:
        sizes = batch_sizes(w, 2024 + rank)
        seeds = [5000 + 100 * rank + i for i in range(len(sizes))]
    lib = hm.lib()

    def ev_time(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    def front():
        cl = []
        for i, n in enumerate(sizes):
            pts = hm.generate_dataset(n, 3, seed=seeds[i], stream=s)
            tree = hm.construct_kdtree(pts, n, 3, 64, stream=s)
            st = hm.construct_hmatrix_structure(tree, hm.BOX_CENTER, w["eta"], stream=s)
            cl.append((n, pts, tree, st))
        return cl

    with torch.cuda.stream(s):
        clouds, front_s = ev_time(front)
        forms = ["mixed", "fp32"] if args.precision == "both" else [args.precision]
        Bs, build_s, tune = {}, {}, {}
        cache = os.path.join(out_dir(), "hm_autotune.txt")
        for f in forms:
            B = hm.Batch([c[2] for c in clouds], [c[3] for c in clouds], stream=s)
            prec = hm.PREC_MIXED if f == "mixed" else hm.PREC_FP32
            _, t = ev_time(lambda: B.build(kernel=kid, ell=w["ell"], nugget=w["nugget"], tol=w["tol"],
                                           max_rank=w["max_rank"], precision=prec, seed=7, stream=s))
            build_s[f] = front_s + t
            tune[f] = hm.autotune(B.hmatrix(), min(nrhs, 128 if f == "mixed" else 16), cache, stream=s)
            Bs[f] = B
        head = forms[0]
        N = Bs[head].n
        X = torch.randn((nrhs, N), device=dev).t()
        Y = torch.empty((nrhs, N), device=dev).t()
        clocks = ClockSampler(os.path.join(out_dir(), "bench_clocks_%d.csv" % rank))
        res = {}
        for f in forms:
            B = Bs[f]
            if f == head:
                clocks.__enter__()
                time.sleep(0.5)
            for _ in range(args.warmup):
                B.matvec(X, Y, s)
            s.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(args.steps):
                B.matvec(X, Y, s)
            e1.record(s)
            s.synchronize()
            if f == head:
                clocks.__exit__()
            ms = ranks.max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
            H = B.hmatrix()
            width = 128 if f == "mixed" else 16  # right-hand sides per pass of the product
            nr = min(width, nrhs)
            kt = kernel_times(hm, lib, H, X, Y, N, nr, s)
            bp, be = ctypes.c_longlong(), ctypes.c_longlong()
            mp, me = ctypes.c_float(), ctypes.c_float()
            hm._check(lib.hm_hmatvec_profile(H.h, nr, hm._ptr(X), N, hm._ptr(Y), N, hm._stream(s), ctypes.byref(mp),
                                             ctypes.byref(me), ctypes.byref(bp), ctypes.byref(be)))
            res[f] = {"ms": ms, "bytes": bp.value + be.value + 12 * N * (nrhs - nr), "kernels": kt,
                      "panels": (nrhs + width - 1) // width, "stats": H.stats()}
        # e2e: host X in, host Y out, product through hm_batch_matvec
        # (copies of step i +- 1 overlap step i's product; the recorded graph
        # reads and writes fixed buffers, filled and drained by device copies)
        B = Bs[head]
        Xh = torch.empty((nrhs, N), pin_memory=True)
        Xh.copy_(X.t().cpu())
        Xg = torch.empty((nrhs, N), device=dev)
        Yg = torch.empty((nrhs, N), device=dev)

        def e2e_product(xd, yd):
            Xg.copy_(xd)
            B.matvec(Xg.t(), Yg.t(), s)
            yd.copy_(Yg)

        def no_barrier():
            if world > 1:
                dist.barrier()

        e2e_ms = CopyPipeline(torch, s, Xh, (nrhs, N), e2e_product).time(args.warmup, args.steps, no_barrier,
                                                                         world)
        # accuracy on sampled rows of a few clouds against the FP64 oracle
        errs = {}
        if rank == 0 and not args.skip_check:
            import oracle

            rng = np.random.default_rng(9)
            pick = rng.choice(len(clouds), 4, replace=False)
            for f in forms:
                Bs[f].matvec(X, Y, s)
                s.synchronize()
                Yn = Y.cpu().numpy()
                num = den = 0.0
                for c in pick:
                    n, pts, tree, st = clouds[c]
                    r0, r1 = Bs[f].row_offsets[c], Bs[f].row_offsets[c + 1]
                    perm = tree.copy_out()["perm"]
                    rows = rng.choice(n, 64, replace=False)
                    Xc = X[r0:r1].cpu().numpy().astype(np.float64)
                    Yref = oracle.dense_rows_matvec(pts.cpu().numpy(), n, 3, perm, kid, w["ell"], w["nugget"], rows,
                                                    Xc.T).T
                    num += float(np.sum((Yn[r0:r1][rows] - Yref) ** 2))
                    den += float(np.sum(Yref ** 2))
                errs[f] = (num / den) ** 0.5
    jobs = 1 if split else world
    all_bytes = float(res[head]["bytes"])
    if world > 1:
        bt = torch.tensor([all_bytes], dtype=torch.float64, device=dev)
        dist.all_reduce(bt)
        all_bytes = float(bt.item())
    if rank == 0:
        hbm, peak_kind = peaks()
        r = res[head]
        value = all_bytes / (r["ms"] * 1e-3) / 1e9
        dom = max(r["kernels"], key=lambda x: x[1])
        ach = dom[2] / (dom[1] * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": jobs * 1e3 / r["ms"], "unit": PRODUCTS, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"], "higher_is_better": True,
            "scaling": "strong" if split else "weak", "vs_baseline": None,
            "dtype": "bf16 hi+lo, f32 acc" if head == "mixed" else "f32",
            "data": "synthetic",
            "config": workload_config(args),
            "parallelism": ("the job's %d clouds spread over %d ranks (size-balanced)" % (w["clouds"], world)
                            if split else ("an independent job per rank" if world > 1 else "single GPU")),
            "n_total": N, "cloud_sizes": sizes, "precision": head, "bytes_per_step": r["bytes"],
            "schedule": tune[head][0],
            "gbs": value, "hbm_frac": value / world / hbm, "build_s": build_s[head], "rel_err_vs_fp64": errs.get(head),
            "hbuild": r["stats"],
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": hbm, "unit": "GB/s",
                         "frac": ach / hbm, "peak_kind": peak_kind, "traffic": None,
                         "kernels": {k: {"ms": t, "bytes": by} for k, t, by in r["kernels"]}},
            "cpu_baseline": None,
            "e2e": {"value": jobs * 1e3 / e2e_ms, "unit": PRODUCTS, "ms_per_step": e2e_ms,
                    "gbs": all_bytes / (e2e_ms * 1e-3) / 1e9,
                    "h2d_bytes_per_step": 4 * N * nrhs, "d2h_bytes_per_step": 4 * N * nrhs},
            "gpu_launches": len(r["kernels"]) * r["panels"] * args.steps,
            "graph_launches_per_step": 1,
            "clocks": clocks.summary(local),
        }
        if "fp32" in res and head != "fp32":
            f = res["fp32"]
            line["fp32_form"] = {"ms_per_step": f["ms"], "gbs": f["bytes"] / (f["ms"] * 1e-3) / 1e9,
                                 "build_s": build_s["fp32"], "rel_err_vs_fp64": errs.get("fp32"),
                                 "schedule": tune["fp32"][0]}
            line["speedup_vs_fp32"] = f["ms"] / r["ms"]
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
    ap.add_argument("--workload", default="precision", choices=sorted(WORKLOADS),
                    help="precision (default, the headline line), scale, or batch")
    ap.add_argument("--n", type=int, default=None, help="points (default: the workload's)")
    ap.add_argument("--nrhs", type=int, default=None, help="right-hand sides (default: the workload's)")
    ap.add_argument("--precision", default="both", choices=["both", "fp32", "mixed"],
                    help="both: the mixed form is the headline, the FP32 form is timed beside it")
    ap.add_argument("--shard", default="none", choices=["none", "rows", "clouds"],
                    help="multi-GPU split: none (an independent cloud per rank, weak scaling), rows (one cloud in "
                         "block-row shards with an all-gather of X per product), clouds (batch workload: the "
                         "job's clouds spread over the ranks)")
    ap.add_argument("--check-rows", type=int, default=4096,
                    help="rows of the FP64 oracle's dense product the error is measured on")
    ap.add_argument("--schedule", default=None,
                    help="mixed form: a schedule in hm_autotune's notation, e.g. "
                         "'mixed chunk_tiles=128 group_tiles=4 p1_ring=0 wide_tc=0'")
    ap.add_argument("--skip-check", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=5.0)
    ap.add_argument("--cg-iters", type=int, default=0,
                    help="also run this many conjugate-gradient iterations (hm_cg_solve, graph-launched "
                         "chunks of 8 on a created stream) with the headline form and report ms per iteration")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
