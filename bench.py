"""Benchmark of the supernodal numeric factorization (one JSON line on stdout, rank 0).

A step is one mixed-precision numeric factorization of the workload matrix followed by a
solve refined in FP64 to backward error <= 1e-12 (default workload grid3d_60: the 3D
7-point Laplacian on 60^3 plus 1e-3 I, n = 216,000, ordered by geometric nested dissection
and analysed by the reference's own symbolic phase; the supernode partition and final
permutation come from tests/golden/sym_grid3d_60.npz).  The metric is the reference's flop
measure fl = sum_j c_j^2 (exact column counts) divided by the step time; the plain FP64
factorization is timed alongside (--mode fp64 makes it the headline).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: values already resident in HBM, K factorizations timed with CUDA events on the
library's stream, bracketed by barrier + synchronize; max over ranks.  `e2e` times the same
step through the public API with host buffers (values and b uploaded, x downloaded).  After
the timed region (rank 0, one GPU): parity of the FP64 factor against the reference's own
factor, forward error against the FP64 solution, the CPU baseline, and one compact record
per other configuration (``configs``).  The reference arm (--impl reference) times the
reference's own CPU executor (oracle/_ref) on the host cores; it loads neither the product
package nor its library (the workload generator is loaded from its file: numpy and scipy
only).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("factorization GFLOP/s (fl = sum c_j^2 / time) of the mixed-precision factor + "
          "FP64-refined solve to backward error <= 1e-12 (FP64 factor timed alongside)")
GOLDEN = os.path.join(ROOT, "tests", "golden")
TOL = 1e-12
HBM_FALLBACK_GBS = 6650.0


def matrices_module():
    """The workload generators (swcholesky_b200/matrices.py, numpy + scipy only), loaded from
    their file so that the reference arm never imports the product package."""
    name = "swc_workload_matrices"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(
        name, os.path.join(ROOT, "swcholesky_b200", "matrices.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload_config(name, n, nnz_lower, nsuper, xsize, fl, nrhs):
    """The `config` object of both arms (identical keys and values for one workload)."""
    return {"workload": name, "n": int(n), "nnz_lower": int(nnz_lower), "nsuper": int(nsuper),
            "xsize": int(xsize), "fl": float(fl), "nrhs": int(nrhs),
            "backward_error_target": TOL,
            "l2": f"inputs larger than L2 (L = {xsize * 8 / 1e9:.2f} GB)"}


def hbm_peak():
    """(GB/s, source) of the measured HBM copy bandwidth, else the recipe's fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "of fallback (6.65 TB/s)"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def load_problem(name):
    from swcholesky_b200 import workloads as W
    # the cond ~1e10 stencil shares the structure (and fixture) of the cond ~1e6 one
    fixture = name[:-3] if name.endswith("c10") else name
    g = dict(np.load(os.path.join(GOLDEN, f"sym_{fixture}.npz")))
    A, perm_in, meta = W.build(name)
    P = W.assemble(A, g["perm"], g["super"])
    return A, perm_in, meta, P, float(g["fl"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms while running.  start()
    returns once the first sample has arrived (nvidia-smi takes a moment to start), and only
    samples that arrive after that moment count, so a timed region of ~0.1 s still holds
    two or more."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0:
            time.sleep(0.005)
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "first", 0):]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_gemm_peak(torch, dev):
    """Dense FP64 GEMM throughput of this GPU measured with cuBLAS (torch.matmul, 8192^3),
    best of 5 after 2 warm-ups; the FP64 roofline denominator (MEASURED_PEAKS.json has
    none for FP64)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def reference_time(A, perm_in, threads, budget_s, max_reps, min_reps=1, keep_L=False):
    """Times the reference's own FP64 executor; returns (median seconds, reps, symbolic,
    the last factor L if keep_L else None)."""
    from oracle import oracle as O
    R = O.RefSymbolic(A, perm_in)
    times = []
    L = None
    t0 = time.time()
    while len(times) < max_reps and (len(times) < min_reps or time.time() - t0 < budget_s):
        L, t, ret = R.factor(threads=threads)
        if ret != 1:
            raise RuntimeError("reference factorization failed")
        times.append(t)
    sym = R.sym
    R.close()
    return float(np.median(times)), len(times), sym, (L if keep_L else None)


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest `value` over all ranks (every rank gets it); the job's time is its
    slowest rank's time."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu summary
    (profiles/<kernel>_<workload>.md, line 'traffic_bytes_per_launch: N'), else None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def run_reference(args, rank, world):
    """The reference arm: the reference's own FP64 executor (sw_cholesky_left_par_05_check,
    built from its sources into oracle/_ref) on the host cores, on this workload; rank 0
    alone runs and prints.  Nothing of the product is imported or loaded."""
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libswref.so not built"}))
        return
    M = matrices_module()
    A, perm_in, _ = M.workload_matrix(args.workload)
    threads = os.cpu_count() or 1
    R = O.RefSymbolic(A, perm_in)
    s = R.sym
    for _ in range(args.warmup):
        R.factor(threads=threads)
    times = []
    for _ in range(args.steps):
        _, t, ret = R.factor(threads=threads)
        assert ret == 1
        times.append(t)
    R.close()
    t = float(np.mean(times))
    fl = s.flops
    val = fl / t / 1e9
    line = {
        "metric": METRIC, "value": round(val, 3), "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator; reference symbolic phase)",
        "config": workload_config(args.workload, s.n, s.A2p[-1], s.nsuper, s.xsize, fl,
                                  args.nrhs),
        "mode": "fp64 (the reference computes in FP64 only)",
        "parallelism": f"{threads} host threads (OpenBLAS)",
        "impl": "reference",
        "cpu_baseline": {"value": round(val, 3), "unit": "GFLOP/s", "cores": threads,
                         "kind": "reference", "cpu_model": cpu_model(),
                         "sample": f"full {args.workload} factorization per step "
                                   f"(sw_cholesky_left_par_05_check + OpenBLAS, {threads} threads)"},
        "e2e": {"value": round(val, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def tf32_gemm_peak(torch, dev, bf16: bool = False):
    """Dense TF32 (or BF16) GEMM throughput measured with cuBLAS (torch.matmul, 8192^3),
    best of 5; a split-TF32 product costs three TF32 products and a BF16x3 product six BF16
    products, so their peaks are a third / a sixth of this."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    dt = torch.bfloat16 if bf16 else torch.float32
    a = torch.randn(n, n, dtype=dt, device=dev)
    b = torch.randn(n, n, dtype=dt, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


def event_ms(torch, stream, fn, reps):
    """Mean device milliseconds of fn() over reps calls, CUDA events on `stream`."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import swcholesky_b200 as swc

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    A, perm_in, meta, P, fl = load_problem(args.workload)
    tol = TOL

    h = swc.Handle(local_rank)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet,
              P.levelPtr, P.parPtr, P.partition)
    plan = swc.plan_stats(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr,
                          P.pruneSet)
    solve_launches = 4 * plan["levels"]
    vals = torch.from_numpy(P.A2x).to(dev)
    nrhs = args.nrhs
    # right-hand sides: (nrhs, n) row-major = n x nrhs column-major, as the library takes them
    b_host = np.random.default_rng(0).standard_normal((nrhs, P.n) if nrhs > 1 else P.n)
    b = torch.from_numpy(b_host).to(dev)
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(h.stream, device=dev)
    mode = {"fp64": swc.SWC_MODE_FP64, "mixed": swc.SWC_MODE_MIXED_TF32X3,
            "bf16": swc.SWC_MODE_MIXED_BF16X3}[args.mode]
    mixed = mode != swc.SWC_MODE_FP64

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, world, dev)

    last = {}

    def step_headline():
        info = h.factor(vals, mode)
        assert info == 0, f"not SPD at column {info - 1}"
        _, berr, iters, meth = h.refine(b, tol=tol, maxit=60, out=x)
        last.update(berr=float(berr.max()), iters=iters, method=meth)

    def step_fp64():
        info = h.factor(vals, swc.SWC_MODE_FP64)
        assert info == 0, f"not SPD at column {info - 1}"

    for _ in range(args.warmup):
        step_fp64()
        step_headline()
    torch.cuda.synchronize()
    ms_fp64 = timed(step_fp64, args.steps)
    ms_fact = timed(lambda: h.factor(vals, mode), args.steps)
    clocks = ClockSampler(local_rank)
    clocks.start()
    ms = timed(step_headline, args.steps)
    clk = clocks.stop()
    x_mixed = x.cpu().numpy().copy()
    # FP64 factor followed by a refined solve, for the like-for-like comparison
    last_fp64 = {}

    def step_fp64_solve():
        step_fp64()
        _, berr, iters, meth = h.refine(b, tol=tol, maxit=60, out=x)
        last_fp64.update(berr=float(berr.max()), iters=iters)
    ms_fp64_solve = timed(step_fp64_solve, max(1, args.steps // 2))
    value = world * fl / (ms * 1e-3) / 1e9
    # one supernodal solve (forward + backward) with the FP64 factor, for the breakdown
    h.solve(b, out=x)
    ms_solve = timed(lambda: h.solve(b, out=x), args.steps)

    # ---- per-kernel roofline (a separate profiled factorization in the headline mode) ----
    prof64 = h.profile(vals, swc.SWC_MODE_FP64) if mixed else None
    prof = h.profile(vals, mode)
    kinds = {k: v for k, v in prof.items() if k != "memset"}
    dom = max(kinds, key=lambda k: kinds[k][1])
    la, kms, kfl, kby = kinds[dom]
    peak64 = fp64_gemm_peak(torch, dev) if rank == 0 else None
    bf16 = mode == swc.SWC_MODE_MIXED_BF16X3
    tf32 = mode == swc.SWC_MODE_MIXED_TF32X3
    peak32 = tf32_gemm_peak(torch, dev, bf16) if rank == 0 and mixed else None
    src64 = "FP64 cuBLAS DGEMM 8192^3 measured in this run"
    src_tf32 = ("cuBLAS TF32 GEMM 8192^3 measured in this run, divided by 3 (a split-TF32 product "
                "executes three TF32 piece products on tcgen05: hi hi' + lo hi' + hi lo')")
    src_bf16 = ("cuBLAS BF16 GEMM 8192^3 measured in this run, divided by 8 (a BF16x3 product "
                "executes eight BF16 piece products on tcgen05: [hi;mid][hi;mid]^T and "
                "[lo;hi][lo;hi]^T)")
    # per compute class: its kernel(s) and the peak of the arithmetic it runs in this mode
    # (split-TF32 mode: descendant updates and trailing SYRK steps on tcgen05; BF16x3 mode:
    # descendant updates on tcgen05, SYRK in FP64; the panel chain always FP64)
    if tf32:
        cls_kernel = {"update": ("k_scatter_tc", peak32 / 3.0, src_tf32),
                      "syrk": ("k_scatter_tc", peak32 / 3.0, src_tf32)}
    elif bf16:
        cls_kernel = {"update": ("k_update_tc", peak32 / 8.0, src_bf16),
                      "syrk": ("k_syrk_step", peak64, src64)}
    else:
        cls_kernel = {"update": ("k_update_tiles", peak64, src64),
                      "syrk": ("k_syrk_step", peak64, src64)}
    cls_kernel["panel"] = ("k_diag_step + k_trsm_step", peak64, src64)
    cls_kernel["small"] = ("k_factor_small*", peak64, src64)
    # the dominant kernel: classes grouped by the kernel that runs them (the split-TF32 scatter
    # kernel runs both the descendant updates and the trailing SYRK steps); the panel class is
    # two kernels (TRSM, diagonal block) of about equal share
    groups = {}
    for k in ("update", "syrk", "panel", "small"):
        kn = cls_kernel[k][0]
        g = groups.setdefault(kn, {"classes": [], "ms": 0.0, "flops": 0.0, "launches": 0})
        g["classes"].append(k)
        g["ms"] += kinds[k][1]
        g["flops"] += kinds[k][2]
        g["launches"] += kinds[k][0]
    kname = max(groups, key=lambda kn: groups[kn]["ms"] / (2.0 if kn.startswith("k_diag") else 1.0))
    dom = "+".join(groups[kname]["classes"])
    la, kms, kfl = groups[kname]["launches"], groups[kname]["ms"], groups[kname]["flops"]
    peak, psrc = {cls_kernel[k][0]: cls_kernel[k][1:] for k in cls_kernel}[kname]
    rooflines = {}
    for k in ("update", "syrk", "panel"):
        lk, mk, fk, _ = kinds[k]
        kn, pk, ps = cls_kernel[k]
        if mk > 0 and pk:
            ach = fk / (mk * 1e-3) / 1e12
            tr = profile_traffic(kn, args.workload) if rank == 0 else None
            rooflines[k] = {"kernel": kn, "launches": lk, "ms": round(mk, 4),
                            "achieved": round(ach, 4), "peak": round(pk, 3), "unit": "TFLOP/s",
                            "frac": round(ach / pk, 4), "peak_source": ps,
                            "traffic_bytes_per_launch": tr}
    hbm, hbm_src = hbm_peak()
    # HBM-bound classes: algorithmic bytes (plan builder) / device time of the class
    hbm_classes = {}
    for k in ("small", "assemble"):
        lk, mk, _, bk = prof[k]
        if mk > 0 and bk > 0:
            gbs = bk / (mk * 1e-3) / 1e9
            hbm_classes[k] = {"launches": lk, "ms": round(mk, 4), "algorithmic_bytes": bk,
                              "achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4)}

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if rank == 0 and not args.no_e2e:
        # pinned host buffers: values and b in, x out
        vals_pin = torch.empty(P.A2x.size, dtype=torch.float64, pin_memory=True).numpy()
        vals_pin[:] = P.A2x
        b_pin = torch.empty(b_host.shape, dtype=torch.float64, pin_memory=True).numpy()
        b_pin[:] = b_host
        x_pin = torch.empty(b_host.shape, dtype=torch.float64, pin_memory=True).numpy()
        if nrhs > 1:   # host arrays of several right-hand sides are n x nrhs, column-major
            b_pin, x_pin = b_pin.T, x_pin.T
        t_e2e, t_f, t_r = [], [], []
        for i in range(max(1, min(3, args.steps)) + 1):
            t0 = time.perf_counter()
            info = h.factor(vals_pin, mode)                                     # values from host
            t1 = time.perf_counter()
            _, berr, iters, meth = h.refine(b_pin, tol=tol, maxit=60, out=x_pin)  # b / x on host
            dt = time.perf_counter() - t0
            assert info == 0 and berr.max() <= tol
            if i > 0:
                t_e2e.append(dt)
                t_f.append(t1 - t0)
                t_r.append(dt - (t1 - t0))
        te = float(np.mean(t_e2e))
        e2e = {"value": round(fl / te / 1e9, 3), "unit": "GFLOP/s",
               "h2d_bytes_per_step": int(P.A2x.nbytes + b_host.nbytes),
               "d2h_bytes_per_step": int(b_host.nbytes),
               "ms_per_step": round(te * 1e3, 3),
               "ms_factor": round(float(np.mean(t_f)) * 1e3, 3),
               "ms_refined_solve": round(float(np.mean(t_r)) * 1e3, 3),
               "note": "swc_factor with host values + swc_refine with host b and x, pinned "
                       "host buffers, host clock"}
        # the reference-facing drop-in call (FP64 factor only, structure re-uploaded)
        L_host = np.zeros(P.xsize, np.float64)
        t_d = []
        for i in range(2):
            t0 = time.perf_counter()
            ret = swc.sw_cholesky_left_par_05(
                P.n, P.A2p, P.A2i, P.A2x, P.lC, P.Ls, P.Li_ptr, L_host, P.super, P.nsuper,
                None, P.prunePtr, P.pruneSet, P.levelPtr.size - 1, P.levelPtr, None, 0,
                P.parPtr, P.partition, 0, 1, 0, 0, None)
            assert ret == 1
            if i > 0:
                t_d.append(time.perf_counter() - t0)
        e2e["dropin_fp64_ms"] = round(float(np.mean(t_d)) * 1e3, 3)

    # ---- CPU baseline (the reference's own executor) and parity against its factor ----
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            threads = os.cpu_count() or 1
            tref, reps, rsym, L_ref = reference_time(A, perm_in, threads, budget_s=15.0,
                                                     max_reps=5, keep_L=True)
            cpu = {"value": round(fl / tref / 1e9, 3), "unit": "GFLOP/s", "cores": threads,
                   "kind": "reference", "cpu_model": cpu_model(),
                   "sample": f"{reps} full {args.workload} FP64 factorizations, median "
                             f"(reference sw_cholesky_left_par_05_check + OpenBLAS)"}
            if not args.no_single_thread:
                t1, r1, _, _ = reference_time(A, perm_in, 1, budget_s=0.0, max_reps=1)
                cpu["single_thread"] = {"value": round(fl / t1 / 1e9, 3), "unit": "GFLOP/s",
                                        "cores": 1, "sample": f"{r1} full {args.workload} "
                                        f"FP64 factorization, OpenBLAS 1 thread"}
            parity = parity_record(torch, swc, h, vals, P, rsym, L_ref, b_host, x_mixed, nrhs)
            del L_ref
        else:
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: oracle/_ref/libswref.so not built"}

    configs = None
    if rank == 0 and world == 1 and not args.no_extras:
        configs = extra_configs(torch, swc, dev)

    if rank == 0:
        achieved = kfl / (kms * 1e-3) / 1e12
        traffic = profile_traffic(kname, args.workload) if kname else None
        tsrc = (f"dram__bytes_read.sum + dram__bytes_write.sum per launch, ncu capture summarised "
                f"in profiles/{kname}_{args.workload}.md" if traffic else None)
        factor_launches = int(sum(v[0] for v in prof.values()))   # this mode's launch list
        per_step = factor_launches + (last.get("iters", 0) + 1) * (solve_launches + 5)
        executed = float(sum(v[2] for k, v in prof.items()))
        gs = dict(np.load(os.path.join(GOLDEN, f"sym_{args.workload}.npz")))
        nnzl = int(gs["nnzl"]) if "nnzl" in gs else None
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "mixed": "f64+tf32x3", "bf16": "f64+bf16x3"}[args.mode],
            "data": "synthetic (seeded generator; reference symbolic phase via fixture)",
            "config": workload_config(args.workload, P.n, P.A2p[-1], P.nsuper, P.xsize, fl, nrhs),
            "mode": args.mode,
            "parallelism": "replicas only" if world > 1 else "single GPU",
            "headline": {"ms_factor_plus_refined_solve": round(ms, 4),
                         "ms_factor": round(ms_fact, 4),
                         "refine_iterations": last.get("iters"),
                         "refine_method": last.get("method"),
                         "backward_error": last.get("berr"),
                         "fp64_ms_factor": round(ms_fp64, 4),
                         "fp64_gflops": round(world * fl / (ms_fp64 * 1e-3) / 1e9, 3),
                         "fp64_ms_factor_plus_refined_solve": round(ms_fp64_solve, 4),
                         "fp64_backward_error": last_fp64.get("berr"),
                         "ms_one_solve": round(ms_solve, 4),
                         "speedup_vs_fp64_factor": round(ms_fp64 / ms, 3),
                         "speedup_vs_fp64_factor_plus_solve": round(ms_fp64_solve / ms, 3)},
            "parity": parity,
            "work": {"fl": fl, "executed_flops": executed,
                     "executed_over_fl": round(executed / fl, 4),
                     "nnz_L_exact": nnzl, "xsize": int(P.xsize),
                     "xsize_over_nnz_L": round(P.xsize / nnzl, 4) if nnzl else None,
                     "note": "executed flops: the plan builder's per-class flop model of one "
                             "factorization on the relaxed structure (tile padding excluded)"},
            "roofline": {"bound": "tensor", "class": dom, "kernel": kname,
                         "achieved": round(achieved, 4),
                         "peak": round(peak, 3) if peak else None, "unit": "TFLOP/s",
                         "frac": round(achieved / peak, 4) if peak else None,
                         "traffic": traffic, "traffic_source": tsrc, "peak_source": psrc,
                         "fp64_peak": round(peak64, 3) if peak64 else None,
                         "launches": la, "kernel_ms": round(kms, 4),
                         "algorithmic_flops": kfl,
                         "classes": {k: {"launches": v[0], "ms": round(v[1], 4),
                                         "gflop": round(v[2] / 1e9, 4)}
                                     for k, v in prof.items()},
                         "classes_fp64": ({k: {"ms": round(v[1], 4)} for k, v in prof64.items()}
                                          if prof64 else None),
                         "hbm_classes": hbm_classes, "hbm_peak_gbs": hbm,
                         "hbm_peak_source": hbm_src, "rooflines": rooflines},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(per_step * args.steps),
            "clocks": clk,
            "configs": configs,
        }
        print(json.dumps(line))
    h.close()


def parity_record(torch, swc, h, vals, P, rsym, L_ref, b_host, x_mixed, nrhs):
    """The FP64 GPU factor against the reference's own FP64 factor of the same structure,
    and the headline solution against the FP64 solution with the reference's factor
    (oracle C restatement of the supernodal solves).  Outside any timed region."""
    from oracle import oracle as O
    same = (int(rsym.xsize) == int(P.xsize) and np.array_equal(rsym.super, P.super) and
            np.array_equal(rsym.Ls, P.Ls))
    rec = {"structure_matches_reference": bool(same)}
    if not same:
        return rec
    assert h.factor(vals, swc.SWC_MODE_FP64) == 0
    L = h.get_L()
    scale = float(np.abs(L_ref).max())
    rec["L_rel_vs_reference"] = float(np.abs(L - L_ref).max() / scale)
    rec["L_zeros_preserved"] = bool(np.all(L[L_ref == 0.0] == 0.0))
    del L
    xr = O.oracle_solve(P.n, P.lC, P.Ls, P.Li_ptr, L_ref, P.super,
                        b_host.T if nrhs > 1 else b_host)
    xm = x_mixed.T if nrhs > 1 else x_mixed
    fe = np.abs(xm - xr).max(axis=0) / np.abs(xr).max(axis=0)
    rec["forward_error_vs_fp64"] = [float(v) for v in np.atleast_1d(fe)]
    rec["forward_error_note"] = ("max |x - x_fp64| / max |x_fp64| per right-hand side; x_fp64 "
                                 "= supernodal solve with the reference's FP64 factor")
    return rec


def extra_configs(torch, swc, dev):
    """One compact record per other configuration, measured after the headline (device
    timing with CUDA events on the handle's stream; no clocks sampling).  Each is
    independent: a failure is recorded as its error message."""
    out = {}
    for name, fn in (("grid2d_100", _extra_grid2d_100), ("stencil27_40", _extra_stencil),
                     ("stencil27_40c10", _extra_stencil), ("batch256", _extra_batch),
                     ("gmrf_500", _extra_gmrf)):
        t0 = time.perf_counter()
        try:
            rec = fn(torch, swc, dev, name)
        except Exception as exc:   # a failed sub-record must not lose the headline line
            rec = {"error": f"{type(exc).__name__}: {exc}"}
        rec["wall_s"] = round(time.perf_counter() - t0, 2)
        out[name] = rec
        torch.cuda.empty_cache()
    return out


def _extra_grid2d_100(torch, swc, dev, name):
    """Config 1: 2D 5-point 100 x 100, the reference's own symbolic arrays and factor
    (small golden fixture).  FP64 factor time and L parity; mixed factor + refined solve."""
    g = dict(np.load(os.path.join(GOLDEN, "small_grid2d_100.npz")))
    h = swc.Handle(dev.index or 0)
    h.analyze(int(g["n"]), g["A2p"], g["A2i"], g["lC"], g["Ls"], g["Li_ptr"], g["super"],
              g["prunePtr"], g["pruneSet"], g["levelPtr"], g["parPtr"], g["partition"])
    st = torch.cuda.ExternalStream(h.stream, device=dev)
    vals = torch.from_numpy(g["A2x"]).to(dev)
    b = torch.from_numpy(g["b"]).to(dev)
    x = torch.zeros_like(b)
    fl = float(g["fl"])
    for _ in range(3):
        h.factor(vals)
    ms64 = event_ms(torch, st, lambda: h.factor(vals), 20)
    L = h.get_L()
    rel = float(np.abs(L - g["L"]).max() / np.abs(g["L"]).max())
    last = {}

    def mx():
        assert h.factor(vals, swc.SWC_MODE_MIXED_TF32X3) == 0
        _, berr, it, _ = h.refine(b, tol=TOL, maxit=60, out=x)
        last.update(berr=float(berr.max()), it=it)
    for _ in range(3):
        mx()
    msmx = event_ms(torch, st, mx, 10)
    h.close()
    return {"n": int(g["n"]), "fl": fl, "fp64_ms_factor": round(ms64, 4),
            "fp64_gflops": round(fl / (ms64 * 1e-3) / 1e9, 3),
            "L_rel_vs_reference": rel,
            "mixed_ms_factor_plus_refined_solve": round(msmx, 4),
            "mixed_backward_error": last.get("berr"), "mixed_refine_iterations": last.get("it")}


def _extra_stencil(torch, swc, dev, name):
    """Config 3: 3-dof 27-point stencil 40^3 (cond ~1e6, or ~1e10 for the c10 variant), 8
    right-hand sides.  FP64 factor; BF16x3 factor + FP64 refinement (CG fallback when it
    stalls); per right-hand side backward error and forward error against the FP64
    solution (FP64 factor refined to 1e-15)."""
    _, _, meta, P, fl = load_problem(name)
    h = swc.Handle(dev.index or 0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    st = torch.cuda.ExternalStream(h.stream, device=dev)
    vals = torch.from_numpy(P.A2x).to(dev)
    nrhs = 8
    b = torch.from_numpy(np.random.default_rng(3).standard_normal((nrhs, P.n))).to(dev)
    x64 = torch.zeros_like(b)
    x = torch.zeros_like(b)
    h.factor(vals)
    ms64 = event_ms(torch, st, lambda: h.factor(vals), 3)
    _, berr64, _, _ = h.refine(b, tol=1e-15, maxit=30, out=x64)
    last = {}

    def mx():
        assert h.factor(vals, swc.SWC_MODE_MIXED_BF16X3) == 0
        _, berr, it, meth = h.refine(b, tol=TOL, maxit=60, out=x)
        last.update(berr=berr, it=it, meth=meth)
    mx()
    msmx = event_ms(torch, st, mx, 2)
    msf = event_ms(torch, st, lambda: h.factor(vals, swc.SWC_MODE_MIXED_BF16X3), 2)
    xa, xr = x.cpu().numpy(), x64.cpu().numpy()
    fe = np.abs(xa - xr).max(axis=1) / np.abs(xr).max(axis=1)
    h.close()
    return {"n": P.n, "fl": fl, "cond_target": meta.get("cond"), "nrhs": nrhs,
            "fp64_ms_factor": round(ms64, 4), "fp64_gflops": round(fl / (ms64 * 1e-3) / 1e9, 3),
            "fp64_backward_error": [float(v) for v in berr64],
            "bf16x3_ms_factor": round(msf, 4),
            "bf16x3_ms_factor_plus_refined_solve": round(msmx, 4),
            "refine_iterations": last["it"],
            "refine_method": {0: "direct", 1: "refinement", 2: "CG fallback"}[last["meth"]],
            "backward_error": [float(v) for v in last["berr"]],
            "forward_error_vs_fp64": [float(v) for v in fe]}


def _extra_batch(torch, swc, dev, name):
    """Config 4: 256 weighted 2D grids (sides 30..200) as one batch; autotuned grouping and
    plan per mode; matrices per second of the factor and of factor + refined solve; the
    largest per-matrix backward error."""
    from swcholesky_b200 import matrices as Mx
    from swcholesky_b200 import workloads as W
    src, sides = W.batch_sources(seed=0)
    mats = [Mx.permute_lower(A, p) for A, p in src]
    nmat = len(mats)
    vals = torch.from_numpy(np.concatenate([m.data for m in mats])).to(dev)
    h = swc.Handle(dev.index or 0)
    h.batch_analyze(mats)
    st = torch.cuda.ExternalStream(h.stream, device=dev)
    b = torch.from_numpy(np.random.default_rng(0).standard_normal(h.n)).to(dev)
    x = torch.zeros_like(b)
    cache = os.path.join(os.environ.get("TMPDIR", "/tmp"), "swc_batch_tune.txt")
    rec = {"matrices": nmat, "n_total": int(h.n), "sides": [int(sides.min()), int(sides.max())]}
    for tag, mode in (("fp64", swc.SWC_MODE_FP64), ("mixed", swc.SWC_MODE_MIXED_TF32X3)):
        choice, _ = h.batch_autotune(vals, mode, cache)

        def fs():
            assert h.factor(vals, mode) == 0
            h.refine(b, tol=TOL, maxit=60, out=x)
        fs()
        msf = event_ms(torch, st, lambda: h.factor(vals, mode), 5)
        msfs = event_ms(torch, st, fs, 3)
        per = h.batch_berr(b, x)
        rec[tag] = {"ms_factor": round(msf, 4), "matrices_per_s": round(nmat / (msf * 1e-3), 1),
                    "ms_factor_plus_refined_solve": round(msfs, 4),
                    "matrices_per_s_factor_plus_solve": round(nmat / (msfs * 1e-3), 1),
                    "berr_max": float(per.max()), "autotune": list(choice),
                    "launches": h.launches}
    h.close()
    return rec


def _extra_gmrf(torch, swc, dev, name):
    """Config 5: GMRF 0.1 I + weighted Laplacian 500 x 500.  Time of the log-det gradient
    and of the solve-loss gradient (after the FP64 factor); fourth-order central finite
    differences on 64 random nonzeros: largest |fd - ad| / |ad| (plain) and with the
    1e-3 max|ad| floor; the split-TF32 factor's log-det gradient against the FP64 one."""
    _, _, _, P, fl = load_problem(name)
    h = swc.Handle(dev.index or 0)
    h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    st = torch.cuda.ExternalStream(h.stream, device=dev)
    v = torch.from_numpy(P.A2x.copy()).to(dev)
    g = torch.zeros(P.A2x.size, dtype=torch.float64, device=dev)
    assert h.factor(v) == 0
    h.logdet_grad(g)
    ms_ld = event_ms(torch, st, lambda: h.logdet_grad(g), 3)
    ad = g.cpu().numpy()
    rng = np.random.default_rng(2024)
    idx = rng.choice(P.A2x.size, 64, replace=False)
    fds = []
    for p in idx:
        a = float(P.A2x[p])
        hh = 1e-3 * max(abs(a), 1.0)
        vals = []
        for d in (2 * hh, hh, -hh, -2 * hh):
            v[p] = a + d
            assert h.factor(v) == 0
            vals.append(h.logdet())
        v[p] = a
        fds.append((-vals[0] + 8 * vals[1] - 8 * vals[2] + vals[3]) / (12 * hh))
    fds = np.array(fds)
    err = np.abs(fds - ad[idx])
    # solve-loss gradient timing: x = A^{-1} b, lam = A^{-1}(x - y)
    b = torch.from_numpy(rng.standard_normal(P.n)).to(dev)
    y = torch.from_numpy(rng.standard_normal(P.n)).to(dev)
    assert h.factor(v) == 0
    x, _, _, _ = h.refine(b, tol=1e-15, maxit=30)
    lam, _, _, _ = h.refine((x - y).contiguous(), tol=1e-15, maxit=30)
    gs = torch.zeros_like(g)
    h.solve_grad(x, lam, gs)
    ms_sg = event_ms(torch, st, lambda: h.solve_grad(x, lam, gs), 3)
    # split-TF32 factor: log-det gradient (selected inverse of the mixed factor)
    assert h.factor(v, swc.SWC_MODE_MIXED_TF32X3) == 0
    h.logdet_grad(g)
    gm = g.cpu().numpy()
    h.close()
    return {"n": P.n, "fl": fl, "ms_logdet_grad": round(ms_ld, 4),
            "ms_solve_grad": round(ms_sg, 4),
            "fd_samples": 64,
            "fd_logdet_max_rel_plain": float((err / np.abs(ad[idx])).max()),
            "fd_logdet_max_rel_floored": float((err / np.maximum(np.abs(ad[idx]),
                                                                 1e-3 * np.abs(ad).max())).max()),
            "mixed_logdet_grad_max_rel_vs_fp64": float(np.abs(gm - ad).max() / np.abs(ad).max()),
            "mixed_note": "the split-TF32 factor's selected inverse is FP32-class; solves are "
                          "refined in FP64"}


def run_batch(args, rank, world, local_rank):
    """Batched workload: 256 independent grids (sides 30..200) as ONE batch split across the
    ranks by factorization work (strong scaling: each rank factors its share as one
    block-diagonal batch; no collective on the data path, per-matrix backward errors
    gathered on the host afterwards).  A step is one factorization of every rank's share;
    the metric is matrices per second of the whole batch."""
    import torch
    import torch.distributed as dist
    import swcholesky_b200 as swc
    from swcholesky_b200 import batch_shard as BS
    from swcholesky_b200 import matrices as M
    from swcholesky_b200 import workloads as W

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    src_all, sides = W.batch_sources(seed=0)
    mats_all = [M.permute_lower(A, p) for A, p in src_all]
    nbatch = len(mats_all)
    costs = [BS.matrix_flops(m) for m in mats_all]
    mine = BS.split_by_cost(costs, world)[rank]
    mats = [mats_all[i] for i in mine]
    src = [src_all[i] for i in mine]
    nmat = len(mats)
    vals_host = np.concatenate([m.data for m in mats])
    h = swc.Handle(local_rank)
    h.batch_analyze(mats)
    vals = torch.from_numpy(vals_host).to(dev)
    b_host = np.random.default_rng(rank).standard_normal(h.n)
    b = torch.from_numpy(b_host).to(dev)
    x = torch.zeros_like(b)
    stream = torch.cuda.ExternalStream(h.stream, device=dev)
    tol = 1e-12
    cache = os.path.join(os.environ.get("TMPDIR", "/tmp"), "swc_batch_tune.txt")

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, world, dev)

    res = {}
    for name, mode in (("fp64", swc.SWC_MODE_FP64), ("mixed", swc.SWC_MODE_MIXED_TF32X3)):
        t0 = time.perf_counter()
        choice, tune_ms = h.batch_autotune(vals, mode, cache)
        tune_s = time.perf_counter() - t0
        last = {}

        def fact():
            assert h.factor(vals, mode) == 0

        def fact_solve():
            fact()
            _, berr, it, meth = h.refine(b, tol=tol, maxit=60, out=x)
            last.update(iters=it, method=meth)

        for _ in range(args.warmup):
            fact_solve()
        ms_f = timed(fact, args.steps)
        clocks = ClockSampler(local_rank)
        clocks.start()
        ms_fs = timed(fact_solve, args.steps)
        clk = clocks.stop()
        per = h.batch_berr(b, x)
        prof = h.profile(vals, mode)
        per_all = BS.gather_results(mine, per, nbatch, world)
        res[name] = {"ms_factor": round(ms_f, 4),
                     "matrices_per_s_factor": round(nbatch / (ms_f * 1e-3), 1),
                     "ms_factor_plus_refined_solve": round(ms_fs, 4),
                     "matrices_per_s_factor_plus_solve": round(nbatch / (ms_fs * 1e-3), 1),
                     "refine_iterations": last.get("iters"),
                     "berr_max": float(per_all.max()), "berr_median": float(np.median(per_all)),
                     "autotune": {"partition": choice[0], "plan": choice[1],
                                  "best_ms": round(tune_ms, 4), "seconds": round(tune_s, 2)},
                     "launches": h.launches,
                     "classes": {k: {"launches": v[0], "ms": round(v[1], 4),
                                     "gflop": round(v[2] / 1e9, 4)} for k, v in prof.items()},
                     "clocks": clk}
    # e2e: host values in, host solution out, FP64 factor + refined solve per step
    e2e = None
    if rank == 0 and not args.no_e2e:
        t_e = []
        for i in range(3):
            t0 = time.perf_counter()
            assert h.factor(vals_host, swc.SWC_MODE_FP64) == 0
            xh, berr, _, _ = h.refine(b_host, tol=tol, maxit=30)
            if i:
                t_e.append(time.perf_counter() - t0)
        te = float(np.mean(t_e))
        e2e = {"value": round(nmat / te, 1), "unit": "matrices/s",
               "h2d_bytes_per_step": int(vals_host.nbytes + b_host.nbytes),
               "d2h_bytes_per_step": int(b_host.nbytes), "ms_per_step": round(te * 1e3, 3)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.ref_available():
            threads = os.cpu_count() or 1
            tot, cnt, t0 = 0.0, 0, time.time()
            for A, p in src:
                tref, _, _, _ = reference_time(A, p, threads, budget_s=0.0, max_reps=1)
                tot += tref
                cnt += 1
                if time.time() - t0 > 15.0:
                    break
            cpu = {"value": round(cnt / tot, 2), "unit": "matrices/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"first {cnt} of the {nmat} matrices, one reference FP64 "
                             f"factorization each (sw_cholesky_left_par_05_check + OpenBLAS)"}
    if rank == 0:
        f64 = res["fp64"]
        line = {
            "metric": "batched factorization throughput (matrices/s), FP64, 256 SPD grids "
                      "n 900..40,000, one graph replay per batch",
            "value": f64["matrices_per_s_factor"], "unit": "matrices/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": f64["ms_factor"],
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded weighted grids, own nested dissection and symbolic)",
            "config": {"workload": "batch256", "matrices": nbatch,
                       "sides": [int(sides.min()), int(sides.max())],
                       "l2": "inputs larger than L2 (L of the whole batch above 126 MB)"},
            "parallelism": (f"one batch split across {world} GPUs by factorization flops "
                            f"(rank 0: {nmat} matrices, n {int(h.n)})") if world > 1
                           else "single GPU",
            "modes": res, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(f64["launches"] * args.steps),
            "clocks": f64["clocks"],
        }
        print(json.dumps(line))
    h.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="grid3d_60")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mode", default="mixed", choices=["mixed", "bf16", "fp64"],
                    help="mixed: split-TF32 Schur updates; bf16: BF16x3; fp64")
    ap.add_argument("--nrhs", type=int, default=1, help="right-hand sides per refined solve")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the per-configuration records after the headline")
    ap.add_argument("--no-single-thread", action="store_true",
                    help="skip the 1-thread reference timing of the CPU baseline")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "batch256":
            run_batch(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
