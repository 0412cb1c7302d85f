"""Runs the numeric factorization of a named workload a given number of times.

    python -m swcholesky_b200.run --workload grid3d_60 --mode fp64 --reps 1 [--solve]
                                  [--plan K] [--profile]
    python -m swcholesky_b200.run --workload batch256 --mode mixed --reps 1 [--batch-count 64]

The single-matrix workloads use the supernode partition stored in tests/golden (the
reference's symbolic phase) when present, else the library's own partition; ``batch256``
is the batched workload.  Prints one line with the sizes and the device milliseconds of
the last factorization.  Meant as the command under a profiler: no warm-up, no extra
kernels besides the factorization (and the solve with ``--solve``).  ``--plan`` selects an
execution-plan candidate (``Handle.set_plan``); ``--profile`` adds, after the runs, one
factorization with per-class event timing and the device time of factorizations and
solves (not for use under a profiler).
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import SWC_MODE_FP64, SWC_MODE_MIXED_BF16X3, SWC_MODE_MIXED_TF32X3, Handle
from . import matrices as M
from . import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests",
                      "golden")


def load(name: str, batch_count: int = 256):
    """(problem or list of matrices, values)."""
    if name == "batch256":
        src, _ = W.batch_sources(count=batch_count)
        mats = [M.permute_lower(A, p) for A, p in src]
        return mats, np.concatenate([m.data for m in mats])
    A, perm, _ = W.build(name)
    fx = os.path.join(GOLDEN, f"sym_{name[:-3] if name.endswith('c10') else name}.npz")
    if os.path.exists(fx):
        g = dict(np.load(fx))
        P = W.assemble(A, g["perm"], g["super"])
    else:
        P = W.assemble_own(A, perm)
    return P, P.A2x


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="grid3d_60")
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed", "bf16"])
    ap.add_argument("--plan", type=int, default=0)
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--solve", action="store_true")
    ap.add_argument("--tune-cache", default=None,
                    help="batched workload: autotune (or reuse the cached choice in this file)")
    ap.add_argument("--batch-count", type=int, default=256,
                    help="matrices of the batched workload (a smaller batch for profiling)")
    args = ap.parse_args()
    mode = {"fp64": SWC_MODE_FP64, "mixed": SWC_MODE_MIXED_TF32X3,
            "bf16": SWC_MODE_MIXED_BF16X3}[args.mode]
    prob, vals = load(args.workload, args.batch_count)
    h = Handle(0)
    h.set_plan(args.plan)
    if isinstance(prob, list):
        h.batch_analyze(prob)
        if args.tune_cache:
            choice, best = h.batch_autotune(vals, mode, args.tune_cache)
            print(f"autotune: partition {choice[0]} plan {choice[1]} ({best:.3f} ms)")
    else:
        P = prob
        h.analyze(P.n, P.A2p, P.A2i, P.lC, P.Ls, P.Li_ptr, P.super, P.prunePtr, P.pruneSet)
    import torch
    v = torch.from_numpy(vals).cuda()
    b = torch.from_numpy(np.random.default_rng(0).standard_normal(h.n)).cuda()
    ms = 0.0
    for _ in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = h.factor(v, mode)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        if info:
            raise SystemExit(f"not positive definite at column {info - 1}")
        if args.solve:
            h.refine(b, tol=1e-12)
    print(f"workload {args.workload} n {h.n} nsuper {h.nsuper} xsize {h.xsize} "
          f"launches {h.launches} last factor {ms:.3f} ms (host clock)")
    if args.profile:
        prof = h.profile(v, mode)
        print("classes (launches, device ms): " +
              ", ".join(f"{k} {la} {t:.3f}" for k, (la, t, _, _) in prof.items()))
        st = torch.cuda.ExternalStream(h.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(5):
            h.factor(v, mode)
        e1.record(st)
        torch.cuda.synchronize()
        x = torch.zeros_like(b)
        h.solve(b, out=x)
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(st)
        for _ in range(10):
            h.solve(b, out=x)
        e3.record(st)
        torch.cuda.synchronize()
        print(f"factor {e0.elapsed_time(e1) / 5:.3f} ms, solve {e2.elapsed_time(e3) / 10:.3f} ms "
              f"(device, CUDA events)")
    h.close()


if __name__ == "__main__":
    main()
