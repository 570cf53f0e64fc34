#!/usr/bin/env python
"""Benchmark of the batched sparse CG path on B200.

Workload (one "step"): the batching configuration's 4096 independent 2D
variable-coefficient diffusion systems (5-point finite volume, kappa = exp(g),
g ~ N(0, 0.5^2), sides ~ U{16..128}, seed 2, FP32 CSR packed into one buffer)
solved to a relative residual of 1e-10 by the mixed-precision solver: FP32 CG
on the Jacobi-scaled systems whose residual is replaced by the FP64 residual
b - A x whenever it has dropped by 0.01 (reliable updates), FP64 solution and
norms, one persistent launch per CTA size. Metric: solves/s. The same line
also carries plain FP64 batched CG on the same batch (the comparison named by
the metric, on the same diagonal layout and CTA tiers), the mixed solve on the
sliced layout (patterns that are not stencils), SpMV GB/s on the 1024^2
Poisson matrix (CSR and ELLPACK), Jacobi-CG on that matrix (configuration 2),
the 256^3 precision configuration (FP32 / BF16 values with FP64 residual
replacement against plain FP64, true residuals), the reference's own
benchmark shapes beside its published times, the roofline of the dominant
kernel, the CPU baseline (the reference's bundled Eigen FP64 Jacobi-CG, all
host threads) and the end-to-end number through the public API with host
buffers. A short summary closes the line ("headline").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
N > 1: launch with torch.distributed.run; every rank solves its own batch
(seed 2 + rank), no collective on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_SYS, SIDE_LO, SIDE_HI, SIGMA, SEED = 4096, 16, 128, 0.5, 2
INNER_TOL, OUTER_TOL, MAX_OUTER = 1e-4, 1e-10, 30
METRIC = "CG solves/s at 1e-10 rel. residual (mixed FP32/FP64-refined, batched)"
UNIT = "solves/s"
L2_BYTES = 126 * 1024 * 1024


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "of measured"
    return 6650.0, "of fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
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

    def summary(self):
        if self.proc is None or self.f is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [c.strip() for c in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_setup(gpus: int):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(world, v: float) -> float:
    """Largest value over all ranks (device timing: the slowest rank sets the step)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int) -> int:
    """Every rank solves its own batch of the batching configuration: seed 2 + rank
    (independent systems shard with no exchange; weak scaling)."""
    return SEED + rank


def whole_job_rate(units_per_rank: int, world: int, ms_max: float) -> float:
    """Units of all ranks per second of the slowest rank."""
    return units_per_rank * world / (ms_max / 1e3)


# ---------------------------------------------------------------------------
# algorithmic bytes (per unit)
# ---------------------------------------------------------------------------

def refined_bytes(bt, inner_iters, outer_steps, inner_value_bytes=4):
    """Per system s: each inner Jacobi-CG iteration streams the matrix
    (nnz * (value + 4-byte column) + (n + 1) * 4) plus 13 FP32 n-vectors (the
    three-pass schedule); each refinement step streams the FP32 matrix once more
    in FP64 arithmetic plus 3 FP64 n-vectors (read x, b; write the residual)."""
    n = np.diff(bt.row_off).astype(np.float64)
    nnz = (bt.row_ptr[bt.row_off[1:]] - bt.row_ptr[bt.row_off[:-1]]).astype(np.float64)
    b_iter = nnz * (inner_value_bytes + 4) + (n + 1) * 4 + 13 * n * 4
    b_outer = nnz * (4 + 4) + (n + 1) * 4 + 3 * n * 8
    return float(np.sum(inner_iters * b_iter + outer_steps * b_outer))


def plain_bytes(bt, iters, vbytes=8, vecbytes=8):
    n = np.diff(bt.row_off).astype(np.float64)
    nnz = (bt.row_ptr[bt.row_off[1:]] - bt.row_ptr[bt.row_off[:-1]]).astype(np.float64)
    return float(np.sum(iters * (nnz * (vbytes + 4) + (n + 1) * 4 + 13 * n * vecbytes)))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def time_device(fn, steps, warmup, stream, world):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = start.elapsed_time(end) / steps
    return max_over_ranks(world, ms)


def spmv_gbs(cm, torch, dev, stream):
    """SpMV y = A x on the 1024^2 Poisson matrix (configuration 2), CSR and
    ELLPACK, over enough matrix copies to exceed L2 (no reuse between calls)."""
    from cumat_b200 import problems as P
    pr = P.poisson2d(1024, 1)
    n, nnz = pr.n, pr.nnz
    idx, ev = P.csr_to_ell(n, pr.row_ptr, pr.col, pr.val)
    csr_bytes = nnz * 8 + (n + 1) * 4 + 2 * n * 4
    ell_bytes = n * 5 * 8 + 2 * n * 4
    copies = int(np.ceil(3 * L2_BYTES / csr_bytes)) + 1
    mats_c, mats_e, xs, ys = [], [], [], []
    for c in range(copies):
        p = cm.SparsityPattern.csr(n, n, pr.row_ptr, pr.col)
        mats_c.append(cm.SparseMatrix(p).setData(pr.val))
        pe = cm.SparsityPattern.ell(n, n, idx)
        mats_e.append(cm.SparseMatrix(pe).setData(ev))
        xs.append(torch.from_numpy(pr.b).to(dev))
        ys.append(torch.empty(n, device=dev))
    out = {}
    for name, mats, byt in [("csr", mats_c, csr_bytes), ("ell", mats_e, ell_bytes)]:
        for i in range(copies):  # warm-up
            mats[i].product(xs[i], out=ys[i])
        torch.cuda.synchronize()
        reps = 100
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for r in range(reps):
            i = r % copies
            mats[i].product(xs[i], out=ys[i])
        e.record(stream)
        torch.cuda.synchronize()
        us = s.elapsed_time(e) * 1000.0 / reps
        out[name] = {"us": round(us, 3), "gbs": round(byt / us / 1e3, 1), "alg_bytes": byt, "copies": copies}
    return out


# The reference's own published benchmarks (ms per call, RTX 2070, from
# benchmarks/CSRMV - 2D-Poisson Matrix.json and benchmarks/Conjugate Gradient -
# 2D-Poisson Matrix.json; see docs/03_Benchmarks.dox)
REF_CSRMV_MS = {10: (0.0178, 0.0136), 100: (0.0160, 0.0151), 1000: (0.1635, 0.1444), 10000: (17.69, 19.62)}
REF_CG_MS = {10: 6.67, 20: 11.47, 50: 28.58, 100: 48.60, 200: 74.14, 500: 201.58, 1000: 599.84}
# benchmarks/Linear Combination - Constant Size.json / Constant Count.json and
# benchmarks/Dotproduct.json ("CuMat" rows; the dot includes reading the result)
REF_LINCOMB_SIZE_MS = [0.03682, 0.04331, 0.05314, 0.06548, 0.0775, 0.09306, 0.09788, 0.10953, 0.12119, 0.13133]
REF_LINCOMB_COUNT_MS = {100: 0.01513, 1000: 0.01483, 10000: 0.01967, 100000: 0.01702, 1000000: 0.04742,
                        10000000: 0.33869, 50000000: 2.00751}
REF_DOT_MS = {10: 0.11192, 100: 0.14819, 1000: 0.16076, 10000: 0.16291, 100000: 0.14098, 1000000: 0.16244,
              10000000: 0.39226, 100000000: 2.37392}


def _boundary_rhs(g: int) -> np.ndarray:
    """Right-hand side of the reference's CG benchmark
    (benchmarks/conjugate_gradient/Implementation_cuMat.cu): zero inside,
    rand()/RAND_MAX on the boundary cells after srand(42), in the order
    x-major then y, cell index y + x * g. The C library's own rand() is called."""
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(42)
    rand_max = 2147483647.0
    b = np.zeros(g * g, np.float32)
    for x in range(g):
        for y in range(g):
            if x == 0 or y == 0 or x == g - 1 or y == g - 1:
                b[y + x * g] = np.float32(libc.rand()) / np.float32(rand_max)
    return b


def reference_suite(cm, torch, dev, stream, hbm_peak):
    """The reference's own benchmark shapes, timed here like the reference times
    them: CSR / ELLPACK SpMV on the 2D Poisson matrix (grids 10..10000), repeated
    calls on one matrix and vector, ms per call; CG on the 2D Poisson matrix
    (grids 10..1000, default Jacobi preconditioner, tolerance 1e-4), solver
    construction + solve, ms per call (wall clock around a device sync), and
    the solve alone on a solver built once (CUDA events)."""
    from cumat_b200 import problems as P

    def ev_ms(fn, reps, warm=3):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    out = {"source": "reference ms per call on an RTX 2070 (benchmarks/*.json); ours on this B200",
           "spmv": [], "cg": []}
    for g in (10, 100, 1000, 10000):
        pr = P.poisson2d(g, 1)
        n, nnz = pr.n, pr.nnz
        A = cm.SparseMatrix(cm.SparsityPattern.csr(n, n, pr.row_ptr, pr.col)).setData(pr.val)
        idx, ev = P.csr_to_ell(n, pr.row_ptr, pr.col, pr.val)
        E = cm.SparseMatrix(cm.SparsityPattern.ell(n, n, idx)).setData(ev)
        del idx, ev
        x = torch.from_numpy(pr.b).to(dev)
        y = torch.empty_like(x)
        reps = 2000 if n < 10 ** 6 else (200 if n < 10 ** 7 else 20)
        tc = ev_ms(lambda: A.product(x, out=y), reps)
        te = ev_ms(lambda: E.product(x, out=y), reps)
        csr_b = nnz * 8 + (n + 1) * 4 + 2 * n * 4
        ell_b = n * 5 * 8 + 2 * n * 4
        rc, re = REF_CSRMV_MS[g]
        out["spmv"].append({"grid": g, "rows": n, "csr_ms": round(tc, 5), "ell_ms": round(te, 5),
                            "csr_gbs": round(csr_b / tc / 1e6, 1), "ell_gbs": round(ell_b / te / 1e6, 1),
                            "csr_frac": round(csr_b / tc / 1e6 / hbm_peak, 3),
                            "ell_frac": round(ell_b / te / 1e6 / hbm_peak, 3),
                            "ref_csr_ms": rc, "ref_ell_ms": re,
                            "speedup_csr": round(rc / tc, 1), "speedup_ell": round(re / te, 1)})
        del A, E, x, y, pr
        torch.cuda.empty_cache()
    for g in sorted(REF_CG_MS):
        pr = P.poisson2d(g, 0)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        b = torch.from_numpy(_boundary_rhs(g)).to(dev)
        x = torch.empty_like(b)
        its = []

        def run():
            cg = cm.ConjugateGradient(A).setTolerance(1e-4)
            cg.solve(b, out=x)
            its.append(cg.iterations())
        run()
        torch.cuda.synchronize()
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            run()
            torch.cuda.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
        ms = statistics.mean(times)
        # the solve alone on a solver built once (the construction's share is
        # ms - solve_ms)
        cg = cm.ConjugateGradient(A).setTolerance(1e-4)
        cg.solve(b, out=x)
        solve_ms = ev_ms(lambda: cg.solve(b, out=x), 3, warm=1)
        out["cg"].append({"grid": g, "ms": round(ms, 4), "iterations": int(its[-1]), "ref_ms": REF_CG_MS[g],
                          "speedup": round(REF_CG_MS[g] / ms, 1), "solve_ms": round(solve_ms, 4),
                          "us_per_iter": round(solve_ms * 1e3 / max(1, cg.iterations()), 2)})
    # linear combinations of FP32 vectors U[0, 1) (the reference's benchmark expression)
    out["lincomb"] = []
    gen = torch.Generator(device=dev).manual_seed(7)

    def lincomb_case(n, k, ref):
        vs = [torch.rand(n, device=dev, generator=gen) for _ in range(k)]
        fs = torch.rand(k, generator=torch.Generator().manual_seed(k)).tolist()
        o = torch.empty(n, device=dev)
        t = ev_ms(lambda: cm.linear_combination(fs, vs, out=o), 200 if n <= 10 ** 7 else 50)
        byt = (k + 1) * n * 4
        out["lincomb"].append({"n": n, "terms": k, "ms": round(t, 5), "gbs": round(byt / t / 1e6, 1),
                               "frac": round(byt / t / 1e6 / hbm_peak, 3), "ref_ms": ref, "speedup": round(ref / t, 1)})
    for k in range(1, 11):
        lincomb_case(10 ** 6, k, REF_LINCOMB_SIZE_MS[k - 1])
    for n, ref in REF_LINCOMB_COUNT_MS.items():
        lincomb_case(n, 2, ref)
    # dot product including the device-to-host read of the result, like the reference's timing
    out["dot"] = []
    for n, ref in REF_DOT_MS.items():
        x = torch.rand(n, device=dev, generator=gen)
        y = torch.rand(n, device=dev, generator=gen)
        h = torch.empty(()).pin_memory()

        def dot_read():
            h.copy_(cm.dot(x, y), non_blocking=True)
            torch.cuda.current_stream().synchronize()
        for _ in range(5):
            dot_read()
        reps = 200 if n <= 10 ** 7 else 50
        t0 = time.perf_counter()
        for _ in range(reps):
            dot_read()
        t = (time.perf_counter() - t0) * 1e3 / reps
        out["dot"].append({"n": n, "ms": round(t, 5), "gbs": round(2 * n * 4 / t / 1e6, 1), "ref_ms": ref,
                           "speedup": round(ref / t, 1)})
    return out


# DRAM bytes per algorithmic (streaming-model) byte of k_mixed_fast, measured
# by ncu (dram__bytes_read.sum + dram__bytes_write.sum over the three CTA-tier
# launches: 577.3 MB) on the first 512 systems of this batch, whose streaming
# model is 136.48 GB (`python bench.py --profile-small`); DRAM traffic grows
# with the work, so the full launch's traffic is this ratio times its model
# bytes. Source capture: the k_mixed_fast profile summary under profiles/.
DRAM_PER_MODEL_BYTE = 0.004229

# L1 / shared-memory data-pipe bytes that k_mixed_fast moves per row and inner
# iteration on a 5-point system in the diagonal block layout with the unit
# middle diagonal: 4 value loads (16 B) and 5 p reads (20 B) in the product,
# r read + write (8 B), p read + write and the x-increment read + write
# (16 B) in the updates. Each FP64 residual replacement moves per row 5 FP32
# values, 5 16-bit columns and 5 FP64 x gathers (70 B), b (8 B) and the new
# FP32 residual (4 B), and its fold x += s * xh (read x, xh, s, write x: 28 B).
L1_BYTES_PER_ROW_ITER = 60
L1_BYTES_PER_ROW_REPLACEMENT = 110
# Nominal L1 data-pipe width: 128 B per clock per SM (32 banks x 4 B).
L1_BYTES_PER_CLK_SM = 128


def l1_model_bytes(bt, inner_iters, outer_steps):
    n = np.diff(bt.row_off).astype(np.float64)
    return float(np.sum(n * (inner_iters * L1_BYTES_PER_ROW_ITER + outer_steps * L1_BYTES_PER_ROW_REPLACEMENT)))


def _ev_time(torch, stream, fn, reps, warm=1):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(reps):
        fn()
    e.record(stream)
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def cg_config2(cm, torch, dev, stream, hbm_peak):
    """The plain method at scale: Jacobi-CG on the 1024^2 Poisson matrix
    (FP32 CSR, b ~ U[-1,1] seed 1) to 1e-6, at most 4000 iterations, one
    system (the grid path). Bytes per iteration follow the three-pass
    schedule: the matrix without the x / y terms (nnz * 8 + (n + 1) * 4) plus
    13 FP32 n-vectors; the whole working set (about 70 MB) fits in L2, so the
    GB/s figure is L2-fed, not an HBM number."""
    from cumat_b200 import problems as P
    pr = P.poisson2d(1024, 1)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    cg = cm.ConjugateGradient(A).setTolerance(1e-6).setMaxIterations(4000)
    b = torch.from_numpy(pr.b).to(dev)
    x = torch.empty_like(b)
    ms = _ev_time(torch, stream, lambda: cg.solve(b, out=x), 3)
    it = cg.iterations()
    per_iter = pr.nnz * 8 + (pr.n + 1) * 4 + 13 * pr.n * 4
    gbs = per_iter * it / (ms / 1e3) / 1e9
    out = {"ms": round(ms, 3), "iterations": int(it), "error": cg.error(),
           "iters_per_s": round(it / (ms / 1e3), 1), "us_per_iter": round(ms * 1e3 / it, 2),
           "gbs_model": round(gbs, 1), "frac_model": round(gbs / hbm_peak, 3)}
    # the other grid-path loop on the same system: the cooperative one-launch
    # solve (one CTA per SM, p staged per CTA in shared memory), which the
    # solver picks for systems up to 2^15 rows (CUMAT_CG_COOP=2 forces it)
    old = os.environ.get("CUMAT_CG_COOP")
    os.environ["CUMAT_CG_COOP"] = "2"
    try:
        cgc = cm.ConjugateGradient(A).setTolerance(1e-6).setMaxIterations(4000)
    finally:
        if old is None:
            del os.environ["CUMAT_CG_COOP"]
        else:
            os.environ["CUMAT_CG_COOP"] = old
    before = cm.launch_count()
    cgc.solve(b, out=x)
    launches = cm.launch_count() - before
    msc = _ev_time(torch, stream, lambda: cgc.solve(b, out=x), 3)
    itc = cgc.iterations()
    out["cooperative"] = {"ms": round(msc, 3), "iterations": int(itc), "error": cgc.error(),
                          "us_per_iter": round(msc * 1e3 / itc, 2), "launches_per_solve": int(launches)}
    return out


# benchmarks/batched_reductions_22.json (RTX 2070, ms per call): 2^22 FP32
# values, N of them reduced per output along one axis, the other two axes
# sqrt(2^22 / N) and the rest (benchmarks/batched_reduction/main.cpp:89-153).
# Per N: the reference's default sum (its "Baseline" column) and the fastest
# of its Thread / Warp / Block / Device kernels.
REF_REDUCE_MS = {
    "Row": {2: (33.7065, 0.071104), 16: (4.46387, 0.105552), 128: (0.525456, 0.0472), 1024: (0.165888, 0.045168),
            8192: (0.173024, 0.04704), 65536: (0.216528, 0.221456), 1048576: (2.53859, 0.073376)},
    "Column": {2: (33.7774, 0.077824), 16: (4.3645, 0.054336), 128: (0.475952, 0.045056), 1024: (0.17608, 0.077648),
               8192: (0.195568, 0.058), 65536: (0.213344, 0.314016), 1048576: (2.52806, 0.106976)},
    "Batch": {2: (34.2191, 0.070992), 16: (4.37658, 0.054528), 128: (0.47696, 0.04416), 1024: (0.180176, 0.076672),
              8192: (0.188512, 0.146992), 65536: (0.222464, 0.537232), 1048576: (2.52939, 0.182544)},
}
_REDUCE_AXIS = {"Row": ("rows",), "Column": ("cols",), "Batch": ("batches",)}


def _reduce_shape(axis, n, total):
    """(rows, cols, batches) of the reference's benchmark: N along the reduced
    axis, the others sqrt(total / N) and the rest."""
    o1 = int(np.sqrt(total / n))
    o2 = total // (n * o1)
    return {"Row": (n, o1, o2), "Column": (o1, n, o2), "Batch": (o1, o2, n)}[axis]


def _block_poisson(g, B, seed):
    """3D-vector 2D Poisson in block CSR: on a g x g grid, diagonal blocks
    5 I + C (C symmetric, entries in [-0.1, 0.1]), off-diagonal blocks -I:
    symmetric positive definite (the Laplacian plus a block diagonal with
    eigenvalues above 0.6)."""
    from cumat_b200 import problems as P
    pr = P.poisson2d(g, 0)
    rows = np.repeat(np.arange(pr.n), np.diff(pr.row_ptr))
    blocks = np.broadcast_to(-np.eye(B, dtype=np.float32), (pr.nnz, B, B)).copy()
    diag = rows == pr.col
    C = np.random.default_rng(seed).uniform(-0.1, 0.1, (int(diag.sum()), B, B)).astype(np.float32)
    blocks[diag] = 5 * np.eye(B, dtype=np.float32) + (C + C.transpose(0, 2, 1)) / 2
    return pr.n, pr.row_ptr, pr.col, blocks


def next_rows(cm, torch, dev, stream, hbm_peak):
    """The rows beside the CG path, measured (ms per call through the public
    API, CUDA events after warm-up and the first call's kernel choice):

    reduce        the reference's batched-reduction benchmark (2^22 FP32
                  values along each axis, against its RTX 2070 times)
    reduce_hbm    2^28 FP32 values (1 GiB, beyond L2) reduced along each axis
                  with N = 1024 and fully: GB/s of the input read
    transposed    4096^2 Poisson (FP32, 84 M entries, beyond L2): A x (CSR),
                  A^T x (transposed product) and A x on the same arrays
                  declared CSC, bytes as for the CSR product
    blocked_cg    Jacobi-CG on a 3 x 3-block Poisson matrix (BSR, 512^2
                  blocks, 786,432 rows) to 1e-6: us per iteration
    """
    def ev_ms(fn, reps, warm=3):
        return _ev_time(torch, stream, fn, reps, warm)

    out = {"reduce": [], "reduce_hbm": []}
    gen = torch.Generator(device=dev).manual_seed(5)
    for axis, table in REF_REDUCE_MS.items():
        for n, (ref_def, ref_best) in table.items():
            R, Cc, B = _reduce_shape(axis, n, 1 << 22)
            x = torch.rand((B, Cc, R), device=dev, generator=gen)
            ax = _REDUCE_AXIS[axis]
            t = ev_ms(lambda: cm.reduce(x, "sum", ax), 100)
            out["reduce"].append({"axis": axis, "n": n, "shape_rcb": [R, Cc, B], "ms": round(t, 5),
                                  "ref_default_ms": ref_def, "ref_best_ms": ref_best,
                                  "speedup_vs_default": round(ref_def / t, 1), "speedup_vs_best": round(ref_best / t, 1)})
            del x
    total = 1 << 28
    x = torch.rand(total, device=dev, generator=gen)
    for axis in ("Row", "Column", "Batch", "All"):
        if axis == "All":
            shape, ax = (1 << 10, 1 << 9, 1 << 9), ("rows", "cols", "batches")
        else:
            shape, ax = _reduce_shape(axis, 1024, total), _REDUCE_AXIS[axis]
        R, Cc, B = shape
        xv = x.view(B, Cc, R)
        o = cm.reduce(xv, "sum", ax)
        t = ev_ms(lambda: cm.reduce(xv, "sum", ax), 20)
        byt = (total + o.numel()) * 4
        out["reduce_hbm"].append({"axis": axis, "shape_rcb": [R, Cc, B], "ms": round(t, 4),
                                  "gbs": round(byt / t / 1e6, 1), "frac": round(byt / t / 1e6 / hbm_peak, 3)})
    del x
    torch.cuda.empty_cache()

    from cumat_b200 import problems as P
    pr = P.poisson2d(4096, 1)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    Ac = cm.SparseMatrix(cm.SparsityPattern.csc(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    xv = torch.from_numpy(pr.b).to(dev)
    y = torch.empty_like(xv)
    byt = pr.nnz * 8 + (pr.n + 1) * 4 + 2 * pr.n * 4
    tr = {"rows": pr.n, "nnz": pr.nnz, "alg_bytes": byt}
    for name, fn in (("csr", lambda: A.product(xv, out=y)), ("transposed", lambda: A.transposed_product(xv, out=y)),
                     ("csc", lambda: Ac.product(xv, out=y))):
        t = ev_ms(fn, 20)
        tr[name] = {"ms": round(t, 4), "gbs": round(byt / t / 1e6, 1), "frac": round(byt / t / 1e6 / hbm_peak, 3)}
    out["transposed"] = tr
    del A, Ac, xv, y, pr
    torch.cuda.empty_cache()

    nb, brp, bci, blocks = _block_poisson(512, 3, 3)
    Ab = cm.SparseMatrix(cm.SparsityPattern.bsr(nb, nb, 3, brp, bci)).setData(blocks.reshape(-1))
    n = nb * 3
    b = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, n).astype(np.float32)).to(dev)
    xs = torch.empty_like(b)
    cg = cm.ConjugateGradient(Ab).setTolerance(1e-6)
    cg.solve(b, out=xs)
    t = ev_ms(lambda: cg.solve(b, out=xs), 3, warm=1)
    its = cg.iterations()
    out["blocked_cg"] = {"block": 3, "block_rows": nb, "rows": n, "nnz": int(bci.size) * 9, "iterations": its,
                         "error": cg.error(), "ms": round(t, 3), "us_per_iter": round(t * 1e3 / max(1, its), 2)}
    return out


def cg_poisson10000(cm, torch, dev, stream, hbm_peak):
    """The grid path's iteration on the 10000^2 Poisson matrix (10^8 rows, FP32,
    Jacobi; every vector 400 MB, far above L2): the per-iteration time is the
    difference of two solves capped at 40 and 10 iterations, over 30. At this
    size (vectors far above L2) the product reads p as stored and a separate
    kernel updates it; the diagonal-layout iteration streams 72 B per row:
    product + p.q (5 values, p, q: 28 B), x / r update + |r|^2 + r.z (x, p, r,
    q, 1/diag read, x, r written: 28 B), p update (r, p, 1/diag read, p
    written: 16 B)."""
    from cumat_b200 import problems as P
    pr = P.poisson2d(10000, 1)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    b = torch.from_numpy(pr.b).to(dev)
    x = torch.empty_like(b)
    del pr
    t = {}
    for k in (10, 40):
        cg = cm.ConjugateGradient(A).setTolerance(1e-12).setMaxIterations(k).set_path(2)
        t[k] = _ev_time(torch, stream, lambda: cg.solve(b, out=x), 2)
        its = cg.iterations()
        del cg
    us = (t[40] - t[10]) * 1e3 / 30
    byt = 72.0 * A.rows
    out = {"rows": A.rows, "us_per_iter": round(us, 2), "gbs_model": round(byt / us / 1e3, 1),
           "frac_model": round(byt / us / 1e3 / hbm_peak, 3), "iterations_checked": int(its)}
    del A, b, x
    torch.cuda.empty_cache()
    return out


def precision_c4(cm, torch, dev, stream, reps=2):
    """The precision configuration: 3D 7-point finite-volume system on a 256^3
    grid (kappa = exp(N(0, 1)), seed 3, values exact in FP32), solved to a
    relative residual of 1e-10 by (a) FP32 values + FP32 inner Jacobi-CG with
    FP64 residual replacement, (b) the same with BF16-stored values, and (c)
    plain FP64 Jacobi-CG (FP64 values and vectors); each solution's true
    relative residual |b - A x| / |b| is computed afterwards on the host in FP64
    (scipy CSR product, outside the timed region)."""
    import scipy.sparse as sp
    from cumat_b200 import problems as P
    pr = P.fv3d(256, 1.0, 3)
    n = pr.n
    A64h = sp.csr_matrix((pr.val.astype(np.float64), pr.col, pr.row_ptr), shape=(n, n))
    b64h = pr.b.astype(np.float64)
    bn = float(np.linalg.norm(b64h))
    pat = cm.SparsityPattern.csr(n, n, pr.row_ptr, pr.col)
    A32 = cm.SparseMatrix(pat, dtype=torch.float32).setData(pr.val)
    b64 = torch.from_numpy(b64h).to(dev)
    x = torch.empty_like(b64)
    out = {"rows": n, "nnz": pr.nnz}

    def true_res():
        xh = x.cpu().numpy()
        return float(np.linalg.norm(b64h - A64h @ xh) / bn)

    for name, mat in [("mixed_f32", A32), ("mixed_bf16", None)]:
        if mat is None:
            mat = cm.SparseMatrix(pat, dtype=torch.bfloat16).setData(pr.val)
        cg = cm.ConjugateGradient(mat).setTolerance(1e-4)
        ms = _ev_time(torch, stream, lambda: cg.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=60, out=x),
                      reps)
        st = cg.system_stats()
        out[name] = {"ms": round(ms, 2), "inner_iterations": int(st["iterations"].max()),
                     "replacements": int(st["outer"].max()), "status": int(st["status"].max()),
                     "fp32_fallback": int(st["fallback"].max()),
                     "reported_error": float(st["error"].max()), "true_rel_residual": true_res()}
        del cg
    A64 = cm.SparseMatrix(pat, dtype=torch.float64).setData(pr.val.astype(np.float64))
    cg64 = cm.ConjugateGradient(A64).setTolerance(1e-10).setMaxIterations(20000)
    ms = _ev_time(torch, stream, lambda: cg64.solve(b64, out=x), reps)
    out["fp64"] = {"ms": round(ms, 2), "iterations": int(cg64.iterations()), "reported_error": cg64.error(),
                   "true_rel_residual": true_res()}
    out["ratio_f32"] = round(out["fp64"]["ms"] / out["mixed_f32"]["ms"], 3)
    out["ratio_bf16"] = round(out["fp64"]["ms"] / out["mixed_bf16"]["ms"], 3)
    del cg64, A64, A32
    torch.cuda.empty_cache()
    return out


def cpu_baseline(bt, budget_s=15.0):
    """Eigen FP64 Jacobi-CG to 1e-10 (the reference's bundled CPU path) on the
    first m systems of the batch (sides are drawn i.i.d., so a prefix is a
    random sample), OpenMP-parallel over systems on all host threads; m is
    sized from a short probe run to take about budget_s seconds."""
    from oracle import oracle as O
    if O.ref_lib() is None:
        return None
    b64 = bt.b.astype(np.float64)
    x64 = np.zeros_like(b64)
    ep = O.EigenPacked(bt.row_off, bt.row_ptr, bt.col, bt.val)
    threads = O.ref_threads()
    m0 = min(bt.n_sys, max(2 * threads, 32))
    t0, _, _ = ep.solve(0, m0, b64, x64, OUTER_TOL, -1, 1, threads)
    m = int(min(bt.n_sys, max(m0, m0 / max(t0, 1e-9) * budget_s)))
    t, it, err = ep.solve(0, m, b64, x64, OUTER_TOL, -1, 1, threads)
    return {"value": round(m / t, 3), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"first {m} of {bt.n_sys} systems, Eigen 3.3.90 ConjugateGradient<SparseMatrix<double,"
                      f"RowMajor>, Lower|Upper, DiagonalPreconditioner> to 1e-10, OpenMP over systems, {t:.1f} s"}


def run_ours(args):
    import torch

    import cumat_b200 as cm
    from cumat_b200 import problems as P

    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    hbm_peak, peak_src = peaks()
    bt = P.fv2d_batch(N_SYS, SIDE_LO, SIDE_HI, SIGMA, rank_seed(rank))
    p = cm.SparsityPattern.csr(bt.n, bt.n, bt.row_ptr, bt.col)
    p.set_systems(bt.row_off)
    A32 = cm.SparseMatrix(p, dtype=torch.float32).setData(bt.val)
    cg = cm.ConjugateGradient(A32).setTolerance(INNER_TOL)
    b64 = torch.from_numpy(bt.b.astype(np.float64)).to(dev)
    x64 = torch.empty_like(b64)

    def step():
        cg.solve_refined(b64, outer=A32, outer_tol=OUTER_TOL, max_outer=MAX_OUTER, out=x64)

    launches0 = cm.launch_count()
    with Clocks(local) as clk:
        ms = time_device(step, args.steps, args.warmup, stream, world)
    launches = (cm.launch_count() - launches0) // (args.steps + args.warmup) * args.steps
    st = cg.system_stats()
    assert np.all(st["status"] == 0), "some systems did not converge"
    assert float(st["error"].max()) < OUTER_TOL
    value = whole_job_rate(N_SYS, world, ms)
    # roofline of the dominant (only) kernel, k_mixed_fast: bound by the L1 /
    # shared-memory data pipe (vectors live in shared memory, the values of the
    # systems in flight in L2); the streaming model is kept as model_speedup
    inner = st["iterations"].astype(np.float64)
    outer = st["outer"].astype(np.float64)
    alg = refined_bytes(bt, inner, outer)
    l1_bytes = l1_model_bytes(bt, inner, outer)
    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
    clk_sum = clk.summary()
    sm_mhz = clk_sum.get("sm_mhz") or 1965.0
    l1_peak = L1_BYTES_PER_CLK_SM * sm_count * sm_mhz * 1e6 / 1e9
    l1_achieved = l1_bytes / (ms / 1e3) / 1e9
    traffic = alg * DRAM_PER_MODEL_BYTE

    # plain FP64 batched CG on the same batch (FP64 values and vectors)
    A64 = cm.SparseMatrix(p, dtype=torch.float64).setData(bt.val.astype(np.float64))
    cg64 = cm.ConjugateGradient(A64).setTolerance(OUTER_TOL)
    xp = torch.empty_like(b64)
    ms64 = time_device(lambda: cg64.solve(b64, out=xp), max(1, args.steps // 2), 1, stream, world)
    st64 = cg64.system_stats()
    fp64 = {"value": round(N_SYS * world / (ms64 / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms64, 3),
            "converged": int((st64["status"] == 0).sum()), "max_error": float(st64["error"].max()),
            "iterations_max": int(st64["iterations"].max()),
            "gbs_alg": round(plain_bytes(bt, st64["iterations"].astype(np.float64)) / (ms64 / 1e3) / 1e9, 1)}

    # the same mixed solve on the sliced layout (CUMAT_CG_DIA=0, read when the
    # solver is created): the number for patterns that are not stencils
    os.environ["CUMAT_CG_DIA"] = "0"
    cg_sl = cm.ConjugateGradient(A32).setTolerance(INNER_TOL)
    del os.environ["CUMAT_CG_DIA"]
    ms_sl = time_device(lambda: cg_sl.solve_refined(b64, outer=A32, outer_tol=OUTER_TOL, max_outer=MAX_OUTER, out=xp),
                        max(1, args.steps // 2), 1, stream, world)
    st_sl = cg_sl.system_stats()
    sliced = {"value": round(N_SYS * world / (ms_sl / 1e3), 1), "unit": UNIT, "ms_per_step": round(ms_sl, 3),
              "converged": int((st_sl["status"] == 0).sum()), "max_error": float(st_sl["error"].max())}
    del cg_sl

    # end to end through the public API with pinned host buffers: every step
    # copies its right-hand sides in and its solutions out; the copies run on
    # a copy stream with two device buffers each, so step k + 1's upload and
    # step k - 1's download overlap step k's solve (as a stream of batches
    # would run in an application)
    hb = torch.from_numpy(bt.b.astype(np.float64)).pin_memory()
    hx = [torch.empty(bt.n, dtype=torch.float64).pin_memory() for _ in range(2)]
    db = [torch.empty_like(b64) for _ in range(2)]
    dx = [torch.empty_like(b64) for _ in range(2)]
    copy = torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_run(steps):
        with torch.cuda.stream(copy):
            db[0].copy_(hb, non_blocking=True)
            ev_in[0].record(copy)
        for i in range(steps):
            j = i % 2
            if i + 1 < steps:
                with torch.cuda.stream(copy):
                    if i >= 1:
                        copy.wait_event(ev_done[1 - j])   # the solve that read db[1 - j]
                    db[1 - j].copy_(hb, non_blocking=True)
                    ev_in[1 - j].record(copy)
            stream.wait_event(ev_in[j])
            if i >= 2:
                stream.wait_event(ev_out[j])              # dx[j]'s previous download
            cg.solve_refined(db[j], outer=A32, outer_tol=OUTER_TOL, max_outer=MAX_OUTER, out=dx[j])
            ev_done[j].record(stream)
            with torch.cuda.stream(copy):
                copy.wait_event(ev_done[j])
                hx[j].copy_(dx[j], non_blocking=True)
                ev_out[j].record(copy)
        stream.wait_stream(copy)

    e2e_run(2)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    copy.wait_stream(stream)   # the first upload starts inside the timed region
    e2e_run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_e2e = max_over_ranks(world, e0.elapsed_time(e1) / args.steps)
    assert np.array_equal(hx[(args.steps - 1) % 2].numpy(), x64.cpu().numpy()), "end-to-end result differs"

    extra = {}
    if rank == 0 and world == 1 and not args.no_spmv:
        extra["spmv_poisson1024"] = spmv_gbs(cm, torch, dev, stream)
        for k in ("csr", "ell"):
            extra["spmv_poisson1024"][k]["frac"] = round(extra["spmv_poisson1024"][k]["gbs"] / hbm_peak, 3)
    if rank == 0 and world == 1 and not args.no_suite:
        extra["reference_suite"] = reference_suite(cm, torch, dev, stream, hbm_peak)
    if rank == 0 and world == 1 and not args.no_configs:
        extra["cg_poisson1024"] = cg_config2(cm, torch, dev, stream, hbm_peak)
        extra["cg_poisson10000"] = cg_poisson10000(cm, torch, dev, stream, hbm_peak)
        extra["precision_c4"] = precision_c4(cm, torch, dev, stream)
    if rank == 0 and world == 1 and not args.no_next:
        extra["next_rows"] = next_rows(cm, torch, dev, stream, hbm_peak)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(bt, args.cpu_budget)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded finite-volume systems)",
            "config": {"workload": "4096 uneven 2D FV diffusion systems (sides 16..128, kappa=exp(N(0,0.25))), "
                                   "Jacobi-scaled FP32 CG with FP64 residual replacement to 1e-10",
                       "systems_per_gpu": N_SYS, "rows_per_gpu": int(bt.n), "nnz_per_gpu": int(bt.nnz),
                       "parallelism": f"batch sharding x{world}, no collective",
                       "l2": "inputs larger than L2 (FP32 CSR batch %.2f GB)" % ((bt.nnz * 8 + bt.n * 4) / 1e9)},
            "roofline": {"bound": "l1_pipe", "achieved": round(l1_achieved, 1), "peak": round(l1_peak, 1),
                         "unit": "GB/s", "frac": round(l1_achieved / l1_peak, 3), "traffic": round(traffic),
                         "kernel": "k_mixed_fast",
                         "peak_source": f"nominal 128 B/clk/SM x {sm_count} SMs x median sampled SM clock {sm_mhz} MHz",
                         "l1_bytes_per_launch": l1_bytes,
                         "dram_frac": round(traffic / (ms / 1e3) / 1e9 / hbm_peak, 4),
                         "dram_peak_gbs": hbm_peak, "dram_peak_source": peak_src,
                         "model_speedup": round(alg / (ms / 1e3) / 1e9 / hbm_peak, 3),
                         # l1tex__data_pipe_lsu_wavefronts pct of peak per CTA tier, from the
                         # k_mixed_fast ncu capture of the first 512 systems (--profile-small)
                         "ncu_l1_pipe_pct_by_tier": {"1024": 54.5, "512": 32.7, "256": 19.3},
                         "note": "achieved = L1-pipe model bytes (60 B per row and inner iteration) / time; traffic = "
                                 "DRAM bytes per launch scaled from an ncu capture; model_speedup = HBM streaming "
                                 "model time / measured time"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(N_SYS * world / (ms_e2e / 1e3), 1), "unit": UNIT,
                    "h2d_bytes_per_step": int(bt.n * 8), "d2h_bytes_per_step": int(bt.n * 8)},
            "gpu_launches": int(launches),
            "clocks": clk_sum,
            "fp64_plain": fp64,
            "mixed_vs_fp64": round(value / fp64["value"], 3),
            "mixed_sliced_layout": sliced,
            "solve_stats": {"inner_iterations_max": int(st["iterations"].max()),
                            "inner_iterations_mean": round(float(st["iterations"].mean()), 1),
                            "outer_steps_max": int(st["outer"].max()), "max_error": float(st["error"].max())},
            **extra,
        }
        # short summary last, so that it survives in any tail of the line
        hl = {"mixed_vs_fp64": line["mixed_vs_fp64"], "fp64_solves_s": fp64["value"],
              "mixed_sliced_solves_s": sliced["value"],
              "e2e_solves_s": line["e2e"]["value"], "l1_frac": line["roofline"]["frac"],
              "dram_frac": line["roofline"]["dram_frac"]}
        if "spmv_poisson1024" in extra:
            sp_ = extra["spmv_poisson1024"]
            hl.update(spmv_csr_gbs=sp_["csr"]["gbs"], spmv_ell_gbs=sp_["ell"]["gbs"],
                      spmv_csr_frac=sp_["csr"]["frac"], spmv_ell_frac=sp_["ell"]["frac"])
        if "cg_poisson1024" in extra:
            c2 = extra["cg_poisson1024"]
            hl.update(c2_iters=c2["iterations"], c2_ms=c2["ms"], c2_us_per_iter=c2["us_per_iter"])
        if "cg_poisson10000" in extra:
            hl.update(cg10000_us_per_iter=extra["cg_poisson10000"]["us_per_iter"],
                      cg10000_frac=extra["cg_poisson10000"]["frac_model"])
        if "precision_c4" in extra:
            c4 = extra["precision_c4"]
            hl.update(c4_f32_ms=c4["mixed_f32"]["ms"], c4_bf16_ms=c4["mixed_bf16"]["ms"], c4_fp64_ms=c4["fp64"]["ms"],
                      c4_ratio_f32=c4["ratio_f32"], c4_ratio_bf16=c4["ratio_bf16"],
                      c4_true_res=[c4["mixed_f32"]["true_rel_residual"], c4["mixed_bf16"]["true_rel_residual"],
                                   c4["fp64"]["true_rel_residual"]])
        if "next_rows" in extra:
            nr = extra["next_rows"]
            hl.update(reduce_hbm_frac={r["axis"]: r["frac"] for r in nr["reduce_hbm"]},
                      reduce_speedup_vs_best_min=min(r["speedup_vs_best"] for r in nr["reduce"]),
                      transposed_frac=nr["transposed"]["transposed"]["frac"], csc_frac=nr["transposed"]["csc"]["frac"],
                      blocked_cg_us_per_iter=nr["blocked_cg"]["us_per_iter"])
        line["headline"] = hl
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# reference arm: the reference's bundled Eigen CPU path on the host cores
# ---------------------------------------------------------------------------

def _standalone_generators():
    """The seeded generators without importing the package (whose import maps
    the CUDA library): cumat_b200/problems.py loaded by path and pointed at the
    oracle's own build of the same generator source (oracle/libgen.so)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_cmgen", ROOT / "cumat_b200" / "problems.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["_cmgen"] = mod   # (its dataclasses look their module up)
    spec.loader.exec_module(mod)
    lib = ROOT / "oracle" / "libgen.so"
    if not lib.exists():
        raise RuntimeError(f"{lib} missing: run `make -C oracle`")
    mod._LIB_PATH = lib
    return mod


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    P = _standalone_generators()
    if O.ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libeigen_ref.so (bundled Eigen) not built"}))
        return
    bt = P.fv2d_batch(N_SYS, SIDE_LO, SIDE_HI, SIGMA, SEED)
    ep = O.EigenPacked(bt.row_off, bt.row_ptr, bt.col, bt.val)
    b64 = bt.b.astype(np.float64)
    x64 = np.zeros_like(b64)
    threads = O.ref_threads()
    # each step solves the whole batch (a few seconds on a server host); a host
    # so slow that K + W such steps would exceed the time budget gets a prefix
    # of the batch per step instead (sides are i.i.d., a prefix is a sample)
    t_probe, _, _ = ep.solve(0, min(N_SYS, 64), b64, x64, OUTER_TOL, -1, 1, threads)
    est_full = t_probe * N_SYS / min(N_SYS, 64)
    per_step = N_SYS if est_full * (args.steps + args.warmup) < 180 else \
        max(64, int(N_SYS * 180 / (est_full * (args.steps + args.warmup))))
    times, solved = [], 0
    for i in range(args.warmup + args.steps):
        s0 = 0
        dt, it, err = ep.solve(s0, s0 + per_step, b64, x64, OUTER_TOL, -1, 1, threads)
        if i >= args.warmup:
            times.append(dt)
            solved += per_step
    secs = sum(times)
    value = solved / secs
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded finite-volume systems)",
            "impl": "reference",
            "config": {"workload": "4096 uneven 2D FV diffusion systems (sides 16..128, kappa=exp(N(0,0.25))), "
                                   "Eigen FP64 Jacobi-CG to 1e-10", "systems_per_step": per_step},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"first {per_step} of {N_SYS} systems per step, Eigen 3.3.90 "
                                       f"ConjugateGradient<SparseMatrix<double,RowMajor>, Lower|Upper, "
                                       f"DiagonalPreconditioner> to 1e-10, OpenMP over systems"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_profile_small():
    """The small case for ncu captures (a few hundred MB on the device): three
    SpMV calls per format on the 1024^2 Poisson matrix, one grid-path Jacobi-CG
    solve of that matrix capped at 50 iterations (the cooperative one-launch
    kernel), then one mixed and one FP64 batched solve of the first 512 systems
    of the batch. Prints the algorithmic bytes of the mixed launch so that its
    DRAM traffic can be compared per unit with the full batch."""
    import torch

    import cumat_b200 as cm
    from cumat_b200 import problems as P
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    pr = P.poisson2d(1024, 1)
    A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
    idx, ev = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
    E = cm.SparseMatrix(cm.SparsityPattern.ell(pr.n, pr.n, idx)).setData(ev)
    x = torch.from_numpy(pr.b).to(dev)
    y = torch.empty_like(x)
    for _ in range(3):
        A.product(x, out=y)
        E.product(x, out=y)
    cgg = cm.ConjugateGradient(A).setTolerance(1e-12).setMaxIterations(50).set_path(2)
    cgg.solve(x, out=y)
    bt = P.fv2d_batch(N_SYS, SIDE_LO, SIDE_HI, SIGMA, SEED)
    k = int(bt.row_off[512])
    kz = int(bt.row_ptr[k])
    row_off = bt.row_off[:513]
    p = cm.SparsityPattern.csr(k, k, bt.row_ptr[:k + 1], bt.col[:kz])
    p.set_systems(row_off)
    A32 = cm.SparseMatrix(p).setData(bt.val[:kz])
    cg = cm.ConjugateGradient(A32).setTolerance(INNER_TOL)
    b64 = torch.from_numpy(bt.b[:k].astype(np.float64)).to(dev)
    cg.solve_refined(b64, outer=A32, outer_tol=OUTER_TOL, max_outer=MAX_OUTER)
    A64 = cm.SparseMatrix(p, dtype=torch.float64).setData(bt.val[:kz].astype(np.float64))
    cg64 = cm.ConjugateGradient(A64).setTolerance(OUTER_TOL)
    cg64.solve(b64)
    torch.cuda.synchronize()
    st = cg.system_stats()

    class _Sub:
        pass
    sub = _Sub()
    sub.row_off, sub.row_ptr = row_off, bt.row_ptr[:k + 1]
    print(json.dumps({"profile_small": True, "systems": 512, "rows": k, "nnz": kz,
                      "mixed_alg_bytes": refined_bytes(sub, st["iterations"].astype(np.float64),
                                                       st["outer"].astype(np.float64)),
                      "mixed_converged": bool(np.all(st["status"] == 0)),
                      "fp64_converged": bool(np.all(cg64.system_stats()["status"] == 0))}))


def run_profile_case(case: str):
    """Small single-purpose workloads for one-kernel ncu captures (each well
    above L2 in its streamed data, a few GB on the device at most):

    grid3d      the 160^3 3D system (kappa = exp(N(0, 1)), seed 3) on the grid
                path: plain FP64 Jacobi-CG and the mixed FP32 / FP64 solve,
                each capped at 20 inner iterations (k_grid_*, k_gmix_*)
    plain_dia   plain FP64 batched CG of the first 512 systems of the batch
                to 1e-10 (k_plain_dia, three CTA tiers)
    vectors     dot, squared norm, linear combination of 4 terms and the
                sampled outer product on n = 64 Mi entries (k_dot, k_lincomb,
                k_sddmm_csr on the 8192^2 Poisson pattern)
    spmv_big    CSR and ELLPACK products on the 8192^2 Poisson matrix (3 each)
    reduce      sums of 2^28 FP32 values along rows, columns, batches (1024
                each) and over all axes, kernel choice included (k_red_*)
    transposed  three transposed products on the 4096^2 Poisson matrix
                (k_spmv_t, after the one-time value gather)
    cg10000     three grid-path Jacobi-CG iterations on the 10000^2 Poisson
                matrix (FP32, diagonal layout: the fused product + p.q kernel;
                about 10 GB on the device: launch lists only)
    cg4096      the same on the 4096^2 Poisson matrix (16.8 M rows, 1.2 GB
                streamed per iteration), for full captures
    cg1024      50 grid-path Jacobi-CG iterations on the 1024^2 Poisson matrix
                (the 2456-iteration solve's shape; data L2-resident)
    cluster200  the 200^2 Poisson matrix (40,000 rows), FP32 Jacobi-CG capped at
                50 iterations: the cluster solve (k_cluster_cg, one launch)
    c4          the 256^3 precision system: 12 plain FP64 Jacobi-CG iterations
                and 12 inner iterations of the mixed FP32 / FP64 solve (one
                launch per kernel under CUMAT_CG_GRAPH=0: the per-kernel share
                of an iteration in a launch list)
    """
    import torch

    import cumat_b200 as cm
    from cumat_b200 import problems as P
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    out = {"profile_case": case}
    if case == "grid3d":
        p3 = P.fv3d(160, 1.0, 3)
        pat = cm.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
        A64 = cm.SparseMatrix(pat, dtype=torch.float64).setData(p3.val.astype(np.float64))
        A32 = cm.SparseMatrix(pat, dtype=torch.float32).setData(p3.val)
        b64 = torch.from_numpy(p3.b.astype(np.float64)).to(dev)
        cg64 = cm.ConjugateGradient(A64).setTolerance(1e-10).setMaxIterations(20).set_path(2)
        cg64.solve(b64)
        cgm = cm.ConjugateGradient(A32).setTolerance(1e-4).setMaxIterations(20).set_path(2)
        cgm.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=3)
        out.update(rows=p3.n, nnz=p3.nnz)
    elif case == "c4":
        p3 = P.fv3d(256, 1.0, 3)
        pat = cm.SparsityPattern.csr(p3.n, p3.n, p3.row_ptr, p3.col)
        A64 = cm.SparseMatrix(pat, dtype=torch.float64).setData(p3.val.astype(np.float64))
        A32 = cm.SparseMatrix(pat, dtype=torch.float32).setData(p3.val)
        b64 = torch.from_numpy(p3.b.astype(np.float64)).to(dev)
        out.update(rows=p3.n, nnz=p3.nnz)
        del p3
        cm.ConjugateGradient(A64).setTolerance(1e-10).setMaxIterations(12).set_path(2).solve(b64)
        cgm = cm.ConjugateGradient(A32).setTolerance(1e-4).setMaxIterations(12).set_path(2)
        cgm.solve_refined(b64, outer=A32, outer_tol=1e-10, max_outer=3)
    elif case == "cluster200":
        pr = P.poisson2d(200, 1)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        b = torch.from_numpy(pr.b).to(dev)
        cm.ConjugateGradient(A).setTolerance(1e-12).setMaxIterations(50).solve(b)
        out.update(rows=pr.n, nnz=pr.nnz)
    elif case in ("cg10000", "cg4096", "cg1024"):
        pr = P.poisson2d({"cg10000": 10000, "cg4096": 4096, "cg1024": 1024}[case], 1)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        b = torch.from_numpy(pr.b).to(dev)
        its = 50 if case == "cg1024" else 3
        cm.ConjugateGradient(A).setTolerance(1e-12).setMaxIterations(its).set_path(2).solve(b)
        out.update(rows=pr.n, nnz=pr.nnz, iterations=its)
    elif case == "plain_dia":
        bt = P.fv2d_batch(N_SYS, SIDE_LO, SIDE_HI, SIGMA, SEED)
        k = int(bt.row_off[512])
        kz = int(bt.row_ptr[k])
        p = cm.SparsityPattern.csr(k, k, bt.row_ptr[:k + 1], bt.col[:kz])
        p.set_systems(bt.row_off[:513])
        A64 = cm.SparseMatrix(p, dtype=torch.float64).setData(bt.val[:kz].astype(np.float64))
        cg64 = cm.ConjugateGradient(A64).setTolerance(OUTER_TOL)
        cg64.solve(torch.from_numpy(bt.b[:k].astype(np.float64)).to(dev))
        st = cg64.system_stats()
        out.update(systems=512, rows=k, nnz=kz, iterations_sum=int(st["iterations"].sum()),
                   converged=bool(np.all(st["status"] == 0)))
    elif case == "vectors":
        n = 64 << 20
        g = torch.Generator(device=dev).manual_seed(3)
        x = torch.rand(n, device=dev, generator=g)
        y = torch.rand(n, device=dev, generator=g)
        cm.dot(x, y)
        cm.squaredNorm(x)
        vs = [torch.rand(n, device=dev, generator=g) for _ in range(4)]
        cm.linear_combination([0.5, -1.0, 2.0, 0.25], vs)
        pr = P.poisson2d(8192, 0)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        u = torch.rand(pr.n, device=dev, generator=g)
        cm.sddmm(A, u, u)
        out.update(n=n, sddmm_rows=pr.n, sddmm_nnz=pr.nnz)
    elif case == "reduce":
        # 2^28 FP32 values (1 GiB) summed along rows, columns and batches (N =
        # 1024 each) and fully; the first call of each shape times its candidates
        x = torch.rand(1 << 28, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
        for axis in ("Row", "Column", "Batch"):
            R, Cc, B = _reduce_shape(axis, 1024, 1 << 28)
            cm.reduce(x.view(B, Cc, R), "sum", _REDUCE_AXIS[axis])
        cm.reduce(x.view(1 << 9, 1 << 9, 1 << 10), "sum", ("rows", "cols", "batches"))
        out.update(n=1 << 28)
    elif case == "transposed":
        pr = P.poisson2d(4096, 1)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        x = torch.from_numpy(pr.b).to(dev)
        for _ in range(3):
            A.transposed_product(x)
        out.update(rows=pr.n, nnz=pr.nnz)
    elif case == "spmv_big":
        pr = P.poisson2d(8192, 1)
        A = cm.SparseMatrix(cm.SparsityPattern.csr(pr.n, pr.n, pr.row_ptr, pr.col)).setData(pr.val)
        idx, ev = P.csr_to_ell(pr.n, pr.row_ptr, pr.col, pr.val)
        E = cm.SparseMatrix(cm.SparsityPattern.ell(pr.n, pr.n, idx)).setData(ev)
        x = torch.from_numpy(pr.b).to(dev)
        for _ in range(3):
            A * x
            E * x
        out.update(rows=pr.n, nnz=pr.nnz)
    else:
        raise SystemExit(f"unknown profile case {case}")
    torch.cuda.synchronize()
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-spmv", action="store_true", help="skip the SpMV GB/s sub-benchmark")
    ap.add_argument("--no-suite", action="store_true",
                    help="skip the reference's own benchmark shapes (SpMV grids 10..10000, CG grids 10..1000)")
    ap.add_argument("--no-next", action="store_true",
                    help="skip the reductions, transposed / CSC products and blocked CG")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 1024^2 Poisson Jacobi-CG and the 256^3 precision comparison")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--profile-small", action="store_true",
                    help="run the small profiling case once (no JSON line): SpMV on the 1024^2 Poisson matrix and the "
                         "mixed and FP64 solvers on the first 512 systems of the batch")
    ap.add_argument("--profile-case", default=None,
                    help="run one small single-purpose workload for ncu (grid3d, plain_dia, vectors, spmv_big, cg10000, cg4096, c4, cluster200)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.profile_case:
        run_profile_case(args.profile_case)
    elif args.profile_small:
        run_profile_small()
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
