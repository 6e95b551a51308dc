#!/usr/bin/env python
"""Benchmark of the HONEI sparse-solver hot path on B200.

Default workload (the SpMV configuration of the north-star configs): ELL SpMV, FP64, on the
2-D Q1 Poisson stiffness matrix of a 2049 x 2049 node grid (4,198,401 rows, 37,720,073
nonzeros, Dirichlet rows identity), x ~ U[-1,1] seeded.  One step = 10 SpMV applications, the
sample the reference's own ELL benchmark times (benchmark/product_ell_file_BENCHMARK.cc).
The matrix (453 MB of Ax + Aj) is larger than L2 (126 MB), so every application streams it
from HBM; x (34 MB) is the gathered, L2-resident operand.

Metric: SpMV GB/s of algorithmic traffic, nnz*(8+4) + 2*n*8 bytes per application (Ax + 32-bit
Aj once, x read once, y written once), against the measured HBM copy bandwidth.
Extras on the same line: plain FP64 CG solves/s and p50/p99 latency on the 257^2 system
(x_true U[-1,1], x0 = 0, relative residual 1e-8), the FP32 SpMV, the batched solve of 512
uneven SPD systems, and a bounded sample of the serving stream (mixed-precision server against
plain FP64 CG on the same requests: solves/s, p50/p99 latency).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: replicas only (one independent system per GPU, no collective; weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

M_SPMV = 2049
M_CG = 257
SPMV_PER_STEP = 10


def spmv_bytes(nnz, n, s):
    return nnz * (s + 4) + 2 * n * s


def q1_nnz(M):
    return (M - 2) ** 2 * 9 + (4 * M - 4)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy burst)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s earlier pool measurement)"


def profile_traffic(name):
    """DRAM bytes per launch from the committed ncu summary profiles/<name>.md, if present."""
    import re
    p = os.path.join(ROOT, "profiles", name + ".md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4,
        "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80, "display_clock_setting": 0x100,
    }

    def __init__(self, device_index=0, period=0.005):
        self.samples, self.reasons = [], set()
        self.period = period
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                mask = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, bit in self.REASONS.items():
                    if mask & bit and k != "gpu_idle":
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples), "source": "nvml" if self.ok else "unavailable"}


def dist_setup():
    from honei_b200 import replicas
    return replicas.env()


# ---------------------------------------------------------------------------------------
# Reference arm: the reference's own CPU path (oracle/_ref, tags::CPU::MultiCore::SSE on all
# host cores), else the C restatement (single core).
# ---------------------------------------------------------------------------------------
_CPU_CASE = {}


def spmv_config(ws):
    """The workload's config dict, the same in both arms."""
    return {"workload": "ell_spmv_q1_2049_f64", "rows": M_SPMV ** 2, "nnz": q1_nnz(M_SPMV),
            "spmv_per_step": SPMV_PER_STEP, "bytes_per_spmv": spmv_bytes(q1_nnz(M_SPMV), M_SPMV ** 2, 8),
            "parallelism": f"replicas{ws}",
            "l2": "matrix 453 MB > L2 each application; no flush (x stays L2-resident by design)"}


def _cpu_case():
    from honei_b200 import problems as P
    if not _CPU_CASE:
        _CPU_CASE["A"] = P.q1_poisson(M_SPMV)
        _CPU_CASE["x"] = P.uniform_vector(_CPU_CASE["A"].rows, 1)
    return _CPU_CASE["A"], _CPU_CASE["x"]


def _ref_handle():
    """The reference's SparseMatrixELL<double> of the workload, built once, with every host
    core given to its MultiCore tags; None without the compiled reference."""
    if "h" in _CPU_CASE:
        return _CPU_CASE["h"]
    h = None
    try:
        from oracle.bindings import REF_SO, Reference
        if os.path.exists(REF_SO):
            R = Reference()
            R.set_threads(os.cpu_count() or 1)
            A, x = _cpu_case()
            h = R.ell_handle(A, x)
    except OSError:
        h = None
    _CPU_CASE["h"] = h
    return h


def cpu_spmv_gbs(budget_s=10.0):
    """The reference's Product<tags::CPU::MultiCore::SSE> on the workload's matrix, built once,
    over a bounded sample (about budget_s of products; median), plus tags::CPU (the oracle's
    order) and tags::CPU::SSE on one core (5 products each).  Without the compiled reference,
    the C restatement of tags::CPU on one core."""
    A, x = _cpu_case()
    nbytes = spmv_bytes(A.nnz, A.rows, 8)
    cores = os.cpu_count() or 1
    h = _ref_handle()
    if h is not None:
        t1 = float(h.spmv("mc-sse", 2)[-1])
        reps = int(max(3, min(200, budget_s / max(t1, 1e-4))))
        t = statistics.median(h.spmv("mc-sse", reps))
        single = {tag: round(nbytes / statistics.median(h.spmv(tag, 5)) / 1e9, 3) for tag in ("cpu", "sse")}
        return {"value": round(nbytes / t / 1e9, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
                "sample": f"tags::CPU::MultiCore::SSE on {cores} threads, {reps} products of the 2049^2 FP64 "
                          "matrix (built once), median",
                "single_core_gbs": {"tags::CPU": single["cpu"], "tags::CPU::SSE": single["sse"]}}
    from oracle.bindings import Oracle
    O = Oracle()
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        O.spmv(A, x)
        ts.append(time.perf_counter() - t0)
    return {"value": round(nbytes / statistics.median(ts) / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": "C restatement of tags::CPU, 5 products of the 2049^2 FP64 matrix, median"}


def run_reference_arm(args):
    """The reference's own CPU path on the same workload: Product<tags::CPU::MultiCore::SSE> on
    all host cores (oracle/_ref, the reference compiled from its sources), the matrix built once;
    one step = SPMV_PER_STEP products, wall-clocked.  Rank 0 only."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    A, x = _cpu_case()
    nbytes = spmv_bytes(A.nnz, A.rows, 8)
    h = _ref_handle()
    cores = os.cpu_count() or 1
    if h is not None:
        def step():
            return float(np.sum(h.spmv("mc-sse", SPMV_PER_STEP)))
        kind, used = "reference", cores
        desc = f"tags::CPU::MultiCore::SSE on {cores} threads, {SPMV_PER_STEP} products of the 2049^2 FP64 matrix per step"
    else:
        from oracle.bindings import Oracle
        O = Oracle()

        def step():
            t0 = time.perf_counter()
            for _ in range(SPMV_PER_STEP):
                O.spmv(A, x)
            return time.perf_counter() - t0
        kind, used = "port", 1
        desc = f"C restatement of tags::CPU, {SPMV_PER_STEP} products of the 2049^2 FP64 matrix per step"
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    wall = time.perf_counter() - t0
    value = nbytes * SPMV_PER_STEP * args.steps / wall / 1e9
    line = {
        "impl": "reference", "metric": "ell_spmv_gbs_q1_2049_f64", "value": round(value, 3), "unit": "GB/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * wall / max(args.steps, 1), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Q1 Poisson 2049^2, x ~ U[-1,1])",
        "config": spmv_config(ws),
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": used, "kind": kind, "sample": desc},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------------------
def _time_us(fn, reps, flush=None):
    """Median CUDA-event time of fn() in microseconds, after 3 warm-up calls; with `flush`
    (a device buffer larger than L2) zeroed between the timed calls, outside the events."""
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e3)
    return statistics.median(ts)


def bench_spmv_variants(la, ctx, M=M_SPMV, seed=5, cpu=True, reps=50):
    """The other SpMV lines of the SpMV configuration: the FP32 product of the 2049^2 matrix; the
    randomly permuted 2049^2 matrix (seeded symmetric row/column permutation) in FP64 and FP32,
    as given and through its Cuthill-McKee ordered copy (SparseMatrixELL.ordered: rows stored
    in the locality order, columns renumbered and packed as 16-bit offsets, x permuted into a
    work vector inside the timed product, y scattered back -- bit-identical to the product on
    the permuted matrix; the sorted, ranked form beside it); the
    1025^2 FP64 product with L2 flushed between products (its 130 MB would otherwise stay
    partly in L2).  GB/s are the algorithmic bytes of the product on the given matrix
    (nnz*(s+4) + 2*n*s)."""
    import torch
    from honei_b200 import problems as P
    peak, _ = measured_peak()
    n = M * M
    nnz = q1_nnz(M)
    out = {"workload": f"ELL SpMV variants: Q1 {M}^2 FP32; Q1 {M}^2 randomly permuted (seed {seed}), FP64 and "
                       "FP32, as given and through the Cuthill-McKee ordered copy; Q1 1025^2 FP64 with L2 flushed"}

    def line(us, s, nn=n, nz=nnz):
        g = spmv_bytes(nz, nn, s) / (us * 1e3)
        return {"us": round(us, 2), "gbs": round(g, 1), "frac_of_peak": round(g / peak, 4)}

    A = la.SparseMatrixELL.q1_poisson(M, ctx=ctx)
    A32 = A.to_float(ctx=ctx)
    x32 = torch.from_numpy(P.uniform_vector(n, 1).astype(np.float32)).cuda()
    y32 = torch.empty_like(x32)
    out["natural_f32"] = line(_time_us(lambda: la.Product.value(y32, A32, x32, ctx=ctx), reps), 4)
    del A, A32
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    Ap, _ = P.q1_poisson_permuted(M, seed=seed)
    out["host_permuted_matrix_s"] = round(time.perf_counter() - t0, 2)
    for name, dt, s in (("f64", np.float64, 8), ("f32", np.float32, 4)):
        Ad = la.SparseMatrixELL.from_reference(Ap.astype(dt) if dt != np.float64 else Ap, ctx)
        x = torch.from_numpy(P.uniform_vector(n, seed + 1).astype(dt)).cuda()
        y = torch.empty_like(x)
        out[f"permuted_{name}"] = line(_time_us(lambda: la.Product.value(y, Ad, x, ctx=ctx), reps), s)
        y0 = y.clone()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B = Ad.ordered(columns=True, ctx=ctx)
        torch.cuda.synchronize()
        t_order = time.perf_counter() - t0
        r = line(_time_us(lambda: la.Product.value(y, B, x, ctx=ctx), reps), s)
        r["same_y_as_permuted"] = bool(torch.equal(y, y0))
        r["ordering_ms"] = round(t_order * 1e3, 1)
        r["levels"], r["bandwidth_before"], r["bandwidth_after"] = int(B.info[0]), Ad.bandwidth(), B.B.bandwidth()
        r["form"] = "packed (16-bit column offsets, slots in their order)" if B.Bd is not None else "ranked"
        # the bytes this form moves: x gathered (order, x, xw) and the product's own arrays
        # (every slot of the K x ld value and index arrays, rank words for the ranked form, order,
        # xw, y)
        idx = 2 if B.Bd is not None else 4
        rk = 0 if B.Bd is not None else 8
        own = (4 + 2 * s) * n + B.B.K * B.B.ld * (s + idx) + (rk + 4 + 2 * s) * n
        r["own_bytes"] = own
        r["own_gbs"] = round(own / (r["us"] * 1e3), 1)
        y.fill_(0)
        R = Ad.ordered(columns=True, packed=False, ctx=ctx)
        r2 = line(_time_us(lambda: la.Product.value(y, R, x, ctx=ctx), reps), s)
        r2["same_y_as_permuted"] = bool(torch.equal(y, y0))
        r["ranked_form"] = r2
        out[f"permuted_ordered_{name}"] = r
        del Ad, B, R, x, y, y0
        torch.cuda.empty_cache()
    if cpu:
        h = None
        try:
            from oracle.bindings import REF_SO, Reference
            if os.path.exists(REF_SO):
                R = Reference()
                R.set_threads(os.cpu_count() or 1)
                h = R.ell_handle(Ap, P.uniform_vector(n, seed + 1))
        except OSError:
            h = None
        if h is not None:
            t = statistics.median(h.spmv("mc-sse", 10))
            out["permuted_f64_cpu_reference_gbs"] = round(spmv_bytes(nnz, n, 8) / t / 1e9, 2)
            h.close()
    del Ap
    M2 = 1025
    n2, nz2 = M2 * M2, q1_nnz(M2)
    A = la.SparseMatrixELL.q1_poisson(M2, ctx=ctx)
    x = torch.from_numpy(P.uniform_vector(n2, 1)).cuda()
    y = torch.empty_like(x)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out["natural_1025_f64_l2_flushed"] = line(_time_us(lambda: la.Product.value(y, A, x, ctx=ctx), reps, flush),
                                              8, n2, nz2)
    out["natural_1025_f64_warm_l2"] = line(_time_us(lambda: la.Product.value(y, A, x, ctx=ctx), reps), 8, n2, nz2)
    del A, flush
    torch.cuda.empty_cache()
    return out


def plugin_e2e(M=M_SPMV, steps=20):
    """The product through HONEI's own API with host DenseVectors (tests/plugin: Product<tags::
    GPU::CUDA>::value through MemoryArbiter and MemoryBackend<tags::GPU::CUDA>, one upload of x
    and one download of y per step): one product per step and ten per step.  None where the
    plugin programs are not built."""
    import subprocess
    exe = os.path.join(ROOT, "tests", "plugin", "_build", "plugin_product_bench")
    if not os.path.exists(exe):
        return None
    try:
        p = subprocess.run([exe, str(M), str(steps)], capture_output=True, text=True, timeout=600)
        return json.loads(p.stdout.strip().splitlines()[-1]) if p.returncode == 0 else {"error": p.stderr[-300:]}
    except (OSError, ValueError, subprocess.SubprocessError, IndexError) as e:
        return {"error": repr(e)}


def bench_batch(la, ctx, n_systems=512, seed=2024):
    """512 independent SPD Q1 systems, side ~ U{17..257}, cell coefficient 10^U(-1,1), b = A x_true:
    one persistent batched launch (FP64 CG, and FP32-inner IR to a 1e-8 FP64 residual) against
    plain FP64 CG solved one system at a time (hb_cg_f64, the whole GPU per solve)."""
    import torch
    from honei_b200 import batch as B

    rng = np.random.default_rng(seed)
    sides = rng.integers(17, 258, size=n_systems)
    out = {"workload": f"{n_systems} SPD Q1 systems, side U{{17..257}}, coef 10^U(-1,1), CG to 1e-8",
           "rows_total": int(sum(int(m) * int(m) for m in sides))}
    for mode in ("cg64", "ir32"):
        systems = B.q1_batch(sides, coef_range=(1e-1, 1e1), seed=seed, mode=mode, eps=1e-8, inner_eps=1e-3)
        solver = B.BatchSolver(systems, ctx=ctx)
        cfg = solver.tune(use_cache=False)
        for sys_ in systems:
            sys_.x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.run(cfg)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res = solver.results()
        out[mode] = {"ms": round(ms, 2), "systems_per_s": round(n_systems / (ms / 1e3), 1),
                     "config": {"cluster": cfg.cluster, "threads": cfg.threads, "rows_per_thread": cfg.rows_per_thread},
                     "iterations_mean": round(float(np.mean([r["iterations"] for r in res])), 1),
                     "max_true_relres": float(max(r["true_relres"] for r in res)),
                     "tune_ms": getattr(solver, "tune_times", None)}
        if mode == "cg64":
            # baseline: the same systems, plain FP64 CG one at a time (grid-wide persistent kernel)
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            for sys_ in systems:
                sys_.x.zero_()
            torch.cuda.synchronize()
            t0.record()
            iters = []
            for sys_ in systems:
                iters.append(la.CGSolver.value(sys_.A64, None, sys_.b, sys_.x, 100000, 1e-8, ctx=ctx))
            t1.record()
            torch.cuda.synchronize()
            bms = t0.elapsed_time(t1)
            out["sequential_cg64"] = {"ms": round(bms, 2), "systems_per_s": round(n_systems / (bms / 1e3), 1),
                                      "iterations_mean": round(float(np.mean(iters)), 1)}
        del solver, systems
        torch.cuda.empty_cache()
    out["speedup_batched_ir32_vs_sequential_cg64"] = round(out["sequential_cg64"]["ms"] / out["ir32"]["ms"], 2)
    out["speedup_batched_cg64_vs_sequential_cg64"] = round(out["sequential_cg64"]["ms"] / out["cg64"]["ms"], 2)
    return out


def bench_cg_permuted(la, ctx, M=M_SPMV, seed=5):
    """Config 2's CG on the randomly permuted 2049^2 matrix: as given (every gather a random
    sector) and through its Cuthill-McKee ordered copy (CGSolver on an OrderedMatrixELL: b and x
    permuted once per solve, the iterations in the copy's numbering)."""
    import torch
    from honei_b200 import problems as P
    Ap, _ = P.q1_poisson_permuted(M, seed=seed)
    Ad = la.SparseMatrixELL.from_reference(Ap, ctx)
    n = Ap.rows
    xt = torch.from_numpy(P.uniform_vector(n, 1)).cuda()
    b = torch.empty_like(xt)
    la.Product.value(b, Ad, xt, ctx=ctx)
    r = torch.empty_like(xt)
    out = {"workload": f"plain FP64 CG, Q1 {M}^2 randomly permuted (seed {seed}), 1e-8 relative, x0 = 0"}
    t0 = time.perf_counter()
    O = Ad.ordered(columns=True, ctx=ctx)
    torch.cuda.synchronize()
    out["ordering_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
    for name, A in (("as_given", Ad), ("ordered_copy", O)):
        x = torch.zeros_like(xt)
        la.CGSolver.value(A, None, b, x, 20, 1e-8, ctx=ctx)          # warm-up
        x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        used = la.CGSolver.value(A, None, b, x, 100000, 1e-8, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        la.Defect.value(r, b, Ad, x, ctx=ctx)
        out[name] = {"iterations": used, "ms": round(ms, 2), "us_per_iteration": round(1e3 * ms / max(used, 1), 2),
                     "relres": float(torch.linalg.norm(r) / torch.linalg.norm(b))}
    out["speedup_ordered"] = round(out["as_given"]["ms"] / out["ordered_copy"]["ms"], 2)
    del Ap, Ad, O
    torch.cuda.empty_cache()
    return out


def bench_cg_large(la, ctx, sizes=(1025, 2049), cpu=True, cpu_iters=10):
    """Plain FP64 CG (config 2's CG) on the Q1 Poisson grids of 1025^2 and 2049^2: b = A x_true
    with x_true ~ U[-1, 1], x0 = 0, 1e-8 relative; the streaming persistent kernel.  Algorithmic
    bytes per iteration nnz*(8 + 4) + 10*n*8 (the matrix once, the vectors of both phases).  With
    the compiled reference present, its MultiCore::SSE CGSolver on the host cores over a bounded
    sample of cpu_iters iterations of the same system (seconds per iteration)."""
    import torch
    from honei_b200 import problems as P
    peak, _ = measured_peak()
    out = {}
    for M in sizes:
        A = la.SparseMatrixELL.q1_poisson(M, ctx=ctx)
        n = A.rows()
        xt = torch.from_numpy(P.uniform_vector(n, 1)).cuda()
        b = torch.empty_like(xt)
        la.Product.value(b, A, xt, ctx=ctx)
        x = torch.zeros_like(xt)
        la.CGSolver.value(A, None, b, x, 20, 1e-8, ctx=ctx)          # warm-up
        x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        used = la.CGSolver.value(A, None, b, x, 100000, 1e-8, ctx=ctx)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        r = torch.empty_like(xt)
        la.Defect.value(r, b, A, x, ctx=ctx)
        nnz = int((A.Aj >= 0).sum())
        per_it = nnz * 12 + 10 * n * 8
        us = 1e3 * ms / max(used, 1)
        row = {"iterations": used, "ms": round(ms, 2), "us_per_iteration": round(us, 2),
               "bytes_per_iteration": per_it, "gbs": round(per_it / (us * 1e3), 1),
               "frac_of_peak": round(per_it / (us * 1e3) / peak, 4),
               "relres": float(torch.linalg.norm(r) / torch.linalg.norm(b))}
        del A, x, r, b, xt
        torch.cuda.empty_cache()
        if cpu:
            R = _ref_cpu()
            if R is not None:
                Ah = P.q1_poisson(M)
                bh, _ = R.spmv(Ah, P.uniform_vector(Ah.rows, 1), tag="mc-sse")
                _, u, sec = R.cg(Ah, bh, max_iters=cpu_iters, eps=1e-30, tag="mc-sse")
                row["cpu_reference"] = {"s_per_iteration": round(sec / max(u, 1), 5), "sample_iterations": u,
                                        "cores": os.cpu_count(), "tag": "tags::CPU::MultiCore::SSE"}
                row["speedup_per_iteration_vs_cpu"] = round(sec / max(u, 1) / (us / 1e6), 1)
        out[f"{M}"] = row
    return {"workload": "plain FP64 CG on Q1 Poisson, 1e-8 relative, x0 = 0 (streaming kernel)", **out}


def bench_cg_cluster(ctx, M=M_CG, n_solves=30):
    """The 257^2 plain FP64 CG solve on one thread-block cluster (batched kernel, batch of 1)."""
    import torch
    from honei_b200 import batch as B

    best = None
    for cluster in (8, 16):
        for threads in (512, 256):
            s = B.q1_batch([M], coef_range=None, seed=1, mode="cg64", symmetric=False, eps=1e-8)
            solver = B.BatchSolver(s, ctx=ctx)
            cfg = B.HbBatchConfig(cluster, threads)
            lat = []
            for i in range(n_solves + 3):
                s[0].x.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = solver.solve(cfg)
                lat.append(time.perf_counter() - t0)
            lat = sorted(1e3 * v for v in lat[3:])
            cand = {"cluster": cluster, "threads": threads, "iterations": r[0]["iterations"],
                    "solves_per_s": round(len(lat) / (sum(lat) / 1e3), 2),
                    "p50_ms": round(statistics.median(lat), 3), "p99_ms": round(lat[-1], 3)}
            if best is None or cand["p50_ms"] < best["p50_ms"]:
                best = cand
    return best


def _ref_cpu():
    """The compiled reference (tags::CPU::MultiCore::SSE on every host core), or None."""
    try:
        from oracle.bindings import REF_SO, Reference
        if not os.path.exists(REF_SO):
            return None
        R = Reference()
        R.set_threads(os.cpu_count() or 1)
        return R
    except OSError:
        return None


def bench_csr(la, ctx, x, ell_s, M=M_SPMV, reps=100, cpu=True):
    """Product on SparseMatrixCSR (csr::blocksize 1) of the same 2049^2 Poisson matrix and x as
    the headline: algorithmic bytes nnz*(8 + 4) + (n + 1)*8 + 2*n*8 per product (values and
    int32 columns once, the int64 row offsets, x once, y once).  ``ell_s`` is the ELL product's
    measured time, for the ratio."""
    import torch
    from honei_b200 import problems as P
    Ch = P.csr_from_ell(P.q1_poisson(M), 1)
    C = la.SparseMatrixCSR.from_reference(Ch, ctx)
    n, nnz = C.rows(), C.nblocks
    y = torch.empty_like(x)
    for _ in range(3):
        la.Product.value(y, C, x, ctx=ctx)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        la.Product.value(y, C, x, ctx=ctx)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    nbytes = nnz * 12 + (n + 1) * 8 + 2 * n * 8
    peak, _ = measured_peak()
    out = {"workload": f"SparseMatrixCSR product (csr::blocksize 1), Poisson {M}^2, FP64", "bytes_per_product": nbytes,
           "us_per_product": round(t * 1e6, 2), "gbs": round(nbytes / t / 1e9, 1),
           "frac_of_peak": round(nbytes / t / 1e9 / peak, 4), "time_vs_ell_product": round(t / ell_s, 3)}
    if cpu:
        R = _ref_cpu()
        if R is not None:
            _, sec = R.csr_spmv(Ch, x.cpu().numpy(), tag="mc-sse", reps=10)
            out["cpu_reference_gbs"] = round(nbytes / sec / 1e9, 2)
            out["cpu_reference"] = f"tags::CPU::MultiCore::SSE, {os.cpu_count()} cores, median of 10"
    del C
    torch.cuda.empty_cache()
    return out


def bench_q1band(la, ctx, x, ell_s, M=M_SPMV, reps=100, cpu=True):
    """Product on BandedMatrixQx<Q1Type> (nine bands of n values, no index array) for the same
    2049^2 Poisson matrix and x as the headline: algorithmic bytes 11*n*8 per product (nine
    bands, x once, y once).  ``ell_s`` is the ELL product's measured time, for the ratio."""
    import torch
    B = la.BandedMatrixQ1.poisson(M, ctx=ctx)
    n = B.rows()
    y = torch.empty_like(x)
    for _ in range(3):
        la.Product.value(y, B, x, ctx=ctx)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        la.Product.value(y, B, x, ctx=ctx)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    nbytes = 11 * n * 8
    peak, _ = measured_peak()
    out = {"workload": f"BandedMatrixQx<Q1Type> product, Poisson {M}^2, FP64", "bytes_per_product": nbytes,
           "us_per_product": round(t * 1e6, 2), "gbs": round(nbytes / t / 1e9, 1),
           "frac_of_peak": round(nbytes / t / 1e9 / peak, 4),
           "speedup_vs_ell_product": round(ell_s / t, 2)}
    if cpu:
        R = _ref_cpu()
        if R is not None:
            bands = R.q1band_poisson(M)
            _, sec = R.q1band_spmv(bands, x.cpu().numpy(), tag="mc-sse", reps=20)
            out["cpu_reference_gbs"] = round(nbytes / sec / 1e9, 2)
            out["cpu_reference"] = f"tags::CPU::MultiCore::SSE, {os.cpu_count()} cores, median of 20"
    del B
    torch.cuda.empty_cache()
    return out


MG_COARSE_ITERS = 100


def mg_cycle_bytes(H, s, banded):
    """Algorithmic bytes of one MGSolver cycle (V(2,2) plus the finest defect and its norm) on
    hierarchy H with s-byte values.  Per level above the coarsest (n rows, n_c coarse rows): four
    Jacobi sweeps x' = x + P (b - A x) (matrix, x, b, P read, x' written), the defect (matrix, x,
    b read, store written), the restriction (store read, d_c written; the ELL cycle also reads
    Res), the zero fill of c_c, prolongation + sum (c_c, x read, x written; ELL also reads Prol).
    Matrix per application: 9 n s banded (nine bands), nnz (s + 4) ELL.  The coarsest level's CG
    (81 rows) is latency, not bytes, and is left out."""
    total = 0
    L = len(H.A)
    for l in range(1, L):
        A = H.A[l]
        n, nc = A.rows, H.A[l - 1].rows
        mat = 9 * n * s if banded else A.nnz * (s + 4)
        sweep = mat + 4 * n * s
        defect = mat + 3 * n * s
        restrict = n * s + nc * s + (0 if banded else H.res[l - 1].nnz * (s + 4))
        prolong = nc * s + 2 * n * s + (0 if banded else H.prol[l - 1].nnz * (s + 4))
        total += 4 * sweep + defect + restrict + nc * s + prolong
    n = H.A[-1].rows
    total += (9 * n * s if banded else H.A[-1].nnz * (s + 4)) + 3 * n * s + n * s
    return int(total)


def bench_mg(la, ctx, M=2049, seed=5, cpu=True):
    """Q1 Poisson M^2 (unit coefficient, the reference's rediscretised hierarchy down to 9^2):
    MGSolver V(2,2), damped Jacobi 0.7, PROLMAT transfers, coarse CG, x0 = 0, b = A x_true.
    FP64 to 1e-8 relative; FP32 to 1e-6 (FP32 stagnates near 1e-7).  The coarse CG is capped at
    MG_COARSE_ITERS iterations, MGUtil::configure's max_iters_coarse in the reference's own MG
    test (honei/math/mg_TEST.cc:421); the 9^2 coarse system (identity Dirichlet rows, not
    symmetric) stagnates well before that, and a run at a cap of 1000 (f64_banded_coarse1000)
    takes the same cycles to the same residual.  When the compiled reference is present, its
    MultiCore::SSE MG solve of the same FP64 system on the host cores.  Each variant reports its
    algorithmic bytes per cycle (mg_cycle_bytes) and the fraction of the HBM peak that gives."""
    import torch
    from honei_b200 import problems as P

    H = P.mg_hierarchy(M)
    xt = P.uniform_vector(M * M, seed)
    out = {"workload": f"MG V(2,2) on Q1 {M}^2, {len(H.sides)} levels, coarse CG on 9^2 (at most "
                       f"{MG_COARSE_ITERS} iterations); *_banded: banded levels and matrix-free transfers, the same "
                       "cycle", "max_iters_coarse": MG_COARSE_ITERS}
    bref = None
    xs_ell = {}
    for name, npdt, tdt, eps, banded, mic in (("f64", np.float64, torch.float64, 1e-8, False, MG_COARSE_ITERS),
                                               ("f32", np.float32, torch.float32, 1e-6, False, MG_COARSE_ITERS),
                                               ("f64_banded", np.float64, torch.float64, 1e-8, True, MG_COARSE_ITERS),
                                               ("f32_banded", np.float32, torch.float32, 1e-6, True, MG_COARSE_ITERS),
                                               ("f64_banded_coarse1000", np.float64, torch.float64, 1e-8, True, 1000)):
        data = la.MGData.from_hierarchy(H, npdt, ctx=ctx, eps=eps, max_iters=100, max_iters_coarse=mic,
                                        banded=banded)
        A = data.A[-1]
        xtd = torch.from_numpy(xt.astype(npdt)).cuda()
        b = torch.empty_like(xtd)
        la.Product.value(b, A, xtd, ctx=ctx)
        if name == "f64":
            bref = b.cpu().numpy()
        x = torch.zeros_like(b)
        la.MGSolver.value(data, b, x)  # warm-up
        x.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        cycles, r0, r1 = la.MGSolver.value(data, b, x)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        err = float(torch.linalg.norm((x - xtd).double()) / torch.linalg.norm(xtd.double()))
        peak, _ = measured_peak()
        cb = mg_cycle_bytes(H, np.dtype(npdt).itemsize, banded)
        gbs = cb / (ms / max(cycles, 1) * 1e6)
        out[name] = {"ms": round(ms, 2), "cycles": cycles, "ms_per_cycle": round(ms / max(cycles, 1), 3),
                     "relres": r1 / r0 if r0 else 0.0, "eps": eps, "err_vs_x_true": err,
                     "bytes_per_cycle": cb, "gbs": round(gbs, 1), "frac_of_peak": round(gbs / peak, 4)}
        if banded and mic == MG_COARSE_ITERS:
            # the banded cycle rounds as the ELL cycle: same iterate
            out[name]["same_x_as_ell"] = bool(torch.equal(x, xs_ell[name.split("_")[0]]))
        else:
            xs_ell[name] = x.clone()
        data.close()
        del data, A, b, xtd
        torch.cuda.empty_cache()
    if cpu:
        R = _ref_cpu()
        if R is not None:
            _, used, sec = R.mg(H, bref, eps=1e-8, max_iters_coarse=MG_COARSE_ITERS, tag="mc-sse")
            out["cpu_reference_f64"] = {"s": round(sec, 3), "cycles": used, "cores": os.cpu_count(),
                                        "tag": "tags::CPU::MultiCore::SSE"}
            out["speedup_f64_vs_cpu"] = round(sec * 1e3 / out["f64"]["ms"], 1)
    return out


def bench_ir(la, ctx, M=2049, seed=3):
    """Mixed precision on Q1 M^2 (SPD form) with a cellwise coefficient 10^U(-2,2): FP64
    refinement to 1e-10 relative around FP32 inner solves to 1e-3 -- MG-preconditioned CG on the
    device-built Galerkin hierarchy (hb_q1_solve), and plain FP32 CG (hb_ir_cg_solve) -- each
    with ||x - x_CG64|| / ||x_CG64|| against plain FP64 CG on the same system run to 1e-12."""
    import torch
    from honei_b200 import problems as P

    coef = torch.from_numpy(P.log_uniform_coef(M, 1e-2, 1e2, seed).ravel()).cuda()
    q = la.Q1System(M, coef, ctx=ctx)
    A = q.A
    xt = torch.from_numpy(P.uniform_vector(M * M, seed + 1)).cuda()
    b = torch.empty_like(xt)
    la.Product.value(b, A, xt, ctx=ctx)
    bn = la.Norm.value(b, root=True, ctx=ctx)
    r = torch.empty_like(b)

    def relres(x):
        la.Defect.value(r, b, A, x, ctx=ctx)
        return la.Norm.value(r, root=True, ctx=ctx) / bn

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = fn()
        e1.record()
        torch.cuda.synchronize()
        return res, e0.elapsed_time(e1)

    x64 = torch.zeros_like(b)
    it64, ms64 = timed(lambda: la.CGSolver.value(A, None, b, x64, 1000000, 1e-12, ctx=ctx))
    ref_norm = float(torch.linalg.norm(x64))
    out = {"workload": f"Q1 {M}^2 SPD, coef 10^U(-2,2), FP64 target 1e-10, inner FP32 to 1e-3",
           "cg64": {"ms": round(ms64, 1), "iterations": it64, "relres": relres(x64)}}
    x = torch.zeros_like(b)
    q.solve(b, x, eps=1e-10)  # warm-up (graph instantiation)
    x.zero_()
    info, ms = timed(lambda: q.solve(b, x, eps=1e-10))
    out["ir_mgpcg32"] = {"ms": round(ms, 2), "outer": info["outer"], "inner_iterations": info["iterations"],
                         "relres": relres(x), "err_vs_cg64": float(torch.linalg.norm(x - x64)) / ref_norm}
    A32 = A.to_float(ctx=ctx)
    x.zero_()
    (outer, _, _, inner), ms = timed(lambda: la.IRSolver.value_cg(A, A32, b, x, eps=1e-10, inner_eps=1e-3, ctx=ctx))
    out["ir_cg32"] = {"ms": round(ms, 1), "outer": outer, "inner_iterations": inner, "relres": relres(x),
                      "err_vs_cg64": float(torch.linalg.norm(x - x64)) / ref_norm}
    out["speedup_ir_mgpcg32_vs_cg64"] = round(ms64 / out["ir_mgpcg32"]["ms"], 1)
    q.close()
    return out


SERVE_RATE = 20.0           # Poisson arrivals per second: about half the plain baselines' capacity
SERVE_LATENCY_REQUESTS = 600


def _cpu_serve_baseline(trace, budget_s=20.0):
    """The reference's CGSolver<tags::CPU::MultiCore::SSE> (plain FP64 CG, 1e-8 relative) on the
    stream's requests in order, on every host core, until about budget_s have passed: solves/s
    of that sample (host-side assembly excluded from the timing)."""
    try:
        from oracle.bindings import REF_SO, Reference
        if not os.path.exists(REF_SO):
            return None
        R = Reference()
        R.set_threads(os.cpu_count() or 1)
    except OSError:
        return None
    from honei_b200 import problems as P
    spent, solved, rows = 0.0, 0, 0
    for i in range(len(trace)):
        req = trace.request(i)
        A = P.q1_poisson(req.M, req.coef.reshape(req.M - 1, req.M - 1), symmetric=True)
        b, _ = R.spmv(A, req.x_true, tag="mc-sse")
        _, used, sec = R.cg(A, b, eps=1e-8, max_iters=1000000, tag="mc-sse")
        spent += sec
        solved += 1
        rows += req.M * req.M
        if spent > budget_s:
            break
    return {"solves_per_s": round(solved / spent, 3), "requests": solved, "rows": rows, "seconds": round(spent, 2),
            "cores": os.cpu_count(), "tag": "CGSolver<tags::CPU::MultiCore::SSE> (plain FP64 CG), the stream's "
                                              "first requests in order"}


def bench_serve(n_requests=20000, prefix=2000, rate=SERVE_RATE, seed=11, device=0, window=256, cpu=True,
                latency_requests=SERVE_LATENCY_REQUESTS):
    """The serving configuration: a stream of Q1 requests, side log-uniform in [33, 1025],
    cellwise coefficient log-uniform in [1e-2, 1e2], b = A x_true, each solved to 1e-8 relative
    FP64 residual, submitted from host buffers and returned to host buffers.

    Capacity (solves/s): the stream served closed-loop (at most `window` requests outstanding,
    each submitted as soon as the server takes one) -- the mixed server on all n_requests; the
    two plain FP64 CG baselines (one request at a time; and with the mixed server's concurrency:
    batched cluster launches for small grids, concurrent whole-GPU CG for the rest) and the mixed
    server again on the first `prefix` requests, for the like-for-like ratios.  Latency (p50/p99,
    arrival to result): the first `latency_requests` requests with Poisson arrivals at `rate` per
    second, a rate every server sustains (about half the plain baselines' capacity), so p99 is
    service time rather than queue growth; the mixed server also at 7.5x that rate."""
    from honei_b200 import serve as S

    full = S.stream_trace(n_requests, rate=0.0, seed=seed)
    pre = full.prefix(prefix)
    timed = S.stream_trace(latency_requests, rate=rate, seed=seed)
    fast = S.stream_trace(latency_requests, rate=7.5 * rate, seed=seed)
    out = {"workload": f"serving stream: {n_requests} requests (side log-U[33,1025], coef log-U[1e-2,1e2], "
                       f"1e-8 FP64); capacity closed-loop ({window} outstanding): the mixed server on all "
                       f"{n_requests}, both plain FP64 CG baselines and the mixed server on the first {prefix}; "
                       f"latency: the first {latency_requests} with Poisson arrivals at {rate:g}/s "
                       f"(mixed also at {7.5 * rate:g}/s)",
           "n_requests": n_requests, "prefix": prefix, "rows_total": full.rows, "rows_prefix": pre.rows,
           "rate_per_s": rate, "window": window}
    # warm-up, untimed: kernels of every path loaded, the stream-ordered pool grown
    warm = S.stream_trace(300, rate=0.0, seed=seed + 1000)
    for mode in ("mixed", "plain_batched"):
        with S.Server(mode=mode) as srv:
            S.replay_stream(srv, warm, realtime=False, window=window)

    def run(mode, trace, realtime):
        with S.Server(mode=mode) as srv, ClockSampler(device) as clk:
            rep = S.replay_stream(srv, trace, realtime=realtime, window=window)
            st = srv.stats()
        return {"requests": rep["completed"], "solves_per_s": round(rep["solves_per_s"], 2),
                "p50_ms": round(rep["p50_ms"], 2), "p99_ms": round(rep["p99_ms"], 2),
                "service_p50_ms": round(rep["service_p50_ms"], 2), "service_p99_ms": round(rep["service_p99_ms"], 2),
                "ok": rep["ok"], "paths": rep["paths"], "max_true_relres": rep["max_true_relres"],
                "makespan_s": round(rep["makespan_s"], 2), "submit_lag_max_ms": round(rep["submit_lag_max_ms"], 2),
                "admitted_bytes_peak": st["bytes_peak"], "pool_used_high": st.get("pool_used_high"),
                "pool_reserved_high": st.get("pool_reserved_high"), "clocks": clk.summary()}

    out["mixed_full"] = run("mixed", full, False)
    out["mixed_prefix"] = run("mixed", pre, False)
    out["plain_batched_prefix"] = run("plain_batched", pre, False)
    out["plain_prefix"] = run("plain", pre, False)
    out["mixed_poisson"] = run("mixed", timed, True)
    out["plain_batched_poisson"] = run("plain_batched", timed, True)
    out["plain_poisson"] = run("plain", timed, True)
    out["mixed_poisson_fast"] = run("mixed", fast, True)
    mp = out["mixed_prefix"]["solves_per_s"]
    out["speedup_vs_plain_batched"] = round(mp / max(out["plain_batched_prefix"]["solves_per_s"], 1e-9), 2)
    out["speedup_vs_plain_one_at_a_time"] = round(mp / max(out["plain_prefix"]["solves_per_s"], 1e-9), 2)
    if cpu:
        cb = _cpu_serve_baseline(full)
        if cb is not None:
            out["cpu_reference"] = cb
    return out


def bench_cg_257(la, ctx, cpu=True):
    """Plain FP64 CG on the 257^2 Q1 system (the CG configuration): solve latency from host b to
    host x (pinned copies inside each timed solve), 30 solves after 3 warm-ups; with the compiled
    reference, its CGSolver<MultiCore::SSE> on the same system on every host core."""
    import torch
    from honei_b200 import problems as P
    Acg = la.SparseMatrixELL.q1_poisson(M_CG, ctx=ctx)
    ncg = Acg.rows()
    xt = torch.from_numpy(P.uniform_vector(ncg, 1)).cuda()
    bcg = torch.empty_like(xt)
    la.Product.value(bcg, Acg, xt, ctx=ctx)
    bh = bcg.cpu().pin_memory()
    xh_cg = torch.empty(ncg, dtype=torch.float64).pin_memory()
    bd, xd_cg = torch.empty_like(bcg), torch.empty_like(bcg)
    lat, iters = [], None
    n_solves = 30
    for i in range(n_solves + 3):
        t0 = time.perf_counter()
        bd.copy_(bh, non_blocking=True)
        xd_cg.zero_()
        iters = la.CGSolver.value(Acg, None, bd, xd_cg, 20000, 1e-8, ctx=ctx)
        xh_cg.copy_(xd_cg, non_blocking=True)
        torch.cuda.synchronize()
        if i >= 3:
            lat.append(time.perf_counter() - t0)
    lat_ms = sorted(1e3 * v for v in lat)
    cg_extra = {"workload": "plain FP64 CG, Q1 257^2, 1e-8 relative, x0 = 0", "iterations": iters,
                "solves_per_s": round(len(lat) / sum(lat), 2),
                "p50_ms": round(statistics.median(lat_ms), 3),
                "p99_ms": round(lat_ms[min(len(lat_ms) - 1, int(0.99 * len(lat_ms)))], 3)}
    if cpu:
        # the reference's own CGSolver<MultiCore::SSE> on the host cores, same system
        R = _ref_cpu()
        if R is not None:
            Ah = P.q1_poisson(M_CG)
            secs = []
            for _ in range(3):
                _, used_ref, sec = R.cg(Ah, bh.numpy(), eps=1e-8, max_iters=20000, tag="mc-sse")
                secs.append(sec)
            cg_extra["cpu_reference"] = {"ms": round(1e3 * statistics.median(secs), 2), "iterations": used_ref,
                                         "cores": os.cpu_count(), "tag": "tags::CPU::MultiCore::SSE"}
            cg_extra["speedup_vs_cpu_reference"] = round(1e3 * statistics.median(secs) / cg_extra["p50_ms"], 1)

    return cg_extra


def run_ours(args):
    import torch
    from honei_b200 import la, problems as P
    from honei_b200 import replicas

    _, _, local = dist_setup()
    torch.cuda.set_device(local)
    ws, rank, local = replicas.init("nccl", timeout_s=120, device=torch.device("cuda", local))
    ctx = la.Context(local)
    stream = torch.cuda.current_stream()

    def barrier():
        replicas.barrier()
        torch.cuda.synchronize()

    # ---- SpMV workload (replica per rank, assembled on the device) ----
    A = la.SparseMatrixELL.q1_poisson(M_SPMV, ctx=ctx)
    n = A.rows()
    nnz = q1_nnz(M_SPMV)
    x = torch.from_numpy(P.uniform_vector(n, 1 + rank)).cuda()
    y = torch.empty_like(x)
    nbytes = spmv_bytes(nnz, n, 8)

    def step():
        for _ in range(SPMV_PER_STEP):
            la.Product.value(y, A, x, ctx=ctx)

    for _ in range(max(args.warmup, 3)):
        step()
    barrier()
    l0 = ctx.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launches() - l0
    ms = ev0.elapsed_time(ev1)
    ms_max = replicas.max_over_ranks(ms)
    apps = args.steps * SPMV_PER_STEP
    per_launch_s = ms / 1e3 / apps
    value = ws * nbytes * apps / (ms_max / 1e3) / 1e9
    achieved = nbytes / per_launch_s / 1e9
    peak, peak_src = measured_peak()

    # ---- e2e through the public API with host buffers (pinned): every step copies its x from
    # pinned host memory to the device, runs its 10 products and copies its y back to pinned
    # host memory.  Serial: the three in order on one stream.  Pipelined (the reported e2e):
    # the same steps on three streams with double buffers, so the upload of step k + 1 and the
    # download of step k - 1 run during the products of step k. ----
    xh = [torch.from_numpy(P.uniform_vector(n, 7 + rank + k)).pin_memory() for k in range(2)]
    yh = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
    xd = [torch.empty_like(x) for _ in range(2)]
    yd = [torch.empty_like(x) for _ in range(2)]

    def e2e_serial_step():
        xd[0].copy_(xh[0], non_blocking=True)
        for _ in range(SPMV_PER_STEP):
            la.Product.value(yd[0], A, xd[0], ctx=ctx)
        yh[0].copy_(yd[0], non_blocking=True)

    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    for k in range(2):
        ev_comp[k].record(stream)
        ev_out[k].record(stream)

    def e2e_step(k):
        b = k % 2
        s_in.wait_event(ev_comp[b])          # step k - 2's products no longer read xd[b]
        with torch.cuda.stream(s_in):
            xd[b].copy_(xh[b], non_blocking=True)
        ev_in[b].record(s_in)
        stream.wait_event(ev_in[b])
        stream.wait_event(ev_out[b])         # step k - 2's download no longer reads yd[b]
        for _ in range(SPMV_PER_STEP):
            la.Product.value(yd[b], A, xd[b], ctx=ctx)
        ev_comp[b].record(stream)
        s_out.wait_event(ev_comp[b])
        with torch.cuda.stream(s_out):
            yh[b].copy_(yd[b], non_blocking=True)
        ev_out[b].record(s_out)

    def timed_e2e(run_step):
        for k in range(3):
            run_step(k)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s_in.wait_event(e0)
        for k in range(args.steps):
            run_step(k)
        stream.wait_event(ev_out[(args.steps - 1) % 2])
        stream.wait_stream(s_out)
        e1.record(stream)
        torch.cuda.synchronize()
        return replicas.max_over_ranks(e0.elapsed_time(e1))

    def e2e_one_step():
        xd[0].copy_(xh[0], non_blocking=True)
        la.Product.value(yd[0], A, xd[0], ctx=ctx)
        yh[0].copy_(yd[0], non_blocking=True)

    e2e_one_ms = timed_e2e(lambda k: e2e_one_step())
    e2e_one_value = ws * nbytes * args.steps / (e2e_one_ms / 1e3) / 1e9
    e2e_serial_ms = timed_e2e(lambda k: e2e_serial_step())
    ems = timed_e2e(e2e_step)
    e2e_value = ws * nbytes * apps / (ems / 1e3) / 1e9
    e2e_serial_value = ws * nbytes * apps / (e2e_serial_ms / 1e3) / 1e9

    # ---- extras: every other workload of the configurations, on one GPU only (the scaling runs
    # time the headline product alone) ----
    spmv_extra = band_extra = csr_extra = cg_extra = cg_cluster = cg_large = cg_perm = None
    batch_extra = serve_extra = mg_extra = ir_extra = None
    if ws == 1 and not args.no_extras:
        cpu_on = not args.no_cpu_baseline
        spmv_extra = bench_spmv_variants(la, ctx, cpu=cpu_on)
        band_extra = bench_q1band(la, ctx, x, per_launch_s, cpu=cpu_on)
        csr_extra = bench_csr(la, ctx, x, per_launch_s, cpu=cpu_on)
        cg_extra = bench_cg_257(la, ctx, cpu=cpu_on)
        cg_cluster = bench_cg_cluster(ctx)
        cg_large = bench_cg_large(la, ctx, cpu=cpu_on) if not args.no_mg else None
        cg_perm = bench_cg_permuted(la, ctx) if not args.no_mg else None
        batch_extra = None if args.no_batch else bench_batch(la, ctx, n_systems=args.batch_systems)
        # the serving stream before the multi-second 2049^2 solves (their heat lowers the clocks)
        serve_extra = None if args.no_serve else bench_serve(args.serve_requests, args.serve_prefix, args.serve_rate,
                                                              device=local, cpu=cpu_on)
        mg_extra = None if args.no_mg else bench_mg(la, ctx, cpu=cpu_on)
        ir_extra = None if args.no_mg else bench_ir(la, ctx)

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            cpu = cpu_spmv_gbs()
        line = {
            "metric": "ell_spmv_gbs_q1_2049_f64", "value": round(value, 2), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Q1 Poisson 2049^2, x ~ U[-1,1])",
            "config": spmv_config(ws),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_src,
                         "traffic": profile_traffic("ell_spmv_q1_2049_f64"),
                         "kernel": "ell_spmv_kernel<double,9,false>"},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": n * 8,
                    "d2h_bytes_per_step": n * 8, "api": "honei_b200.la.Product.value (C ABI hb_spmv_f64)",
                    "pipeline": "steps on three streams, double-buffered: upload of step k+1 and download of "
                                "step k-1 overlap the products of step k",
                    "serial_value": round(e2e_serial_value, 2),
                    "one_product_per_step": round(e2e_one_value, 2),
                    "honei_plugin": plugin_e2e() if ws == 1 else None},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "extra": {"spmv": spmv_extra, "q1band_2049": band_extra, "csr_2049": csr_extra,
                      "cg_257": cg_extra,
                      "cg_257_cluster": cg_cluster, "cg_large": cg_large, "cg_permuted_2049": cg_perm,
                      "mg_2049": mg_extra, "ir_2049": ir_extra, "batch_512": batch_extra, "serve": serve_extra},
        }
        print(json.dumps(line), flush=True)
    barrier()
    replicas.finish()
    return 0


def run_case(name):
    """One small workload for a profiler capture (ncu -k <kernel> ... python bench.py --case NAME):
    spmv / spmv_permuted / spmv_ordered (2049^2 FP64 products), spmv_f32 (the FP32 product), cg_2049 (the streaming CG kernel,
    200 iterations), mg_2049 (one banded FP64 V(2,2) solve), batch_512 / batch_128 (the
    512-system batch or its first 128 systems, tuned shape), q1batch (48 mid-size served systems in one batched MG-PCG launch), blas1 (dot,
    norm and axpy on 2049^2 vectors).  Prints 'ok' and the case's own figure."""
    import torch
    from honei_b200 import la, problems as P
    torch.cuda.set_device(0)
    ctx = la.Context(0)
    if name == "spmv_f32":
        A = la.SparseMatrixELL.q1_poisson(M_SPMV, ctx=ctx).to_float(ctx=ctx)
        x = torch.from_numpy(P.uniform_vector(M_SPMV ** 2, 6).astype(np.float32)).cuda()
        y = torch.empty_like(x)
        for _ in range(4):
            la.Product.value(y, A, x, ctx=ctx)
    elif name in ("spmv", "spmv_permuted", "spmv_ordered"):
        if name == "spmv":
            A = la.SparseMatrixELL.q1_poisson(M_SPMV, ctx=ctx)
        else:
            A = la.SparseMatrixELL.from_reference(P.q1_poisson_permuted(M_SPMV, 5)[0], ctx)
            if name == "spmv_ordered":
                A = A.ordered(columns=True, ctx=ctx)
        x = torch.from_numpy(P.uniform_vector(M_SPMV ** 2, 6)).cuda()
        y = torch.empty_like(x)
        for _ in range(4):
            la.Product.value(y, A, x, ctx=ctx)
    elif name == "cg_2049":
        A = la.SparseMatrixELL.q1_poisson(M_SPMV, ctx=ctx)
        xt = torch.from_numpy(P.uniform_vector(A.rows(), 1)).cuda()
        b = torch.empty_like(xt)
        la.Product.value(b, A, xt, ctx=ctx)
        print([la.CGSolver.value(A, None, b, torch.zeros_like(xt), 200, 1e-8, ctx=ctx) for _ in range(2)])
    elif name == "mg_2049":
        H = P.mg_hierarchy(M_SPMV)
        data = la.MGData.from_hierarchy(H, np.float64, ctx=ctx, eps=1e-8, max_iters=100,
                                        max_iters_coarse=MG_COARSE_ITERS, banded=True)
        b = torch.from_numpy(P.uniform_vector(M_SPMV ** 2, 5)).cuda()
        print(la.MGSolver.value(data, b, torch.zeros_like(b)))
    elif name in ("batch_512", "batch_128"):
        from honei_b200 import batch as B
        sides = np.random.default_rng(2024).integers(17, 258, size=512)[:int(name.split("_")[1])]
        systems = B.q1_batch(sides, coef_range=(1e-1, 1e1), seed=2024, mode="cg64", eps=1e-8)
        res = B.BatchSolver(systems, ctx=ctx).solve(B.HbBatchConfig(8, 256, 0, 1))
        print(sum(r["iterations"] for r in res))
    elif name == "q1batch":
        from honei_b200 import serve as S
        tr = S.poisson_trace(48, rate=0.0, side_range=(97, 300), seed=3)
        with S.Server(mode="mixed", small_max_side=96, mid_max_side=300) as srv:
            print(S.replay(srv, tr, realtime=False)["paths"])
    elif name == "blas1":
        n = M_SPMV ** 2
        x = torch.from_numpy(P.uniform_vector(n, 1)).cuda()
        y = torch.from_numpy(P.uniform_vector(n, 2)).cuda()
        for _ in range(3):
            la.DotProduct.value(x, y, ctx=ctx)
            la.Norm.value(x, root=True, ctx=ctx)
            la.ScaledSum.value(x, y, 0.5, ctx=ctx)
    else:
        raise SystemExit(f"unknown case {name}")
    torch.cuda.synchronize()
    print("ok")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="the headline product only")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-system batched workload")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream workload")
    ap.add_argument("--batch-systems", type=int, default=512, help="systems in the batched workload")
    ap.add_argument("--no-mg", action="store_true", help="skip the 2049^2 MG and mixed-precision workloads")
    ap.add_argument("--serve-requests", type=int, default=20000, help="requests in the serving stream")
    ap.add_argument("--serve-prefix", type=int, default=2000,
                    help="first requests of the stream served by the plain FP64 CG baselines")
    ap.add_argument("--serve-rate", type=float, default=SERVE_RATE, help="Poisson arrivals per second (latency)")
    ap.add_argument("--case", default=None, help="run one small workload for a profiler capture and exit")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
