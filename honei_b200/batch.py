"""Batched solves: many independent systems in one persistent launch (hb_batch_* in the C ABI).

    systems = q1_batch(sides, coef_range=(1e-1, 1e1), seed=0, mode="ir32")
    solver = BatchSolver(systems)             # workspace + device descriptors
    cfg = solver.tune()                       # autotuner (cached in a JSON file)
    results = solver.solve(cfg)               # list of dicts, one per system

Each system is solved by one thread-block cluster; the launch shape (CTAs per cluster,
threads per CTA) is the tunable.  The autotuner times every shape on the batch and caches the
winner in a JSON file keyed by GPU, mode, precision and the batch's size profile
(``$HONEI_B200_TUNE_CACHE``, default ``~/.cache/honei_b200/batch_tune.json``).
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np
import torch

from . import problems as P
from ._lib import HbEll, check, lib
from .la import SparseMatrixELL, default_context

HB_BATCH_CG64, HB_BATCH_IR32 = 0, 1
CLUSTERS = (1, 2, 4, 8, 16)
THREADS = (256, 512)
ROWS_PER_THREAD = (4, 1)


class HbBatchSystem(C.Structure):
    _fields_ = [("A64", HbEll), ("A32", HbEll), ("b", C.c_void_p), ("x", C.c_void_p), ("mode", C.c_int32),
                ("pad_", C.c_int32), ("max_iters", C.c_int64), ("max_outer", C.c_int64), ("eps", C.c_double),
                ("inner_eps", C.c_double)]


class HbBatchResult(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("outer", C.c_int64), ("defect0", C.c_double), ("defect", C.c_double),
                ("true_relres", C.c_double), ("status", C.c_int32), ("pad_", C.c_int32)]


class HbBatchConfig(C.Structure):
    _fields_ = [("cluster", C.c_int32), ("threads", C.c_int32), ("max_clusters", C.c_int32),
                ("rows_per_thread", C.c_int32)]


def _register():
    L = lib()
    vp, i64 = C.c_void_p, C.c_int64
    L.hb_batch_workspace_bytes.argtypes = [C.POINTER(HbBatchSystem), i64, C.POINTER(C.c_size_t)]
    L.hb_batch_solve.argtypes = [vp, C.POINTER(HbBatchSystem), i64, vp, C.POINTER(HbBatchConfig),
                                 C.POINTER(HbBatchResult)]
    L.hb_batch_prepare.argtypes = [vp, C.POINTER(HbBatchSystem), i64, vp]
    L.hb_batch_run.argtypes = [vp, i64, vp, C.POINTER(HbBatchConfig)]
    L.hb_batch_results.argtypes = [vp, i64, vp, C.POINTER(HbBatchResult)]
    L.hb_batch_tune.argtypes = [vp, C.POINTER(HbBatchSystem), i64, vp, C.POINTER(HbBatchConfig),
                                C.POINTER(C.c_double)]
    for n in ("hb_batch_workspace_bytes", "hb_batch_solve", "hb_batch_prepare", "hb_batch_run",
              "hb_batch_results", "hb_batch_tune"):
        getattr(L, n).restype = C.c_int
    return L


class System:
    """One system of a batch: device matrix (FP64, plus FP32 values sharing its index array for
    the mixed-precision mode), right-hand side and solution vector."""

    def __init__(self, A64: SparseMatrixELL, b: torch.Tensor, x: torch.Tensor | None = None, mode="ir32",
                 eps=1e-8, inner_eps=1e-3, max_iters=100000, max_outer=50, A32: SparseMatrixELL | None = None):
        self.A64 = A64
        self.mode = HB_BATCH_IR32 if mode in ("ir32", HB_BATCH_IR32) else HB_BATCH_CG64
        if self.mode == HB_BATCH_IR32 and A32 is None:
            Ax32 = torch.empty(A64.K * A64.ld, dtype=torch.float32, device=A64.Ax.device)
            A32 = SparseMatrixELL(A64.rows(), A64.columns(), A64.K, A64.ld, A64.Aj, Ax32)
            check(lib().hb_ell_cast_f64_f32(default_context().handle, C.byref(A64.struct), C.byref(A32.struct)),
                  "hb_ell_cast_f64_f32")
        self.A32 = A32
        self.b = b
        self.x = torch.zeros_like(b) if x is None else x
        self.eps, self.inner_eps, self.max_iters, self.max_outer = eps, inner_eps, max_iters, max_outer

    @property
    def n(self):
        return self.A64.rows()

    def struct(self) -> HbBatchSystem:
        a32 = self.A32.struct if self.A32 is not None else HbEll()
        return HbBatchSystem(self.A64.struct, a32, self.b.data_ptr(), self.x.data_ptr(), self.mode, 0,
                             self.max_iters, self.max_outer, self.eps, self.inner_eps)


def q1_system(M: int, coef_range=(1e-1, 1e1), seed: int = 0, mode="ir32", symmetric=True, **kw) -> System:
    """Seeded Q1 Poisson system: cellwise log-uniform coefficient, b = A x_true, x_true ~ U[-1,1].

    symmetric=True (default for batches): Dirichlet couplings eliminated, so the system is SPD."""
    ctx = default_context()
    coef = None
    if coef_range is not None:
        coef = torch.from_numpy(P.log_uniform_coef(M, coef_range[0], coef_range[1], seed).ravel()).cuda()
    A = SparseMatrixELL.q1_poisson(M, coef, ctx=ctx, symmetric=symmetric)
    xt = torch.from_numpy(P.uniform_vector(M * M, seed + 1)).cuda()
    b = torch.empty_like(xt)
    from .la import Product
    Product.value(b, A, xt, ctx=ctx)
    s = System(A, b, mode=mode, **kw)
    s.x_true = xt
    return s


def q1_batch(sides, coef_range=(1e-1, 1e1), seed=0, mode="ir32", symmetric=True, **kw) -> list:
    """One seeded system per grid side (seeds = seed + i)."""
    return [q1_system(int(M), coef_range, seed + i, mode, symmetric, **kw) for i, M in enumerate(sides)]


def _cache_path():
    return os.environ.get("HONEI_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "honei_b200", "batch_tune.json"))


class BatchSolver:
    """Workspace, descriptors and launches for one batch of systems."""

    def __init__(self, systems, ctx=None):
        self.L = _register()
        self.ctx = ctx or default_context()
        self.systems = list(systems)
        self.count = len(self.systems)
        self._arr = (HbBatchSystem * max(self.count, 1))(*[s.struct() for s in self.systems])
        nbytes = C.c_size_t(0)
        check(self.L.hb_batch_workspace_bytes(self._arr, self.count, C.byref(nbytes)), "hb_batch_workspace_bytes")
        self.workspace = torch.empty(nbytes.value + 256, dtype=torch.uint8, device="cuda")
        self._ws = (self.workspace.data_ptr() + 255) // 256 * 256
        self.prepared = False

    def signature(self) -> str:
        """Cache key: GPU, modes and the size profile of the batch (log2 buckets of rows)."""
        gpu = torch.cuda.get_device_name()
        modes = sorted({s.mode for s in self.systems})
        hist = np.bincount([int(np.log2(max(s.n, 1))) for s in self.systems], minlength=32)
        return f"{gpu}|modes={modes}|n={self.count}|hist={','.join(map(str, hist))}"

    def prepare(self):
        check(self.L.hb_batch_prepare(self.ctx.handle, self._arr, self.count, C.c_void_p(self._ws)),
              "hb_batch_prepare", self.ctx.handle)
        self.prepared = True

    def run(self, cfg: HbBatchConfig | None = None):
        """Asynchronous launch on the context stream (after prepare)."""
        if not self.prepared:
            self.prepare()
        check(self.L.hb_batch_run(self.ctx.handle, self.count, C.c_void_p(self._ws),
                                  C.byref(cfg) if cfg is not None else None), "hb_batch_run", self.ctx.handle)

    def results(self) -> list:
        res = (HbBatchResult * max(self.count, 1))()
        check(self.L.hb_batch_results(self.ctx.handle, self.count, C.c_void_p(self._ws), res), "hb_batch_results",
              self.ctx.handle)
        return [dict(iterations=r.iterations, outer=r.outer, defect0=r.defect0, defect=r.defect,
                     true_relres=r.true_relres, status=r.status) for r in res[: self.count]]

    def solve(self, cfg: HbBatchConfig | None = None) -> list:
        self.run(cfg)
        return self.results()

    def tune(self, use_cache=True) -> HbBatchConfig:
        """Autotuner: times every (rows per thread, cluster, threads) shape, keeps the fastest,
        caches it."""
        key = self.signature()
        path = _cache_path()
        cache = {}
        if use_cache and os.path.exists(path):
            try:
                cache = json.load(open(path))
            except (OSError, ValueError):
                cache = {}
        if use_cache and key in cache:
            c = cache[key]
            return HbBatchConfig(int(c["cluster"]), int(c["threads"]), 0, int(c.get("rows_per_thread", 4)))
        best = HbBatchConfig(4, 512, 0, 4)
        n = len(ROWS_PER_THREAD) * len(CLUSTERS) * len(THREADS)
        times = (C.c_double * n)()
        check(self.L.hb_batch_tune(self.ctx.handle, self._arr, self.count, C.c_void_p(self._ws), C.byref(best), times),
              "hb_batch_tune", self.ctx.handle)
        self.prepared = True
        self.tune_times = {f"r{r}_c{c}_t{t}": round(times[(k * len(CLUSTERS) + i) * len(THREADS) + j], 4)
                           for k, r in enumerate(ROWS_PER_THREAD) for i, c in enumerate(CLUSTERS)
                           for j, t in enumerate(THREADS)}
        cache[key] = {"cluster": best.cluster, "threads": best.threads, "rows_per_thread": best.rows_per_thread,
                      "times_ms": self.tune_times}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            json.dump(cache, open(path, "w"), indent=1)
        except OSError:
            pass
        for s in self.systems:      # the tuner overwrote x
            s.x.zero_()
        return best
