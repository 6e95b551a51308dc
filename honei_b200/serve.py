"""The serving loop (hb_server_* in the C ABI): Q1 solve requests admitted by an HBM budget and
served concurrently on the device, with a trace generator and a replay driver that reports
p50/p99 latency and solves/s.

    trace = poisson_trace(200, rate=150.0, seed=0)      # arrivals, sides, coefficients, x_true
    with Server(mode="mixed") as srv:
        report = replay(srv, trace)                     # latencies, solves/s, per-request records

A request is one M x M node Q1 system in the SPD form (Dirichlet rows and columns eliminated)
with a cellwise coefficient and b = A x_true; the server assembles it on the device, solves it to
``eps`` relative FP64 residual and copies x back into the request's host array.  ``mode="mixed"``
serves small grids in batched cluster launches (FP32 CG inside FP64 refinement) and large grids on
MG-preconditioned mixed-precision workers; ``mode="plain"`` is the baseline on the same queue:
plain FP64 CG, one request at a time; ``mode="plain_batched"`` is plain FP64 CG with the mixed
server's concurrency (batched cluster launches up to ``mid_max_side``, concurrent whole-GPU CG
workers above).  No reference counterpart: HONEI solves one system per call.

Long streams (the 20,000-request configuration) are generated on demand: ``stream_trace`` holds
only sides, arrival times and seeds, and ``replay_stream`` stages each request's host buffers
shortly before it is submitted and lets them go once it completes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import problems as P
from ._lib import HBError, lib, status_string
from .batch import HbBatchConfig

HB_SERVE_MIXED, HB_SERVE_PLAIN_CG64, HB_SERVE_PLAIN_CG64_BATCHED = 0, 1, 2
MODES = {"mixed": HB_SERVE_MIXED, "plain": HB_SERVE_PLAIN_CG64, "plain_batched": HB_SERVE_PLAIN_CG64_BATCHED}
PATHS = {0: "batch", 1: "mgpcg", 2: "cg64", 3: "mgbatch", 4: "batch_cg64"}


class HbServerParams(C.Structure):
    _fields_ = [("mode", C.c_int32), ("device", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("large_workers", C.c_int32), ("small_workers", C.c_int32), ("small_max_side", C.c_int64),
                ("max_batch", C.c_int32), ("pad_", C.c_int32), ("batch_cfg", HbBatchConfig),
                ("eps", C.c_double), ("inner_eps", C.c_double), ("mid_max_side", C.c_int64),
                ("mid_workers", C.c_int32), ("pad2_", C.c_int32), ("mid_cfg", HbBatchConfig), ("pad3_", C.c_int32)]


class HbRequest(C.Structure):
    _fields_ = [("M", C.c_int64), ("coef", C.c_void_p), ("b", C.c_void_p), ("x_true", C.c_void_p),
                ("x", C.c_void_p), ("tag", C.c_uint64)]


class HbCompletion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int32), ("path", C.c_int32), ("iterations", C.c_int64),
                ("outer", C.c_int64), ("true_relres", C.c_double), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("bytes", C.c_int64)]


def _register():
    L = lib()
    vp, i32, P_i64 = C.c_void_p, C.c_int, C.POINTER(C.c_int64)
    L.hb_server_create.argtypes = [C.POINTER(HbServerParams), C.POINTER(vp)]
    L.hb_server_submit.argtypes = [vp, C.POINTER(HbRequest)]
    L.hb_server_poll.argtypes = [vp, C.POINTER(HbCompletion), i32, C.POINTER(i32), i32]
    L.hb_server_drain.argtypes = [vp]
    L.hb_server_clock.argtypes = [vp]
    L.hb_server_clock.restype = C.c_double
    L.hb_server_stats.argtypes = [vp, P_i64, P_i64, P_i64, P_i64]
    L.hb_server_pool_stats.argtypes = [vp, P_i64, P_i64]
    L.hb_server_destroy.argtypes = [vp]
    for n in ("hb_server_create", "hb_server_submit", "hb_server_poll", "hb_server_drain", "hb_server_stats",
              "hb_server_pool_stats", "hb_server_destroy"):
        getattr(L, n).restype = C.c_int
    return L


def _host_array(n: int, pinned: bool) -> np.ndarray:
    """A float64 host array; page-locked (through torch) when asked, so the server's copies are
    asynchronous DMA transfers."""
    if pinned:
        import torch
        if torch.cuda.is_available():
            # the array's base is the tensor, which keeps the pinned block alive
            return torch.empty(max(n, 1), dtype=torch.float64, pin_memory=True).numpy()[:n]
    return np.empty(n, dtype=np.float64)


def _as_host(a: np.ndarray | None, pinned: bool) -> np.ndarray | None:
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    if not pinned:
        return a
    h = _host_array(a.size, True)
    h[:] = a
    return h


@dataclass
class Request:
    """One solve request: grid side M, optional (M-1)^2 cell coefficients, and either b or x_true
    (b = A x_true, formed on the device)."""
    M: int
    coef: np.ndarray | None = None
    x_true: np.ndarray | None = None
    b: np.ndarray | None = None
    arrival: float = 0.0
    tag: int = 0


@dataclass
class Trace:
    requests: list
    rate: float
    seed: int
    side_range: tuple
    coef_range: tuple

    @property
    def rows(self) -> int:
        return int(sum(r.M * r.M for r in self.requests))


class StreamTrace:
    """A serving stream whose requests are generated on demand.  Request i's side, arrival time,
    coefficient and x_true depend only on (seed, i) and the ranges, so the first k requests of a
    long stream are the k-request stream of the same seed, and ``request(i)`` always returns the
    same data."""

    def __init__(self, count: int, rate: float, side_range=(33, 1025), coef_range=(1e-2, 1e2), seed: int = 0,
                 arrival_seed: int | None = None):
        rng = np.random.default_rng(seed)
        lo, hi = side_range
        sides = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)
        self.sides = np.clip(sides, lo, hi)
        arng = np.random.default_rng(seed + 1 if arrival_seed is None else arrival_seed)
        gaps = arng.exponential(1.0 / rate, size=count) if rate > 0 else np.zeros(count)
        self.arrivals = np.cumsum(gaps) - (gaps[0] if count else 0.0)
        self.rate, self.seed = rate, seed
        self.side_range, self.coef_range = tuple(side_range), tuple(coef_range)
        self.arrival_seed = arrival_seed

    def __len__(self) -> int:
        return len(self.sides)

    @property
    def rows(self) -> int:
        return int(np.sum(self.sides.astype(np.int64) ** 2))

    def request(self, i: int) -> Request:
        M = int(self.sides[i])
        lo, hi = self.coef_range
        coef = P.log_uniform_coef(M, lo, hi, self.seed * 1000003 + i).ravel()
        xt = P.uniform_vector(M * M, self.seed * 1000003 + i + 7)
        return Request(M=M, coef=coef, x_true=xt, arrival=float(self.arrivals[i]), tag=i)

    def prefix(self, k: int) -> "StreamTrace":
        t = StreamTrace.__new__(StreamTrace)
        t.__dict__.update(self.__dict__)
        t.sides, t.arrivals = self.sides[:k], self.arrivals[:k]
        return t


def stream_trace(count: int, rate: float, side_range=(33, 1025), coef_range=(1e-2, 1e2), seed: int = 0,
                 arrival_seed: int | None = None) -> StreamTrace:
    """``count`` requests with Poisson-process arrivals of ``rate`` per second (exponential gaps;
    rate 0: all at once), grid side log-uniform in ``side_range`` (rounded to an integer), a
    log-uniform cellwise coefficient in ``coef_range`` and x_true uniform in [-1, 1], all from
    ``seed``; generated on demand."""
    return StreamTrace(count, rate, side_range, coef_range, seed, arrival_seed)


def poisson_trace(count: int, rate: float, side_range=(33, 1025), coef_range=(1e-2, 1e2), seed: int = 0,
                  arrival_seed: int | None = None) -> Trace:
    """The requests of ``stream_trace(count, rate, ...)``, all generated now."""
    st = StreamTrace(count, rate, side_range, coef_range, seed, arrival_seed)
    return Trace([st.request(i) for i in range(count)], rate, seed, tuple(side_range), tuple(coef_range))


@dataclass
class Completion:
    tag: int
    status: int
    path: str
    iterations: int
    outer: int
    true_relres: float
    t_submit: float
    t_admit: float
    t_done: float
    bytes: int
    x: np.ndarray = field(repr=False, default=None)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class Server:
    """Owns an ``hb_server``.  ``mode``: "mixed" (batched small grids, optionally batched MG-PCG
    cluster launches for grids up to ``mid_max_side``, MG-PCG workers for the large ones) or
    "plain" (FP64 CG one request at a time).  ``budget_bytes`` bounds the estimated
    device bytes of the admitted requests; a request above the budget alone is refused at
    submit with HB_ERR_CAPACITY."""

    def __init__(self, mode: str = "mixed", budget_bytes: int = 64 << 30, large_workers: int = 16,
                 small_workers: int = 2, small_max_side: int = 96, max_batch: int = 32, cluster: int = 2,
                 threads: int = 512, max_clusters: int = 0, eps: float = 1e-8, inner_eps: float = 1e-3,
                 device: int = 0, pinned: bool = True, mid_max_side: int = 300, mid_workers: int = 3,
                 mid_cluster: int = 16, mid_threads: int = 512, mid_max_clusters: int = 0):
        self._lib = _register()
        prm = HbServerParams()
        prm.mode = MODES[mode]
        prm.device = device
        prm.hbm_budget_bytes = int(budget_bytes)
        prm.large_workers = large_workers
        prm.small_workers = small_workers
        prm.small_max_side = small_max_side
        prm.max_batch = max_batch
        prm.batch_cfg = HbBatchConfig(cluster, threads, max_clusters)
        prm.eps = eps
        prm.inner_eps = inner_eps
        prm.mid_max_side = mid_max_side
        prm.mid_workers = mid_workers
        prm.mid_cfg = HbBatchConfig(mid_cluster, mid_threads, mid_max_clusters)
        self.mode = mode
        self.params = prm
        self.pinned = pinned
        h = C.c_void_p()
        st = self._lib.hb_server_create(C.byref(prm), C.byref(h))
        if st:
            raise HBError(st, "hb_server_create")
        self.handle = h
        self._live = {}

    def stage(self, req: Request):
        """The request's host buffers (page-locked when the server is) and its C record: the
        input data as it sits in host memory before the request arrives."""
        n = req.M * req.M
        coef = _as_host(req.coef, self.pinned)
        b = _as_host(req.b, self.pinned)
        xt = _as_host(req.x_true, self.pinned) if b is None else None
        x = _host_array(n, self.pinned)
        r = HbRequest(req.M, coef.ctypes.data if coef is not None else None,
                      b.ctypes.data if b is not None else None, xt.ctypes.data if xt is not None else None,
                      x.ctypes.data, req.tag)
        return r, (coef, b, xt, x)

    def submit(self, req: Request, staged=None) -> int:
        """Queues ``req`` (staged by ``stage`` or now); returns its tag.  The host arrays stay
        referenced until it completes."""
        r, held = staged if staged is not None else self.stage(req)
        self._live[req.tag] = held
        st = self._lib.hb_server_submit(self.handle, C.byref(r))
        if st:
            del self._live[req.tag]
            raise HBError(st, "hb_server_submit", status_string(st))
        return req.tag

    def poll(self, max_items: int = 256, wait_ms: int = 0) -> list:
        buf = (HbCompletion * max_items)()
        n = C.c_int()
        st = self._lib.hb_server_poll(self.handle, buf, max_items, C.byref(n), wait_ms)
        if st:
            raise HBError(st, "hb_server_poll")
        out = []
        for c in buf[:n.value]:
            held = self._live.pop(c.tag, None)
            out.append(Completion(int(c.tag), int(c.status), PATHS.get(c.path, str(c.path)), int(c.iterations),
                                  int(c.outer), float(c.true_relres), c.t_submit, c.t_admit, c.t_done,
                                  int(c.bytes), held[3] if held else None))
        return out

    def drain(self) -> list:
        st = self._lib.hb_server_drain(self.handle)
        if st:
            raise HBError(st, "hb_server_drain")
        return self.poll(max(1, len(self._live) + 1))

    def clock(self) -> float:
        return self._lib.hb_server_clock(self.handle)

    def stats(self) -> dict:
        v = [C.c_int64() for _ in range(4)]
        self._lib.hb_server_stats(self.handle, *[C.byref(x) for x in v])
        out = dict(zip(("bytes_in_use", "bytes_peak", "submitted", "completed"), (x.value for x in v)))
        u, r = C.c_int64(), C.c_int64()
        if self._lib.hb_server_pool_stats(self.handle, C.byref(u), C.byref(r)) == 0:
            out["pool_used_high"], out["pool_reserved_high"] = u.value, r.value
        return out

    def close(self):
        if self.handle:
            self._lib.hb_server_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def replay(server: Server, trace: Trace, realtime: bool = True) -> dict:
    """Stages every request's host buffers, then submits the requests at their arrival times (on
    the server clock; all at once when ``realtime`` is false), collects every completion and
    summarises them: solves/s over the
    makespan (first submit to last completion), latency percentiles (submit to completion, so
    queueing included) and service times (admission to completion)."""
    done = []
    staged = [server.stage(req) for req in trace.requests]
    t_base = server.clock()
    for req, st in zip(trace.requests, staged):
        if realtime:
            while True:
                lag = t_base + req.arrival - server.clock()
                if lag <= 0:
                    break
                done += server.poll(256, wait_ms=max(0, min(int(lag * 1000), 20)))
                if lag < 0.001:
                    while server.clock() < t_base + req.arrival:
                        pass
                    break
        server.submit(req, st)
    done += server.drain()
    return summarise(done)


def replay_stream(server: Server, trace: StreamTrace, realtime: bool = True, window: int = 512,
                  lookahead: int = 256, producers: int = 4, keep_x: bool = False) -> dict:
    """Serves a stream that is generated while it runs.  Producer threads build and stage request
    i (its host buffers, page-locked when the server is) ahead of its turn, at most
    ``lookahead`` requests ahead.  With ``realtime`` the requests are submitted at their arrival
    times (open loop; a request staged late is submitted late, and its latency counts from its
    scheduled arrival); without it, as fast as the server takes them with at most ``window``
    requests outstanding (closed loop: the server's capacity).  A request's host buffers are
    released when its completion is collected (its solution too, unless ``keep_x``)."""
    import threading

    n = len(trace)
    ready: dict = {}
    cv = threading.Condition()
    state = {"next": 0, "submitted": 0, "stop": False, "error": None}

    def produce():
        try:
            while True:
                with cv:
                    cv.wait_for(lambda: state["stop"] or state["next"] >= n
                                or state["next"] < state["submitted"] + lookahead)
                    if state["stop"] or state["next"] >= n:
                        return
                    i = state["next"]
                    state["next"] += 1
                req = trace.request(i)
                staged = server.stage(req)
                req.coef = req.x_true = None          # the staged copies are what the server reads
                with cv:
                    ready[i] = (req, staged)
                    cv.notify_all()
        except BaseException as e:  # reported by the submitting thread
            with cv:
                state["error"] = e
                state["stop"] = True
                cv.notify_all()

    threads = [threading.Thread(target=produce, daemon=True) for _ in range(max(1, producers))]
    for t in threads:
        t.start()
    done, lag_max = [], 0.0
    outstanding = 0

    def collect(wait_ms):
        nonlocal outstanding
        got = server.poll(256, wait_ms=wait_ms)
        for c in got:
            if not keep_x:
                c.x = None
        outstanding -= len(got)
        done.extend(got)

    t_base = server.clock()
    sched = {}
    try:
        for i in range(n):
            with cv:
                cv.wait_for(lambda: i in ready or state["stop"])
                if state["error"] is not None:
                    raise state["error"]
                req, staged = ready.pop(i)
            if realtime:
                target = t_base + float(trace.arrivals[i])
                while True:
                    lag = target - server.clock()
                    if lag <= 0:
                        break
                    collect(max(0, min(int(lag * 1000), 20)))
                    if lag < 0.001:
                        while server.clock() < target:
                            pass
                        break
                sched[req.tag] = target
            else:
                while outstanding >= window:
                    collect(20)
            server.submit(req, staged)
            outstanding += 1
            if realtime:
                lag_max = max(lag_max, server.clock() - sched[req.tag])
            with cv:
                state["submitted"] = i + 1
                cv.notify_all()
            if outstanding and i % 16 == 0:
                collect(0)
    finally:
        with cv:
            state["stop"] = True
            cv.notify_all()
        for t in threads:
            t.join()
    rest = server.drain()
    for c in rest:
        if not keep_x:
            c.x = None
    done.extend(rest)
    if realtime:
        # latency from the scheduled arrival (covers a late submission)
        for c in done:
            c.t_submit = min(c.t_submit, sched.get(c.tag, c.t_submit))
    out = summarise(done)
    out["submit_lag_max_ms"] = lag_max * 1e3
    out["mode"] = "open loop (arrival times)" if realtime else f"closed loop, {window} outstanding"
    return out


def summarise(done: list) -> dict:
    lat = np.array([c.latency for c in done]) if done else np.zeros(1)
    svc = np.array([c.t_done - c.t_admit for c in done]) if done else np.zeros(1)
    t0 = min((c.t_submit for c in done), default=0.0)
    t1 = max((c.t_done for c in done), default=0.0)
    ok = [c for c in done if c.status == 0]
    paths = {}
    for c in done:
        paths[c.path] = paths.get(c.path, 0) + 1
    return {
        "completed": len(done),
        "ok": len(ok),
        "makespan_s": t1 - t0,
        "solves_per_s": len(ok) / (t1 - t0) if t1 > t0 else 0.0,
        "p50_ms": float(np.percentile(lat, 50) * 1e3),
        "p99_ms": float(np.percentile(lat, 99) * 1e3),
        "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
        "service_p99_ms": float(np.percentile(svc, 99) * 1e3),
        "max_true_relres": max((c.true_relres for c in ok), default=float("nan")),
        "paths": paths,
        "records": done,
    }
