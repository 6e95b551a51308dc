"""ctypes bindings to the parity oracles.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``    -- oracle/_build/libhonei_oracle.so, the plain-C restatement (honei_oracle.c).
* ``Reference`` -- oracle/_ref/libhonei_ref.so, the reference's own CPU path compiled from the
                   unmodified HONEI sources plus ref_shim.cc (present where it was built).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhonei_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhonei_ref.so")

_c = ctypes
_u64 = _c.c_uint64
_vp = _c.c_void_p

TAGS = {"cpu": 0, "generic": 1, "sse": 2, "mc-generic": 3, "mc-sse": 4}


def build_oracle() -> None:
    """Compiles the C restatement (and the reference shim when the HONEI tree is present)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


class _OraEll(_c.Structure):
    _fields_ = [("rows", _u64), ("cols", _u64), ("stride", _u64), ("ncpr", _u64),
                ("threads", _u64), ("Aj", _vp), ("Ax", _vp), ("Arl", _vp)]


class _OraMG(_c.Structure):
    _fields_ = [("nlevels", _c.c_int), ("A", _c.POINTER(_OraEll)), ("prol", _c.POINTER(_OraEll)),
                ("res", _c.POINTER(_OraEll)), ("max_iters", _u64), ("max_iters_coarse", _u64),
                ("n_pre", _u64), ("n_post", _u64)]


class _OraCsr(_c.Structure):
    _fields_ = [("rows", _u64), ("cols", _u64), ("blocksize", _u64), ("Ar", _vp), ("Aj", _vp), ("Ax", _vp)]


def _csr(A):
    e = _OraCsr(A.rows, A.cols, A.blocksize, A.Ar.ctypes.data, A.Aj.ctypes.data, A.Ax.ctypes.data)
    e._keep = A
    return e


def _ell(A):
    e = _OraEll(A.rows, A.cols, A.stride, A.ncpr, A.threads, A.Aj.ctypes.data, A.Ax.ctypes.data,
                A.Arl.ctypes.data)
    e._keep = A
    return e


class Oracle:
    """The plain-C restatement of the HONEI path."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        self.lib = _c.CDLL(path)
        L = self.lib
        for name, res in [("ora_dot_f64", _c.c_double), ("ora_dot_f32", _c.c_float)]:
            getattr(L, name).restype = res
        L.ora_dot_f64.argtypes = [_u64, _vp, _vp]
        L.ora_dot_f32.argtypes = [_u64, _vp, _vp]
        L.ora_cg_f64.argtypes = [_vp, _vp, _vp, _u64, _c.c_double, _c.POINTER(_u64), _vp]
        L.ora_cg_f32.argtypes = [_vp, _vp, _vp, _u64, _c.c_float, _c.POINTER(_u64), _vp]
        L.ora_mg_f64.argtypes = [_vp, _c.c_double, _vp, _vp, _c.c_double, _c.POINTER(_u64), _vp]
        L.ora_mg_f32.argtypes = [_vp, _c.c_float, _vp, _vp, _c.c_float, _c.POINTER(_u64), _vp]
        L.ora_ir_mg.argtypes = [_vp, _vp, _c.c_float, _vp, _vp, _c.c_double, _c.c_float, _u64,
                                _c.c_int, _c.POINTER(_u64), _vp]
        L.ora_ir_cg.argtypes = [_vp, _vp, _vp, _vp, _c.c_double, _c.c_float, _u64, _u64,
                                _c.POINTER(_u64), _c.POINTER(_u64), _vp]
        L.ora_ir_pcg.argtypes = [_vp, _vp, _c.c_float, _vp, _vp, _c.c_double, _c.c_float, _u64, _u64,
                                 _c.POINTER(_u64), _c.POINTER(_u64), _vp]
        for n in ("ora_scaled_sum_f64", "ora_scale_f64"):
            getattr(L, n).argtypes = [_u64, _vp, _vp, _c.c_double] if n == "ora_scaled_sum_f64" \
                else [_u64, _vp, _c.c_double]
        L.ora_scaled_sum3_f64.argtypes = [_u64, _vp, _vp, _vp, _c.c_double]

    @staticmethod
    def _suffix(dtype):
        return "f64" if np.dtype(dtype) == np.float64 else "f32"

    def spmv(self, A, x):
        s = self._suffix(A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        y = np.zeros(A.rows, A.dtype)
        e = _ell(A)
        getattr(self.lib, f"ora_spmv_{s}")(_c.byref(e), _ptr(x), _ptr(y))
        return y

    def csr_spmv(self, A, x):
        """Product<tags::CPU>(DV, SparseMatrixCSR, DV) restated; A a problems.CsrMatrix."""
        s = self._suffix(A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        y = np.zeros(A.rows, A.dtype)
        e = _csr(A)
        getattr(self.lib, f"ora_csr_spmv_{s}")(_c.byref(e), _ptr(x), _ptr(y))
        return y

    def csr_defect(self, A, b, x):
        s = self._suffix(A.dtype)
        b = np.ascontiguousarray(b, A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        r = np.zeros(A.rows, A.dtype)
        e = _csr(A)
        getattr(self.lib, f"ora_csr_defect_{s}")(_c.byref(e), _ptr(b), _ptr(x), _ptr(r))
        return r

    def defect(self, A, b, x):
        s = self._suffix(A.dtype)
        b = np.ascontiguousarray(b, A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        r = np.zeros(A.rows, A.dtype)
        e = _ell(A)
        getattr(self.lib, f"ora_defect_{s}")(_c.byref(e), _ptr(b), _ptr(x), _ptr(r))
        return r

    @staticmethod
    def _bands(bands, dtype):
        bands = [np.ascontiguousarray(b, dtype) for b in bands]
        return bands, (_vp * 9)(*[b.ctypes.data for b in bands])

    def q1band_spmv(self, bands, x):
        """Product<tags::CPU> on BandedMatrixQx<Q1Type> (bands: 9 arrays, LL..UU)."""
        dt = np.asarray(bands[0]).dtype
        keep, bp = self._bands(bands, dt)
        x = np.ascontiguousarray(x, dt)
        y = np.zeros(len(x), dt)
        getattr(self.lib, f"ora_q1band_spmv_{self._suffix(dt)}")(_u64(len(x)), bp, _ptr(x), _ptr(y))
        return y

    def q1band_defect(self, bands, b, x):
        dt = np.asarray(bands[0]).dtype
        keep, bp = self._bands(bands, dt)
        b = np.ascontiguousarray(b, dt)
        x = np.ascontiguousarray(x, dt)
        r = np.zeros(len(x), dt)
        getattr(self.lib, f"ora_q1band_defect_{self._suffix(dt)}")(_u64(len(x)), bp, _ptr(b), _ptr(x), _ptr(r))
        return r

    def q1band_poisson(self, M):
        out = [np.zeros(M * M) for _ in range(9)]
        bp = (_vp * 9)(*[b.ctypes.data for b in out])
        self.lib.ora_q1band_poisson_f64(_u64(M * M), bp)
        return out

    def prolongate(self, coarse, mask, n_fine):
        """Prolongation<methods::NONE>: the fine vector (n_fine entries) from `coarse`."""
        coarse = np.ascontiguousarray(coarse)
        fine = np.zeros(n_fine, coarse.dtype)
        m = np.ascontiguousarray(mask, np.uint64)
        getattr(self.lib, f"ora_prolongate_{self._suffix(coarse.dtype)}")(_u64(n_fine), _ptr(fine), _ptr(coarse),
                                                                          _ptr(m))
        return fine

    def restrict(self, fine, mask):
        """Restriction<methods::NONE>: the coarse vector of `fine`."""
        fine = np.ascontiguousarray(fine)
        side = int(round(np.sqrt(len(fine))))
        nc = ((side - 1) // 2 + 1) ** 2
        coarse = np.zeros(nc, fine.dtype)
        m = np.ascontiguousarray(mask, np.uint64)
        getattr(self.lib, f"ora_restrict_{self._suffix(fine.dtype)}")(_u64(len(fine)), _ptr(coarse), _ptr(fine),
                                                                       _ptr(m))
        return coarse

    def dot(self, x, y):
        x = np.ascontiguousarray(x)
        y = np.ascontiguousarray(y, x.dtype)
        f = self.lib.ora_dot_f64 if x.dtype == np.float64 else self.lib.ora_dot_f32
        return f(len(x), _ptr(x), _ptr(y))

    def cg(self, A, b, x0=None, max_iters=10000, eps=1e-8, history=False):
        """Returns (x, used_iters[, sqrt(alpha) history])."""
        s = self._suffix(A.dtype)
        b = np.ascontiguousarray(b, A.dtype)
        x = np.zeros(A.rows, A.dtype) if x0 is None else np.array(x0, A.dtype)
        used = _u64(0)
        hist = np.zeros(max_iters + 1, A.dtype)
        e = _ell(A)
        getattr(self.lib, f"ora_cg_{s}")(_c.byref(e), _ptr(b), _ptr(x), max_iters, eps,
                                         _c.byref(used), _ptr(hist))
        if history:
            return x, used.value, hist[: used.value + 1]
        return x, used.value

    def cg_var(self, A, P, b, x0=None, max_iters=10000, eps=1e-8):
        """CGSolver<VAR>: P a vector (element product) or an EllMatrix.  (x, used_iters)."""
        s = self._suffix(A.dtype)
        b = np.ascontiguousarray(b, A.dtype)
        x = np.zeros(A.rows, A.dtype) if x0 is None else np.array(x0, A.dtype)
        used = _u64(0)
        e = _ell(A)
        f = getattr(self.lib, f"ora_cg_var_{s}")
        f.argtypes = [_vp, _vp, _vp, _vp, _vp, _u64, _c.c_double if s == "f64" else _c.c_float, _c.POINTER(_u64)]
        if isinstance(P, np.ndarray):
            Pd = np.ascontiguousarray(P, A.dtype)
            f(_c.byref(e), _ptr(Pd), None, _ptr(b), _ptr(x), max_iters, eps, _c.byref(used))
        else:
            pe = _ell(P)
            f(_c.byref(e), None, _c.byref(pe), _ptr(b), _ptr(x), max_iters, eps, _c.byref(used))
        return x, used.value

    def _mg_struct(self, H, max_iters, max_iters_coarse, n_pre, n_post):
        L = len(H.A)
        A = (_OraEll * L)(*[_ell(a) for a in H.A])
        P = (_OraEll * max(L - 1, 1))(*[_ell(a) for a in H.prol])
        R = (_OraEll * max(L - 1, 1))(*[_ell(a) for a in H.res])
        mg = _OraMG(L, A, P, R, max_iters, max_iters_coarse, n_pre, n_post)
        mg._keep = (A, P, R, H)
        return mg

    def mg(self, H, b, x0=None, damping=0.7, eps=1e-8, max_iters=100, max_iters_coarse=1000,
           n_pre=2, n_post=2, history=False):
        """V(n_pre, n_post) MG, Jacobi smoother, PROLMAT transfers, CG coarse solve."""
        dt = H.A[-1].dtype
        s = self._suffix(dt)
        b = np.ascontiguousarray(b, dt)
        x = np.zeros(H.A[-1].rows, dt) if x0 is None else np.array(x0, dt)
        mg = self._mg_struct(H, max_iters, max_iters_coarse, n_pre, n_post)
        used = _u64(0)
        hist = np.zeros(max_iters + 1, dt)
        getattr(self.lib, f"ora_mg_{s}")(_c.byref(mg), damping, _ptr(b), _ptr(x), eps,
                                         _c.byref(used), _ptr(hist))
        if history:
            return x, used.value, hist[: used.value + 1]
        return x, used.value

    def ir_mg(self, A64, H32, b, x0=None, damping=0.7, eps=1e-10, inner_eps=1e-3, max_iters=100,
              inner_max_iters=100, max_iters_coarse=1000, n_pre=2, n_post=2, warm_start=True):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A64.rows) if x0 is None else np.array(x0, np.float64)
        mg = self._mg_struct(H32, inner_max_iters, max_iters_coarse, n_pre, n_post)
        used = _u64(0)
        hist = np.zeros(max_iters + 1)
        e = _ell(A64)
        self.lib.ora_ir_mg(_c.byref(e), _c.byref(mg), damping, _ptr(b), _ptr(x), eps, inner_eps,
                           max_iters, int(warm_start), _c.byref(used), _ptr(hist))
        return x, used.value, hist[: used.value + 1]

    def ir_pcg(self, A64, H32, b, x0=None, eps=1e-8, inner_eps=1e-3, max_outer=50, max_inner=1000,
               damping=0.7):
        """IR + FP32 MG-preconditioned CG (V(2,2), coarse CG 200 iterations, eps 1e-6)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A64.rows) if x0 is None else np.array(x0, np.float64)
        mg = self._mg_struct(H32, 1, 200, 2, 2)
        outer, inner = _u64(0), _u64(0)
        hist = np.zeros(max_outer + 2)
        e = _ell(A64)
        self.lib.ora_ir_pcg(_c.byref(e), _c.byref(mg), damping, _ptr(b), _ptr(x), eps, inner_eps, max_outer,
                            max_inner, _c.byref(outer), _c.byref(inner), _ptr(hist))
        return x, outer.value, inner.value, hist[: outer.value + 1]

    def ir_cg(self, A64, A32, b, x0=None, eps=1e-10, inner_eps=1e-3, inner_max_iters=100000,
              max_iters=100):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(A64.rows) if x0 is None else np.array(x0, np.float64)
        used, inner = _u64(0), _u64(0)
        hist = np.zeros(max_iters + 1)
        e64, e32 = _ell(A64), _ell(A32)
        self.lib.ora_ir_cg(_c.byref(e64), _c.byref(e32), _ptr(b), _ptr(x), eps, inner_eps,
                           inner_max_iters, max_iters, _c.byref(used), _c.byref(inner), _ptr(hist))
        return x, used.value, inner.value, hist[: used.value + 1]


    def spai2(self, A, col_start=0, col_end=0, Mx=None):
        """SPAI2<tags::CPU::SSE> restated (ora_spai2.inc): M's values in A's ELL layout.  Columns
        outside [col_start, col_end) keep Mx's values (A's when Mx is None); col_end 0 = all."""
        s = self._suffix(A.dtype)
        Mx = np.array(A.Ax if Mx is None else Mx, A.dtype)
        f = getattr(self.lib, f"ora_spai2_{s}")
        f.argtypes = [_vp, _vp, _u64, _u64]
        e = _ell(A)
        if f(_c.byref(e), _ptr(Mx), col_start, col_end) != 0:
            raise RuntimeError("oracle SPAI2: matrix not square or out of memory")
        return Mx


class RefEllHandle:
    """The reference's SparseMatrixELL<double> and input vector, built once (ref_ell_create_f64);
    ``spmv(tag, reps)`` runs Product<tag> reps times and returns the per-product seconds."""

    def __init__(self, R, A, x):
        self.R = R
        L = R.lib
        ul = _c.c_ulong
        L.ref_ell_create_f64.argtypes = [ul] * 5 + [_vp, _vp, _vp, _c.POINTER(_vp)]
        L.ref_ell_spmv_f64.argtypes = [_c.c_int, _vp, _c.c_int, _vp, _vp]
        L.ref_ell_destroy.argtypes = [_vp]
        self.rows = A.rows
        h = _vp()
        x = np.ascontiguousarray(x, np.float64)
        R._check(L.ref_ell_create_f64(A.rows, A.cols, A.stride, A.ncpr, A.threads, _ptr(A.Aj), _ptr(A.Ax),
                                      _ptr(x), _c.byref(h)))
        self.h = h

    def spmv(self, tag="mc-sse", reps=1, want_y=False):
        sec = np.zeros(max(reps, 1))
        y = np.zeros(self.rows) if want_y else None
        self.R._check(self.R.lib.ref_ell_spmv_f64(TAGS[tag], self.h, reps, _ptr(sec),
                                                  _ptr(y) if want_y else None))
        return (sec[:reps], y) if want_y else sec[:reps]

    def close(self):
        if self.h:
            self.R.lib.ref_ell_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Reference:
    """The reference's own CPU path (unmodified HONEI sources + ref_shim.cc)."""

    def __init__(self, path: str = REF_SO):
        self.lib = _c.CDLL(path)
        # The reference's MultiCore thread pool pins the calling thread to one core when it
        # starts (honei/backends/multicore/thread_pool.cc:395-399, mc::affinity defaults to
        # true); every thread this process creates afterwards would inherit that mask.
        # _check() puts the caller's mask back after each call.
        self._mask = os.sched_getaffinity(0) if hasattr(os, "sched_getaffinity") else None
        L = self.lib
        L.ref_last_error.restype = _c.c_char_p
        ul = _c.c_ulong
        ell_args = [ul] * 5 + [_vp, _vp]
        L.ref_spmv_f64.argtypes = [_c.c_int] + ell_args + [_vp, _vp, _c.c_int, _c.POINTER(_c.c_double)]
        L.ref_spmv_f32.argtypes = L.ref_spmv_f64.argtypes
        L.ref_defect_f64.argtypes = [_c.c_int] + ell_args + [_vp, _vp, _vp]
        L.ref_defect_f32.argtypes = L.ref_defect_f64.argtypes
        L.ref_dot_f64.argtypes = [_c.c_int, ul, _vp, _vp, _vp]
        L.ref_dot_f32.argtypes = L.ref_dot_f64.argtypes
        L.ref_cg_f64.argtypes = [_c.c_int] + ell_args + [_vp, _vp, ul, _c.c_double,
                                                         _c.POINTER(ul), _c.POINTER(_c.c_double)]
        L.ref_cg_f32.argtypes = [_c.c_int] + ell_args + [_vp, _vp, ul, _c.c_float,
                                                         _c.POINTER(ul), _c.POINTER(_c.c_double)]
        L.ref_q1_poisson_f64.argtypes = [ul, _vp, _vp, _vp, _vp]
        L.ref_read_ell_f64.argtypes = [_c.c_char_p, _vp, _vp, _vp, _vp]
        L.ref_read_exp_f64.argtypes = [_c.c_char_p, _c.POINTER(ul), _vp]
        L.ref_set_threads.argtypes = [_c.c_int]
        mg_args = [_c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ref_mg_f64.argtypes = mg_args + [_c.c_double, ul, ul, ul, ul, _c.c_double,
                                           _c.POINTER(ul), _c.POINTER(_c.c_double), _vp, _vp, _vp]
        L.ref_mg_f32.argtypes = mg_args + [_c.c_float, ul, ul, ul, ul, _c.c_float,
                                           _c.POINTER(ul), _c.POINTER(_c.c_double), _vp, _vp, _vp]
        L.ref_q1band_spmv_f64.argtypes = [_c.c_int, ul, _vp, _vp, _vp, _c.c_int, _c.POINTER(_c.c_double)]
        L.ref_q1band_spmv_f32.argtypes = L.ref_q1band_spmv_f64.argtypes
        L.ref_q1band_defect_f64.argtypes = [ul, _vp, _vp, _vp, _vp]
        L.ref_q1band_poisson_f64.argtypes = [ul, _vp]
        L.ref_q1band_from_ell_f64.argtypes = [_vp, _vp, _vp, _vp]
        L.ref_ir_mg.argtypes = [_c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                _c.c_float, ul, ul, ul, ul, _c.c_float, _c.c_double, ul,
                                _c.POINTER(ul), _c.POINTER(_c.c_double), _vp, _vp, _vp]

    def ell_handle(self, A, x):
        """A SparseMatrixELL<double> built once from A with the input vector x, for timing
        products alone: returns a RefEllHandle."""
        return RefEllHandle(self, A, x)

    def _check(self, rc):
        if self._mask is not None:
            os.sched_setaffinity(0, self._mask)
        if rc != 0:
            raise RuntimeError("reference: " + self.lib.ref_last_error().decode())

    def set_threads(self, n: int):
        self._check(self.lib.ref_set_threads(n))

    @staticmethod
    def _args(A):
        return [A.rows, A.cols, A.stride, A.ncpr, A.threads, _ptr(A.Aj), _ptr(A.Ax)]

    def q1_poisson(self, M):
        from honei_b200.problems import EllMatrix
        info = (_c.c_ulong * 6)()
        self._check(self.lib.ref_q1_poisson_f64(M, info, None, None, None))
        rows, cols, stride, ncpr, T, nnz = list(info)
        Aj = np.zeros(ncpr * stride, np.uint64)
        Ax = np.zeros(ncpr * stride)
        Arl = np.zeros(rows, np.uint64)
        self._check(self.lib.ref_q1_poisson_f64(M, info, _ptr(Aj), _ptr(Ax), _ptr(Arl)))
        return EllMatrix(rows, cols, stride, ncpr, T, Aj, Ax, Arl, nnz)

    def cg_var(self, A, P, b, x0=None, max_iters=10000, eps=1e-8, tag="cpu"):
        """CGSolver<tag, methods::VAR>: P a vector or an EllMatrix.  (x, used_iters, seconds)."""
        s = "f64" if A.dtype == np.float64 else "f32"
        b = np.ascontiguousarray(b, A.dtype)
        x = np.zeros(A.rows, A.dtype) if x0 is None else np.array(x0, A.dtype)
        ainfo = np.array([A.rows, A.cols, A.stride, A.ncpr, A.threads], np.uint64)
        used, sec = _c.c_ulong(0), _c.c_double(0)
        f = getattr(self.lib, f"ref_cg_var_{s}")
        f.argtypes = [_c.c_int] + [_vp] * 9 + [_c.c_ulong, _c.c_double if s == "f64" else _c.c_float,
                                               _c.POINTER(_c.c_ulong), _c.POINTER(_c.c_double)]
        if isinstance(P, np.ndarray):
            Pd = np.ascontiguousarray(P, A.dtype)
            rc = f(TAGS[tag], _ptr(ainfo), _ptr(A.Aj), _ptr(A.Ax), _ptr(Pd), None, None, None, _ptr(b), _ptr(x),
                   max_iters, eps, _c.byref(used), _c.byref(sec))
        else:
            pinfo = np.array([P.rows, P.cols, P.stride, P.ncpr, P.threads], np.uint64)
            rc = f(TAGS[tag], _ptr(ainfo), _ptr(A.Aj), _ptr(A.Ax), None, _ptr(pinfo), _ptr(P.Aj), _ptr(P.Ax),
                   _ptr(b), _ptr(x), max_iters, eps, _c.byref(used), _c.byref(sec))
        self._check(rc)
        return x, used.value, sec.value

    def spai2(self, A, tag="sse"):
        """SPAI2<tag>::value(M, A) with M = A.copy() (tag "sse" or "mc-sse"): M's values in A's
        ELL layout (0 in empty slots), and the seconds the call took."""
        s = "f64" if A.dtype == np.float64 else "f32"
        ainfo = np.array([A.rows, A.cols, A.stride, A.ncpr, A.threads], np.uint64)
        Mx = np.zeros_like(A.Ax)
        sec = _c.c_double(0)
        f = getattr(self.lib, f"ref_spai2_{s}")
        f.argtypes = [_c.c_int, _vp, _vp, _vp, _vp, _c.POINTER(_c.c_double)]
        self._check(f(TAGS[tag], _ptr(ainfo), _ptr(A.Aj), _ptr(A.Ax), _ptr(Mx), _c.byref(sec)))
        return Mx, sec.value

    def q1band_spmv(self, bands, x, tag="cpu", reps=0):
        """Product<tag> on BandedMatrixQx<Q1Type>: (y, median seconds of `reps` timed calls);
        tags "cpu", "sse", "mc-sse"."""
        dt = np.asarray(bands[0]).dtype
        bands = [np.ascontiguousarray(b, dt) for b in bands]
        bp = (_vp * 9)(*[b.ctypes.data for b in bands])
        x = np.ascontiguousarray(x, dt)
        y = np.zeros(len(x), dt)
        sec = _c.c_double(0)
        s = "f64" if dt == np.float64 else "f32"
        self._check(getattr(self.lib, f"ref_q1band_spmv_{s}")(TAGS[tag], len(x), bp, _ptr(x), _ptr(y), reps,
                                                               _c.byref(sec)))
        return y, sec.value

    def q1band_defect(self, bands, b, x):
        bands = [np.ascontiguousarray(v, np.float64) for v in bands]
        bp = (_vp * 9)(*[v.ctypes.data for v in bands])
        b = np.ascontiguousarray(b, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        r = np.zeros(len(x))
        self._check(self.lib.ref_q1band_defect_f64(len(x), bp, _ptr(b), _ptr(x), _ptr(r)))
        return r

    def q1band_poisson(self, M):
        out = [np.zeros(M * M) for _ in range(9)]
        bp = (_vp * 9)(*[b.ctypes.data for b in out])
        self._check(self.lib.ref_q1band_poisson_f64(M, bp))
        return out

    def q1band_from_ell(self, A):
        """BandedMatrixQx(SparseMatrixELL &) of an FP64 reference-layout matrix: 9 bands."""
        info = np.array([A.rows, A.cols, A.stride, A.ncpr, A.threads], np.uint64)
        out = [np.zeros(A.rows) for _ in range(9)]
        bp = (_vp * 9)(*[b.ctypes.data for b in out])
        self._check(self.lib.ref_q1band_from_ell_f64(_ptr(info), _ptr(A.Aj), _ptr(A.Ax), bp))
        return out

    def read_ell(self, path):
        from honei_b200.problems import EllMatrix
        info = (_c.c_ulong * 6)()
        p = path.encode()
        self._check(self.lib.ref_read_ell_f64(p, info, None, None, None))
        rows, cols, stride, ncpr, T, nnz = list(info)
        Aj = np.zeros(ncpr * stride, np.uint64)
        Ax = np.zeros(ncpr * stride)
        Arl = np.zeros(rows, np.uint64)
        self._check(self.lib.ref_read_ell_f64(p, info, _ptr(Aj), _ptr(Ax), _ptr(Arl)))
        return EllMatrix(rows, cols, stride, ncpr, T, Aj, Ax, Arl, nnz)

    def prolongate(self, coarse, mask, n_fine):
        coarse = np.ascontiguousarray(coarse)
        s = "f64" if coarse.dtype == np.float64 else "f32"
        fine = np.zeros(n_fine, coarse.dtype)
        m = np.ascontiguousarray(mask, np.uint64)
        f = getattr(self.lib, f"ref_prolongate_{s}")
        f.argtypes = [_c.c_ulong, _vp, _vp, _c.c_ulong, _vp]
        self._check(f(n_fine, _ptr(fine), _ptr(coarse), len(coarse), _ptr(m)))
        return fine

    def restrict(self, fine, mask):
        fine = np.ascontiguousarray(fine)
        s = "f64" if fine.dtype == np.float64 else "f32"
        side = int(round(np.sqrt(len(fine))))
        nc = ((side - 1) // 2 + 1) ** 2
        coarse = np.zeros(nc, fine.dtype)
        m = np.ascontiguousarray(mask, np.uint64)
        f = getattr(self.lib, f"ref_restrict_{s}")
        f.argtypes = [_c.c_ulong, _vp, _vp, _c.c_ulong, _vp]
        self._check(f(len(fine), _ptr(coarse), _ptr(fine), nc, _ptr(m)))
        return coarse

    def read_mtx(self, path):
        """MatrixIO<io_formats::MTX>::read_matrix -> SparseMatrixELL (the mtxtoell client)."""
        from honei_b200.problems import EllMatrix
        f = self.lib.ref_read_mtx_f64
        f.argtypes = [_c.c_char_p, _vp, _vp, _vp, _vp]
        info = (_c.c_ulong * 6)()
        p = path.encode()
        self._check(f(p, info, None, None, None))
        rows, cols, stride, ncpr, T, nnz = list(info)
        Aj = np.zeros(ncpr * stride, np.uint64)
        Ax = np.zeros(ncpr * stride)
        Arl = np.zeros(rows, np.uint64)
        self._check(f(p, info, _ptr(Aj), _ptr(Ax), _ptr(Arl)))
        return EllMatrix(rows, cols, stride, ncpr, T, Aj, Ax, Arl, nnz)

    def read_exp(self, path):
        n = _c.c_ulong(0)
        self._check(self.lib.ref_read_exp_f64(path.encode(), _c.byref(n), None))
        out = np.zeros(n.value)
        self._check(self.lib.ref_read_exp_f64(path.encode(), _c.byref(n), _ptr(out)))
        return out

    def spmv(self, A, x, tag="cpu", reps=0):
        """Returns (y, median seconds of `reps` timed calls after one warm-up)."""
        s = "f64" if A.dtype == np.float64 else "f32"
        x = np.ascontiguousarray(x, A.dtype)
        y = np.zeros(A.rows, A.dtype)
        sec = _c.c_double(0)
        self._check(getattr(self.lib, f"ref_spmv_{s}")(TAGS[tag], *self._args(A), _ptr(x), _ptr(y),
                                                        reps, _c.byref(sec)))
        return y, sec.value

    def csr_product_test(self, size, blocksize):
        """The reference's CSR product test case (product_TEST.cc:936-948) converted with
        csr::blocksize: (CsrMatrix, x, y = Product<tags::CPU>(A, x))."""
        from honei_b200.problems import CsrMatrix
        f = self.lib.ref_csr_product_test_f64
        f.argtypes = [_c.c_ulong, _c.c_ulong, _vp, _vp, _vp, _vp, _vp, _vp]
        info = (_c.c_ulong * 5)()
        self._check(f(size, blocksize, info, None, None, None, None, None))
        rows, cols, bs, nb, used = list(info)
        Ar = np.zeros(rows + 1, np.uint64)
        Aj = np.zeros(max(nb, 1), np.uint64)
        Ax = np.zeros(max(nb * bs, 1))
        x = np.zeros(cols)
        y = np.zeros(rows)
        self._check(f(size, blocksize, info, _ptr(Ar), _ptr(Aj), _ptr(Ax), _ptr(x), _ptr(y)))
        return CsrMatrix(rows, cols, bs, Ar, Aj[:nb], Ax[:nb * bs], used), x, y

    def csr_from_ell(self, A, blocksize):
        """SparseMatrixCSR(SparseMatrixELL) with csr::blocksize (FP64)."""
        from honei_b200.problems import CsrMatrix
        f = self.lib.ref_csr_from_ell_f64
        f.argtypes = [_c.c_ulong] * 5 + [_vp, _vp, _c.c_ulong, _vp, _vp, _vp, _vp]
        info = (_c.c_ulong * 5)()
        args = self._args(A)
        self._check(f(*args, blocksize, info, None, None, None))
        rows, cols, bs, nb, used = list(info)
        Ar = np.zeros(rows + 1, np.uint64)
        Aj = np.zeros(max(nb, 1), np.uint64)
        Ax = np.zeros(max(nb * bs, 1))
        self._check(f(*args, blocksize, info, _ptr(Ar), _ptr(Aj), _ptr(Ax)))
        return CsrMatrix(rows, cols, bs, Ar, Aj[:nb], Ax[:nb * bs], used)

    def _csr_args(self, A, s):
        Aj = np.ascontiguousarray(A.Aj if len(A.Aj) else np.zeros(1, np.uint64), np.uint64)
        Ax = np.ascontiguousarray(A.Ax if len(A.Ax) else np.zeros(1, A.dtype), A.dtype)
        self._keep_csr = (Aj, Ax)
        return [A.rows, A.cols, A.blocksize, A.used, _ptr(np.ascontiguousarray(A.Ar, np.uint64)), _ptr(Aj), _ptr(Ax)]

    def csr_spmv(self, A, x, tag="cpu", reps=0):
        """Product<tag>(DV, SparseMatrixCSR, DV): (y, median seconds of reps timed calls)."""
        s = "f64" if A.dtype == np.float64 else "f32"
        f = getattr(self.lib, f"ref_csr_spmv_{s}")
        f.argtypes = [_c.c_int] + [_c.c_ulong] * 4 + [_vp] * 5 + [_c.c_int, _c.POINTER(_c.c_double)]
        x = np.ascontiguousarray(x, A.dtype)
        y = np.zeros(A.rows, A.dtype)
        Ar = np.ascontiguousarray(A.Ar, np.uint64)
        args = self._csr_args(A, s)
        args[4] = _ptr(Ar)
        sec = _c.c_double(0)
        self._check(f(TAGS[tag], *args, _ptr(x), _ptr(y), reps, _c.byref(sec)))
        return y, sec.value

    def csr_defect(self, A, b, x, tag="cpu"):
        s = "f64" if A.dtype == np.float64 else "f32"
        f = getattr(self.lib, f"ref_csr_defect_{s}")
        f.argtypes = [_c.c_int] + [_c.c_ulong] * 4 + [_vp] * 6
        b = np.ascontiguousarray(b, A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        r = np.zeros(A.rows, A.dtype)
        Ar = np.ascontiguousarray(A.Ar, np.uint64)
        args = self._csr_args(A, s)
        args[4] = _ptr(Ar)
        self._check(f(TAGS[tag], *args, _ptr(b), _ptr(x), _ptr(r)))
        return r

    def defect(self, A, b, x, tag="cpu"):
        s = "f64" if A.dtype == np.float64 else "f32"
        b = np.ascontiguousarray(b, A.dtype)
        x = np.ascontiguousarray(x, A.dtype)
        r = np.zeros(A.rows, A.dtype)
        self._check(getattr(self.lib, f"ref_defect_{s}")(TAGS[tag], *self._args(A), _ptr(b), _ptr(x), _ptr(r)))
        return r

    def dot(self, x, y, tag="cpu"):
        x = np.ascontiguousarray(x)
        y = np.ascontiguousarray(y, x.dtype)
        out = np.zeros(1, x.dtype)
        f = self.lib.ref_dot_f64 if x.dtype == np.float64 else self.lib.ref_dot_f32
        self._check(f(TAGS[tag], len(x), _ptr(x), _ptr(y), _ptr(out)))
        return out[0]

    def cg(self, A, b, x0=None, max_iters=10000, eps=1e-8, tag="cpu"):
        """Returns (x, used_iters, seconds)."""
        s = "f64" if A.dtype == np.float64 else "f32"
        b = np.ascontiguousarray(b, A.dtype)
        x = np.zeros(A.rows, A.dtype) if x0 is None else np.array(x0, A.dtype)
        used = _c.c_ulong(0)
        sec = _c.c_double(0)
        self._check(getattr(self.lib, f"ref_cg_{s}")(TAGS[tag], *self._args(A), _ptr(b), _ptr(x),
                                                      max_iters, eps, _c.byref(used), _c.byref(sec)))
        return x, used.value, sec.value

    @staticmethod
    def _res_arrays(H):
        """The restriction matrices H.res (Res_l = Prol_l^T, the entries of each row in
        ascending column order, as the reference's Transposition gives them)."""
        n = max(len(H.res), 1)
        rinfo = np.array([r.info() for r in H.res] or [[0] * 5], np.uint64).ravel()
        Rj = (_vp * n)(*[r.Aj.ctypes.data for r in H.res])
        Rx = (_vp * n)(*[r.Ax.ctypes.data for r in H.res])
        return rinfo, Rj, Rx

    def _mg_arrays(self, H):
        L = len(H.A)
        ainfo = np.array([a.info() for a in H.A], np.uint64).ravel()
        pinfo = np.array([p.info() for p in H.prol] or [[0] * 5], np.uint64).ravel()
        Aj = (_vp * L)(*[a.Aj.ctypes.data for a in H.A])
        Ax = (_vp * L)(*[a.Ax.ctypes.data for a in H.A])
        Pj = (_vp * max(L - 1, 1))(*[p.Aj.ctypes.data for p in H.prol])
        Px = (_vp * max(L - 1, 1))(*[p.Ax.ctypes.data for p in H.prol])
        return L, ainfo, pinfo, Aj, Ax, Pj, Px

    def mg(self, H, b, x0=None, damping=0.7, eps=1e-8, max_iters=100, max_iters_coarse=1000,
           n_pre=2, n_post=2, tag="cpu"):
        dt = H.A[-1].dtype
        s = "f64" if dt == np.float64 else "f32"
        L, ainfo, pinfo, Aj, Ax, Pj, Px = self._mg_arrays(H)
        b = np.ascontiguousarray(b, dt)
        x = np.zeros(H.A[-1].rows, dt) if x0 is None else np.array(x0, dt)
        used = _c.c_ulong(0)
        sec = _c.c_double(0)
        rinfo, Rj, Rx = self._res_arrays(H)
        self._check(getattr(self.lib, f"ref_mg_{s}")(TAGS[tag], L, _ptr(ainfo), Aj, Ax, _ptr(pinfo), Pj, Px,
                                                      _ptr(b), _ptr(x), damping, max_iters, max_iters_coarse,
                                                      n_pre, n_post, eps, _c.byref(used), _c.byref(sec),
                                                      _ptr(rinfo) if len(H.res) else None, Rj, Rx))
        return x, used.value, sec.value

    def ir_mg(self, H64, H32, b, x0=None, damping=0.7, eps=1e-10, inner_eps=1e-3, max_iters=100,
              inner_max_iters=100, max_iters_coarse=1000, n_pre=2, n_post=2, tag="cpu"):
        L, ainfo, pinfo, Aj, Ax64, Pj, _ = self._mg_arrays(H64)
        Ax32 = (_vp * L)(*[a.Ax.ctypes.data for a in H32.A])
        Px32 = (_vp * max(L - 1, 1))(*[p.Ax.ctypes.data for p in H32.prol])
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(H64.A[-1].rows) if x0 is None else np.array(x0, np.float64)
        used = _c.c_ulong(0)
        sec = _c.c_double(0)
        rinfo, Rj, _ = self._res_arrays(H64)
        Rx32 = (_vp * max(len(H32.res), 1))(*[r.Ax.ctypes.data for r in H32.res])
        self._check(self.lib.ref_ir_mg(TAGS[tag], L, _ptr(ainfo), Aj, Ax64, Ax32, _ptr(pinfo), Pj, Px32, _ptr(b),
                                       _ptr(x), damping, inner_max_iters, max_iters_coarse, n_pre, n_post,
                                       inner_eps, eps, max_iters, _c.byref(used), _c.byref(sec),
                                       _ptr(rinfo) if len(H64.res) else None, Rj, Rx32))
        return x, used.value, sec.value
