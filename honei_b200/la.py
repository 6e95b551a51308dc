"""Host-side mirror of HONEI's tag-dispatched operator API for the B200 backend.

The C++ plugin (honei_b200/plugin) is the drop-in for HONEI itself; this module offers the
same operators to Python callers, with the reference's names, argument order and error
behaviour (size mismatches raise ``VectorSizeDoesNotMatch`` before anything is launched, as
honei/la/product.hh:154-161 does).  Dense vectors are CUDA ``torch.Tensor`` objects (float64
or float32, contiguous): torch provides device memory and streams only; every operation runs
in libhonei_b200.so.

    A = SparseMatrixELL.from_reference(ell)        # problems.EllMatrix, reference layout
    Product.value(y, A, x)                           # Product<tags::GPU::CUDA>::value
    r = Defect.value(r, b, A, x)
    d = DotProduct.value(x, y); n = Norm.value(x, root=True)
    used = CGSolver.value(A, None, b, x, max_iters=10000, eps_relative=1e-8)
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import torch

from . import _lib
from ._lib import HbCsr, HbEll, check, lib

HB_ERR_UNSUPPORTED = 6                 # hb_status: shape outside what a kernel supports


class VectorSizeDoesNotMatch(ValueError):
    """honei/la/vector_error.hh: VectorSizeDoesNotMatch(size, expected)."""

    def __init__(self, size, expected):
        super().__init__(f"Vector size does not match: {size} != {expected}")


class MatrixRowsDoNotMatch(ValueError):
    """honei/la/matrix_error.hh: MatrixRowsDoNotMatch(rows, expected)."""

    def __init__(self, rows, expected):
        super().__init__(f"Matrix rows do not match: {rows} != {expected}")


_DT = {torch.float64: 0, torch.float32: 1}
_SUF = {torch.float64: "f64", torch.float32: "f32"}


class Context:
    """An hb_context bound to one device and (by default) torch's current stream."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        check(lib().hb_create(C.byref(h), device), "hb_create")
        self.handle = h
        self.bind_stream()

    def bind_stream(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        check(lib().hb_set_stream(self.handle, C.c_void_p(s.cuda_stream)), "hb_set_stream", self.handle)

    def launches(self) -> int:
        return int(lib().hb_launch_count(self.handle))

    def reserve(self, n: int) -> None:
        check(lib().hb_reserve(self.handle, n), "hb_reserve", self.handle)

    def synchronize(self):
        check(lib().hb_synchronize(self.handle), "hb_synchronize", self.handle)

    def close(self):
        if self.handle:
            lib().hb_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_ctx_lock = threading.Lock()
_ctx_by_dev: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    dev = torch.cuda.current_device() if device is None else device
    with _ctx_lock:
        c = _ctx_by_dev.get(dev)
        if c is None:
            c = _ctx_by_dev[dev] = Context(dev)
        c.bind_stream()
        return c


def _vec(t: torch.Tensor, dtype, name: str) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t.data_ptr()


BLOCK_FAMILIES = {"ell": 0, "q1band": 1, "vector": 2}


def set_block_size(family: str, threads: int, ctx: Context | None = None) -> int:
    """Threads per block of a kernel family on ctx (hb_set_block_size): "ell" (ELL product,
    defect, Jacobi sweep; 32..256), "q1band" (banded Q1 kernels; 32..256) or "vector"
    (elementwise kernels; 32..1024), a multiple of 32, or 0 for the default.  The knob HONEI's
    honeirc block-size keys set; results do not depend on it.  Returns the previous value."""
    ctx = ctx or default_context()
    prev = lib().hb_set_block_size(ctx.handle, BLOCK_FAMILIES[family], int(threads))
    if prev < 0:
        raise ValueError(f"block size {threads} is not valid for {family}")
    return prev


class _DeviceArray:
    """__cuda_array_interface__ view of device memory owned elsewhere (zero copy)."""

    _TYPESTR = {torch.float64: "<f8", torch.float32: "<f4", torch.int32: "<i4"}

    def __init__(self, ptr, n, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": self._TYPESTR[dtype],
                                         "data": (int(ptr), False), "version": 2, "strides": None}


def _wrap_device(ptr, n, dtype):
    """A torch view of n elements of device memory owned elsewhere (the owner keeps it alive)."""
    if n == 0 or not ptr:
        return torch.empty(0, dtype=dtype, device="cuda")
    return torch.as_tensor(_DeviceArray(ptr, n, dtype), device="cuda")


class SparseMatrixELL:
    """Device mirror of a HONEI SparseMatrixELL (honei/la/sparse_matrix_ell.hh:44-129)."""

    def __init__(self, rows, cols, K, ld, Aj: torch.Tensor, Ax: torch.Tensor):
        self._rows, self._cols, self.K, self.ld = int(rows), int(cols), int(K), int(ld)
        self.Aj, self.Ax = Aj, Ax
        self.dtype = Ax.dtype
        self._s = HbEll(self._rows, self._cols, self.K, self.ld, Aj.data_ptr(), Ax.data_ptr(),
                        _DT[Ax.dtype], 0)

    def rows(self) -> int:
        return self._rows

    def columns(self) -> int:
        return self._cols

    @property
    def struct(self) -> HbEll:
        return self._s

    @staticmethod
    def layout(rows, ncpr, threads=1):
        K, ld = C.c_int64(), C.c_int64()
        check(lib().hb_ell_layout(rows, ncpr, threads, C.byref(K), C.byref(ld)), "hb_ell_layout")
        return K.value, ld.value

    @classmethod
    def from_reference(cls, ell, ctx: Context | None = None, device="cuda") -> "SparseMatrixELL":
        """Uploads the reference-layout arrays (u64 Aj, Ax, u64 Arl) and imports them."""
        ctx = ctx or default_context()
        dt = torch.float64 if ell.Ax.dtype == np.float64 else torch.float32
        K, ld = cls.layout(ell.rows, ell.ncpr, ell.threads)
        Aj_ref = torch.from_numpy(ell.Aj.view(np.int64)).to(device)
        Ax_ref = torch.from_numpy(ell.Ax).to(device)
        Arl = torch.from_numpy(ell.Arl.view(np.int64)).to(device)
        Aj = torch.empty(K * ld, dtype=torch.int32, device=device)
        Ax = torch.empty(K * ld, dtype=dt, device=device)
        out = HbEll(ell.rows, ell.cols, K, ld, Aj.data_ptr(), Ax.data_ptr(), _DT[dt], 0)
        fn = lib().hb_ell_import_f64 if dt == torch.float64 else lib().hb_ell_import_f32
        check(fn(ctx.handle, ell.rows, ell.cols, ell.stride, ell.ncpr, ell.threads, Aj_ref.data_ptr(),
                 Ax_ref.data_ptr(), Arl.data_ptr(), C.byref(out)), "hb_ell_import", ctx.handle)
        return cls(ell.rows, ell.cols, K, ld, Aj, Ax)

    def validate(self, ctx: Context | None = None) -> int:
        """Number of slots whose column is neither padding (-1) nor inside [0, cols)
        (hb_ell_validate); 0 for every matrix the import and the assemblers build."""
        ctx = ctx or default_context()
        n = C.c_int64(0)
        check(lib().hb_ell_validate(ctx.handle, C.byref(self.struct), C.byref(n)), "hb_ell_validate", ctx.handle)
        return n.value

    @classmethod
    def q1_poisson(cls, M: int, coef: torch.Tensor | None = None, ctx: Context | None = None,
                   device="cuda", symmetric: bool = False) -> "SparseMatrixELL":
        """Q1 Poisson (Dirichlet rows identity) assembled on the device, FP64; symmetric=True
        drops the interior rows' boundary couplings (SPD form)."""
        ctx = ctx or default_context()
        N = M * M
        K, ld = cls.layout(N, 9, 1)
        Aj = torch.empty(K * ld, dtype=torch.int32, device=device)
        Ax = torch.empty(K * ld, dtype=torch.float64, device=device)
        out = HbEll(N, N, K, ld, Aj.data_ptr(), Ax.data_ptr(), 0, 0)
        cptr = None
        if coef is not None:
            cptr = _vec(coef, torch.float64, "coef")
            if coef.numel() != (M - 1) * (M - 1):
                raise VectorSizeDoesNotMatch(coef.numel(), (M - 1) * (M - 1))
        check(lib().hb_q1_assemble_f64(ctx.handle, M, cptr, int(symmetric), C.byref(out)), "hb_q1_assemble_f64",
              ctx.handle)
        return cls(N, N, K, ld, Aj, Ax)

    @classmethod
    def from_struct(cls, e: HbEll) -> "SparseMatrixELL":
        """Wraps device arrays described by an hb_ell (no copy; the owner keeps them alive)."""
        n = int(e.K * e.ld)
        dt = torch.float64 if e.dtype == 0 else torch.float32
        Aj = _wrap_device(e.Aj, n, torch.int32)
        Ax = _wrap_device(e.Ax, n, dt)
        return cls(e.rows, e.cols, e.K, e.ld, Aj, Ax)

    def to_host(self):
        """The matrix in the reference layout (problems.EllMatrix, one lane per row): the
        valid slots of every row in slot order."""
        from . import problems as P
        torch.cuda.synchronize()
        Aj = self.Aj.cpu().numpy().reshape(self.K, self.ld)[:, : self._rows]
        Ax = self.Ax.cpu().numpy().reshape(self.K, self.ld)[:, : self._rows]
        valid = Aj.T >= 0
        counts = valid.sum(axis=1)
        indptr = np.zeros(self._rows + 1, np.int64)
        np.cumsum(counts, out=indptr[1:])
        dtype = np.float64 if self.dtype == torch.float64 else np.float32
        return P.ell_from_csr(self._rows, self._cols, indptr, Aj.T[valid].astype(np.int64), Ax.T[valid], 1, dtype)

    @classmethod
    def read_file(cls, path: str, dtype=torch.float64, ctx: Context | None = None) -> "SparseMatrixELL":
        """MatrixIO<io_formats::ELL>::read_matrix straight to the device (hb_ell_read_file_*)."""
        ctx = ctx or default_context()
        info = (C.c_int64 * 5)()
        check(lib().hb_ell_file_info(str(path).encode(), info), f"hb_ell_file_info({path})")
        size, rows, cols, stride, ncpr = list(info)
        K, ld = cls.layout(rows, ncpr, 1)
        Aj = torch.empty(K * ld, dtype=torch.int32, device="cuda")
        Ax = torch.empty(K * ld, dtype=dtype, device="cuda")
        s = HbEll(rows, cols, K, ld, Aj.data_ptr(), Ax.data_ptr(), 0 if dtype == torch.float64 else 1, 0)
        fn = lib().hb_ell_read_file_f64 if dtype == torch.float64 else lib().hb_ell_read_file_f32
        check(fn(ctx.handle, str(path).encode(), C.byref(s)), f"hb_ell_read_file({path})", ctx.handle)
        return cls(rows, cols, K, ld, Aj, Ax)

    def write_file(self, path: str, ctx: Context | None = None) -> None:
        """MatrixIO<io_formats::ELL>::write_matrix of an FP64 matrix (hb_ell_write_file)."""
        ctx = ctx or default_context()
        check(lib().hb_ell_write_file(ctx.handle, C.byref(self._s), str(path).encode()), f"hb_ell_write_file({path})",
              ctx.handle)

    def to_float(self, ctx: Context | None = None) -> "SparseMatrixELL":
        """Same pattern with FP32 values (the reference fills FP32 matrices from FP64 values)."""
        ctx = ctx or default_context()
        Ax = torch.empty(self.K * self.ld, dtype=torch.float32, device=self.Ax.device)
        Aj = torch.empty_like(self.Aj)
        dst = HbEll(self._rows, self._cols, self.K, self.ld, Aj.data_ptr(), Ax.data_ptr(), 1, 0)
        check(lib().hb_ell_cast_f64_f32(ctx.handle, C.byref(self._s), C.byref(dst)), "hb_ell_cast", ctx.handle)
        return SparseMatrixELL(self._rows, self._cols, self.K, self.ld, Aj, Ax)

    def cm_order(self, ctx: Context | None = None):
        """(order, pos, info): the Cuthill-McKee locality order of the matrix graph
        (hb_ell_cm_order); order[k] = the row placed at position k, pos its inverse, info =
        (levels, rows reached, start row)."""
        ctx = ctx or default_context()
        n = self._rows
        order = torch.empty(max(n, 4), dtype=torch.int32, device=self.Aj.device)
        pos = torch.empty(max(n, 4), dtype=torch.int32, device=self.Aj.device)
        info = (C.c_int64 * 3)()
        check(lib().hb_ell_cm_order(ctx.handle, C.byref(self._s), order.data_ptr(), pos.data_ptr(), info),
              "hb_ell_cm_order", ctx.handle)
        return order[:n], pos[:n], tuple(info)

    def bandwidth(self, pos: torch.Tensor | None = None, ctx: Context | None = None) -> int:
        """max |pos[c] - pos[r]| over the stored entries (the matrix's own numbering by default)."""
        ctx = ctx or default_context()
        bw = C.c_int64(0)
        check(lib().hb_ell_bandwidth(ctx.handle, C.byref(self._s), None if pos is None else pos.data_ptr(),
                                     C.byref(bw)), "hb_ell_bandwidth", ctx.handle)
        return bw.value

    def ordered(self, columns: bool = True, packed: bool = True, ctx: Context | None = None) -> "OrderedMatrixELL":
        """A copy stored in the Cuthill-McKee locality order, for products with a badly numbered
        matrix (e.g. a randomly permuted grid).  Product.value on the copy gives y = A x bit for
        bit.  columns=True renumbers the columns too (local gathers; x is permuted into a work
        vector first): packed=True keeps each row's slots in their order with the columns as
        16-bit offsets from the row (hb_ell_pack_offsets; K <= 9 and a reordered bandwidth within
        +-32767), otherwise -- or where that does not fit -- the slots are sorted by new column
        with their summation ranks (hb_ell_permute_sorted).  columns=False keeps A's columns (no
        work vector; gathers stay scattered, rows that share columns run together)."""
        ctx = ctx or default_context()
        order, pos, info = self.cm_order(ctx)
        Aj = torch.empty_like(self.Aj)
        Ax = torch.empty_like(self.Ax)
        B = HbEll(self._rows, self._cols, self.K, self.ld, Aj.data_ptr(), Ax.data_ptr(), _DT[self.dtype], 0)
        if not columns:
            check(lib().hb_ell_permute(ctx.handle, C.byref(self._s), order.data_ptr(), None, C.byref(B)),
                  "hb_ell_permute", ctx.handle)
            return OrderedMatrixELL(SparseMatrixELL(self._rows, self._cols, self.K, self.ld, Aj, Ax), order, pos,
                                    False, info)
        if packed and self.K <= 9 and self._rows > 0:
            check(lib().hb_ell_permute(ctx.handle, C.byref(self._s), order.data_ptr(), pos.data_ptr(), C.byref(B)),
                  "hb_ell_permute", ctx.handle)
            O = OrderedMatrixELL(SparseMatrixELL(self._rows, self._cols, self.K, self.ld, Aj, Ax), order, pos,
                                 True, info)
            Bd = torch.empty((self.K, self.ld), dtype=torch.int16, device=self.Aj.device)
            st = lib().hb_ell_pack_offsets(ctx.handle, C.byref(O.B.struct), Bd.data_ptr())
            if st == 0:
                O.Bd = Bd
                return O
            if st != HB_ERR_UNSUPPORTED:
                check(st, "hb_ell_pack_offsets", ctx.handle)
        ranks = torch.empty(max(self._rows, 1), dtype=torch.int64, device=self.Aj.device)
        check(lib().hb_ell_permute_sorted(ctx.handle, C.byref(self._s), order.data_ptr(), pos.data_ptr(),
                                          C.byref(B), ranks.data_ptr()), "hb_ell_permute_sorted", ctx.handle)
        return OrderedMatrixELL(SparseMatrixELL(self._rows, self._cols, self.K, self.ld, Aj, Ax), order, pos,
                                True, info, ranks)


class OrderedMatrixELL:
    """A SparseMatrixELL stored in a locality order (SparseMatrixELL.ordered): B = the rows of
    A in `order`, with its columns renumbered through `pos` when `columns` (packed: Bd holds the
    columns as 16-bit offsets; ranked: the slots sorted by new column, ranks their summation
    order).  Products through it equal A's bit for bit."""

    def __init__(self, B: SparseMatrixELL, order: torch.Tensor, pos: torch.Tensor, columns: bool, info=None,
                 ranks: torch.Tensor | None = None):
        self.B, self.order, self.pos, self.columns_renumbered = B, order, pos, columns
        self.info = info
        self.ranks = ranks                              # the sorted, ranked form
        self.Bd = None                                  # the packed form: 16-bit column offsets
        self.dtype = B.dtype
        self._xw = None

    def rows(self) -> int:
        return self.B.rows()

    def columns(self) -> int:
        return self.B.columns()

    def product(self, y: torch.Tensor, x: torch.Tensor, ctx: Context):
        suf = _SUF[self.dtype]
        xp = _vec(x, self.dtype, "x")
        if self.columns_renumbered:
            if self._xw is None or self._xw.device != x.device:
                self._xw = torch.empty(self.B.ld, dtype=self.dtype, device=x.device)
            check(getattr(lib(), f"hb_gather_{suf}")(ctx.handle, self.B.rows(), self.order.data_ptr(), xp,
                                                     self._xw.data_ptr()), "hb_gather", ctx.handle)
            xp = self._xw.data_ptr()
            if self.Bd is not None:
                check(getattr(lib(), f"hb_spmv_packed_{suf}")(ctx.handle, C.byref(self.B.struct), self.Bd.data_ptr(),
                                                              self.order.data_ptr(), xp, _vec(y, self.dtype, "y")),
                      "Product", ctx.handle)
            else:
                check(getattr(lib(), f"hb_spmv_ranked_{suf}")(ctx.handle, C.byref(self.B.struct),
                                                              self.order.data_ptr(), self.ranks.data_ptr(), xp,
                                                              _vec(y, self.dtype, "y")), "Product", ctx.handle)
            return y
        check(getattr(lib(), f"hb_spmv_rows_{suf}")(ctx.handle, C.byref(self.B.struct), self.order.data_ptr(), xp,
                                                    _vec(y, self.dtype, "y")), "Product", ctx.handle)
        return y


class BandedMatrixQ1:
    """BandedMatrixQx<Q1Type, DT> (honei/la/banded_matrix_qx.hh): nine bands of n values in the
    order LL, LD, LU, DL, DD, DU, UL, UD, UU, on the device.  ``bands`` is a (9, ldb) tensor,
    ldb = n rounded up to 4 so that every band starts 16-byte aligned.

        A = BandedMatrixQ1.poisson(M)                   # FillMatrix<POISSON, DIRICHLET_0>
        A = BandedMatrixQ1.from_ell(E)                  # BandedMatrixQx(SparseMatrixELL &)
        A = BandedMatrixQ1.from_bands([ll, ld, ...])    # nine host or device arrays
    """

    LL, LD, LU, DL, DD, DU, UL, UD, UU = range(9)

    def __init__(self, n: int, bands: torch.Tensor, root: int | None = None):
        from ._lib import HbQ1Band
        self.n = int(n)
        self.bands = bands
        self.dtype = bands.dtype
        self.root = int(root if root is not None else lib().hb_q1band_root(self.n))
        self._s = HbQ1Band()
        self._s.n = self.n
        self._s.root = self.root
        for k in range(9):
            self._s.band[k] = bands[k].data_ptr()
        self._s.dtype = 0 if self.dtype == torch.float64 else 1

    @staticmethod
    def _empty(n: int, dtype, device="cuda") -> torch.Tensor:
        ldb = max(4, (n + 3) // 4 * 4)
        return torch.zeros((9, ldb), dtype=dtype, device=device)

    @classmethod
    def poisson(cls, M: int, dtype=torch.float64, ctx: Context | None = None) -> "BandedMatrixQ1":
        ctx = ctx or default_context()
        A = cls(M * M, cls._empty(M * M, dtype))
        check(lib().hb_q1band_fill_poisson(ctx.handle, M, C.byref(A._s)), "hb_q1band_fill_poisson", ctx.handle)
        A.root = A._s.root
        return A

    @classmethod
    def from_ell(cls, E: SparseMatrixELL, ctx: Context | None = None) -> "BandedMatrixQ1":
        ctx = ctx or default_context()
        A = cls(E.rows(), cls._empty(E.rows(), E.dtype))
        check(lib().hb_q1band_from_ell(ctx.handle, C.byref(E.struct), C.byref(A._s)), "hb_q1band_from_ell",
              ctx.handle)
        A.root = A._s.root
        return A

    @classmethod
    def from_bands(cls, bands, dtype=torch.float64) -> "BandedMatrixQ1":
        bands = [torch.as_tensor(b, dtype=dtype) for b in bands]
        if len(bands) != 9 or len({b.numel() for b in bands}) != 1:
            raise ValueError("nine bands of equal size expected")
        n = bands[0].numel()
        t = cls._empty(n, dtype)
        for k, b in enumerate(bands):
            t[k, :n].copy_(b.reshape(-1))
        return cls(n, t)

    @property
    def struct(self):
        return self._s

    def rows(self) -> int:
        return self.n

    def columns(self) -> int:
        return self.n

    def band(self, k: int) -> torch.Tensor:
        return self.bands[k, : self.n]


class SparseMatrixCSR:
    """Device mirror of a HONEI SparseMatrixCSR (honei/la/sparse_matrix_csr.hh): Ar int64[rows + 1]
    block offsets, Aj int32[nblocks] first column of each block, Ax [nblocks * blocksize]."""

    def __init__(self, rows, cols, blocksize, Ar: torch.Tensor, Aj: torch.Tensor, Ax: torch.Tensor):
        self._rows, self._cols, self._bs = int(rows), int(cols), int(blocksize)
        self.Ar, self.Aj, self.Ax = Ar, Aj, Ax
        self.dtype = Ax.dtype
        self.nblocks = int(Aj.numel())
        self._s = HbCsr(self._rows, self._cols, self._bs, self.nblocks, Ar.data_ptr(), Aj.data_ptr(),
                        Ax.data_ptr(), _DT[Ax.dtype], 0)

    def rows(self) -> int:
        return self._rows

    def columns(self) -> int:
        return self._cols

    def blocksize(self) -> int:
        return self._bs

    @property
    def struct(self) -> HbCsr:
        return self._s

    @classmethod
    def from_reference(cls, csr, ctx: Context | None = None, device="cuda") -> "SparseMatrixCSR":
        """Uploads the reference-layout arrays (u64 Ar, u64 Aj, Ax; problems.CsrMatrix) and
        imports them (hb_csr_import_*)."""
        ctx = ctx or default_context()
        dt = torch.float64 if csr.Ax.dtype == np.float64 else torch.float32
        nb = int(csr.Ar[-1]) if len(csr.Ar) else 0
        Ar_ref = torch.from_numpy(np.ascontiguousarray(csr.Ar, np.uint64).view(np.int64)).to(device)
        Aj_ref = torch.from_numpy(np.ascontiguousarray(csr.Aj[:nb], np.uint64).view(np.int64)).to(device)
        Ax_ref = torch.from_numpy(np.ascontiguousarray(csr.Ax[:nb * csr.blocksize])).to(device)
        Ar = torch.empty(csr.rows + 1, dtype=torch.int64, device=device)
        Aj = torch.empty(max(nb, 1), dtype=torch.int32, device=device)[:nb]
        Ax = torch.empty(max(nb * csr.blocksize, 1), dtype=dt, device=device)[:nb * csr.blocksize]
        out = HbCsr(csr.rows, csr.cols, csr.blocksize, nb, Ar.data_ptr(), Aj.data_ptr(), Ax.data_ptr(), _DT[dt], 0)
        fn = lib().hb_csr_import_f64 if dt == torch.float64 else lib().hb_csr_import_f32
        check(fn(ctx.handle, Ar_ref.data_ptr(), Aj_ref.data_ptr(), Ax_ref.data_ptr(), C.byref(out)),
              "hb_csr_import", ctx.handle)
        return cls(csr.rows, csr.cols, csr.blocksize, Ar, Aj, Ax)


def _spmv_fn(A, kind: str):
    if isinstance(A, BandedMatrixQ1):
        return getattr(lib(), f"hb_q1band_{kind}_{_SUF[A.dtype]}")
    if isinstance(A, SparseMatrixCSR):
        return getattr(lib(), f"hb_csr_{kind}_{_SUF[A.dtype]}")
    return getattr(lib(), f"hb_{kind}_{_SUF[A.dtype]}")


class Product:
    """Product<tags::GPU::CUDA>::value(y, A, x): y = A x, for a SparseMatrixELL
    (honei/la/product.hh:1758-1760), a SparseMatrixCSR (honei/la/product.hh:1762-1764) or a
    BandedMatrixQ1 (honei/la/product.hh:1750-1756)."""

    @staticmethod
    def value(y: torch.Tensor, A, x: torch.Tensor, ctx: Context | None = None):
        if x.numel() != A.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A.columns())
        if A.rows() != y.numel():
            raise VectorSizeDoesNotMatch(A.rows(), y.numel())
        ctx = ctx or default_context()
        if isinstance(A, OrderedMatrixELL):
            return A.product(y, x, ctx)
        fn = _spmv_fn(A, "spmv")
        check(fn(ctx.handle, C.byref(A.struct), _vec(x, A.dtype, "x"), _vec(y, A.dtype, "y")), "Product", ctx.handle)
        return y


class Defect:
    """Defect<tags::GPU::CUDA>::value(r, b, A, x): r = b - A x for a SparseMatrixELL
    (honei/math/defect.hh:660-670), a SparseMatrixCSR (honei/math/defect.hh:673-676) or a
    BandedMatrixQ1 (honei/math/defect.hh:645-658)."""

    @staticmethod
    def value(r: torch.Tensor, b: torch.Tensor, A, x: torch.Tensor, ctx: Context | None = None):
        if x.numel() != A.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A.columns())
        if b.numel() != A.rows():
            raise VectorSizeDoesNotMatch(b.numel(), A.rows())
        if r.numel() != A.rows():
            raise VectorSizeDoesNotMatch(r.numel(), A.rows())
        ctx = ctx or default_context()
        fn = _spmv_fn(A, "defect")
        check(fn(ctx.handle, C.byref(A.struct), _vec(b, A.dtype, "b"), _vec(x, A.dtype, "x"),
                 _vec(r, A.dtype, "r")), "Defect", ctx.handle)
        return r


def _mask8(mask):
    m = (C.c_uint64 * 8)(*[int(v) for v in mask])
    if len(mask) != 8:
        raise ValueError("the Dirichlet mask has 8 entries")
    return m


def _coarse_size(n_fine: int) -> int:
    side = int(round(n_fine ** 0.5))
    return ((side - 1) // 2 + 1) ** 2


class Prolongation:
    """Prolongation<tags::GPU::CUDA, methods::NONE>::value(fine, coarse, mask) -- the matrix-free
    bilinear prolongation of a (2^k + 1)^2 grid (honei/math/prolongation.hh:42-139) followed by
    ApplyDirichletBoundaries with the 8-entry mask."""

    @staticmethod
    def value(fine: torch.Tensor, coarse: torch.Tensor, mask, ctx: Context | None = None):
        if coarse.numel() != _coarse_size(fine.numel()):
            raise VectorSizeDoesNotMatch(coarse.numel(), _coarse_size(fine.numel()))
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_prolongate_{_SUF[fine.dtype]}")
        check(fn(ctx.handle, fine.numel(), _vec(fine, fine.dtype, "fine"), _vec(coarse, fine.dtype, "coarse"),
                 _mask8(mask)), "Prolongation<NONE>", ctx.handle)
        return fine


class Restriction:
    """Restriction<tags::GPU::CUDA, methods::NONE>::value(coarse, fine, mask) -- the matrix-free
    full-weighting restriction (honei/math/restriction.hh:41-170) followed by
    ApplyDirichletBoundaries with the 8-entry mask."""

    @staticmethod
    def value(coarse: torch.Tensor, fine: torch.Tensor, mask, ctx: Context | None = None):
        if coarse.numel() != _coarse_size(fine.numel()):
            raise VectorSizeDoesNotMatch(coarse.numel(), _coarse_size(fine.numel()))
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_restrict_{_SUF[fine.dtype]}")
        check(fn(ctx.handle, fine.numel(), _vec(coarse, fine.dtype, "coarse"), _vec(fine, fine.dtype, "fine"),
                 _mask8(mask)), "Restriction<NONE>", ctx.handle)
        return coarse


def _pair(x, y):
    if x.numel() != y.numel():
        raise VectorSizeDoesNotMatch(y.numel(), x.numel())


class DotProduct:
    """DotProduct<tags::GPU::CUDA>::value(x, y) -> scalar (honei/la/dot_product.hh:358-360)."""

    @staticmethod
    def value(x: torch.Tensor, y: torch.Tensor, ctx: Context | None = None) -> float:
        _pair(x, y)
        ctx = ctx or default_context()
        out = C.c_double() if x.dtype == torch.float64 else C.c_float()
        fn = getattr(lib(), f"hb_dot_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y"), C.byref(out)),
              "DotProduct", ctx.handle)
        return out.value


class Norm:
    """Norm<vnt_l_two, root, tags::GPU::CUDA>::value(x); root=False returns the squared norm."""

    @staticmethod
    def value(x: torch.Tensor, root: bool = False, ctx: Context | None = None) -> float:
        ctx = ctx or default_context()
        out = C.c_double() if x.dtype == torch.float64 else C.c_float()
        fn = getattr(lib(), f"hb_norm_l2_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(x, x.dtype, "x"), int(root), C.byref(out)), "Norm", ctx.handle)
        return out.value


class ScaledSum:
    """ScaledSum<tags::GPU::CUDA>::value(x, y, b): x += b y;  value(r, x, y, b): r = x + b y."""

    @staticmethod
    def value(*args, ctx: Context | None = None):
        ctx = ctx or default_context()
        if len(args) == 3:
            x, y, b = args
            _pair(x, y)
            fn = getattr(lib(), f"hb_scaled_sum_{_SUF[x.dtype]}")
            check(fn(ctx.handle, x.numel(), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y"), b), "ScaledSum", ctx.handle)
            return x
        r, x, y, b = args
        _pair(x, y)
        _pair(x, r)
        fn = getattr(lib(), f"hb_scaled_sum3_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(r, x.dtype, "r"), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y"), b),
              "ScaledSum", ctx.handle)
        return r


class Scale:
    """Scale<tags::GPU::CUDA>::value(x, a): x *= a (honei/la/scale.hh:263)."""

    @staticmethod
    def value(x: torch.Tensor, a: float, ctx: Context | None = None):
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_scale_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(x, x.dtype, "x"), a), "Scale", ctx.handle)
        return x


class Sum:
    """Sum<tags::GPU::CUDA>::value(x, y): x += y (honei/la/sum.hh:684)."""

    @staticmethod
    def value(x: torch.Tensor, y: torch.Tensor, ctx: Context | None = None):
        _pair(x, y)
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_sum_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y")), "Sum", ctx.handle)
        return x


class Difference:
    """Difference: r = x - y."""

    @staticmethod
    def value(r: torch.Tensor, x: torch.Tensor, y: torch.Tensor, ctx: Context | None = None):
        _pair(x, y)
        _pair(x, r)
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_difference_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(r, x.dtype, "r"), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y")),
              "Difference", ctx.handle)
        return r


class ElementProduct:
    """ElementProduct: r = x * y elementwise (the Jacobi apply Product(DV, DV, DV))."""

    @staticmethod
    def value(r: torch.Tensor, x: torch.Tensor, y: torch.Tensor, ctx: Context | None = None):
        _pair(x, y)
        _pair(x, r)
        ctx = ctx or default_context()
        fn = getattr(lib(), f"hb_element_product_{_SUF[x.dtype]}")
        check(fn(ctx.handle, x.numel(), _vec(r, x.dtype, "r"), _vec(x, x.dtype, "x"), _vec(y, x.dtype, "y")),
              "ElementProduct", ctx.handle)
        return r


def convert(dst: torch.Tensor, src: torch.Tensor, ctx: Context | None = None):
    """convert<Tag>(copy, orig) (honei/la/algorithm.hh:163-198): FP64 <-> FP32."""
    _pair(dst, src)
    ctx = ctx or default_context()
    if src.dtype == torch.float64 and dst.dtype == torch.float32:
        check(lib().hb_convert_f64_f32(ctx.handle, src.numel(), dst.data_ptr(), _vec(src, src.dtype, "src")),
              "convert", ctx.handle)
    elif src.dtype == torch.float32 and dst.dtype == torch.float64:
        check(lib().hb_convert_f32_f64(ctx.handle, src.numel(), dst.data_ptr(), _vec(src, src.dtype, "src")),
              "convert", ctx.handle)
    else:
        raise TypeError("convert needs one float64 and one float32 vector")
    return dst


class CGSolver:
    """CGSolver<tags::GPU::CUDA, methods::NONE>::value (honei/math/cg.hh:63-133).

    ``value(A, P, b, x, max_iters, eps_relative=1e-8)`` solves in place into x (x holds x0)
    and returns used_iters; ``last_defect`` holds sqrt(alpha) at exit.
    """

    last_defect = None

    @staticmethod
    def value(A: SparseMatrixELL, P, b: torch.Tensor, x: torch.Tensor, max_iters: int,
              eps_relative: float = 1e-8, ctx: Context | None = None) -> int:
        if b.numel() != A.rows():
            raise VectorSizeDoesNotMatch(b.numel(), A.rows())
        if x.numel() != A.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A.columns())
        ctx = ctx or default_context()
        if isinstance(A, OrderedMatrixELL):
            return CGSolver._value_ordered(A, b, x, max_iters, eps_relative, ctx)
        used = C.c_int64(0)
        d = C.c_double() if A.dtype == torch.float64 else C.c_float()
        fn = getattr(lib(), f"hb_cg_{_SUF[A.dtype]}")
        check(fn(ctx.handle, C.byref(A.struct), _vec(b, A.dtype, "b"), _vec(x, A.dtype, "x"), int(max_iters),
                 eps_relative, C.byref(used), C.byref(d)), "CGSolver", ctx.handle)
        CGSolver.last_defect = d.value
        return used.value

    @staticmethod
    def _value_ordered(O: "OrderedMatrixELL", b, x, max_iters, eps_relative, ctx) -> int:
        """CG on a matrix through its ordered copy (columns renumbered): b and x0 are permuted
        into the copy's numbering once (hb_gather with order), the solve runs on the copy B =
        P A P^T, whose gathers are local, and x is permuted back (hb_gather with pos: x[i] =
        xw[pos[i]]).  The same CG; its dot products add the entries in the copy's order (and in
        the sorted, ranked form each row of B sums its slots in ascending new column), so the
        iterates agree with CG on A to rounding (the parity bar of any reordered reduction)."""
        if not O.columns_renumbered:
            raise ValueError("CG through an ordered copy needs its columns renumbered (ordered(columns=True))")
        n = O.rows()
        suf = _SUF[O.dtype]
        gather = getattr(lib(), f"hb_gather_{suf}")
        bw = torch.empty(n, dtype=O.dtype, device=b.device)
        xw = torch.empty(n, dtype=O.dtype, device=b.device)
        check(gather(ctx.handle, n, O.order.data_ptr(), _vec(b, O.dtype, "b"), bw.data_ptr()), "hb_gather", ctx.handle)
        check(gather(ctx.handle, n, O.order.data_ptr(), _vec(x, O.dtype, "x"), xw.data_ptr()), "hb_gather", ctx.handle)
        used = CGSolver.value(O.B, None, bw, xw, max_iters, eps_relative, ctx=ctx)
        check(gather(ctx.handle, n, O.pos.data_ptr(), xw.data_ptr(), x.data_ptr()), "hb_gather", ctx.handle)
        return used

    @staticmethod
    def set_resident(enable: bool, ctx: Context | None = None) -> bool:
        """Whether CG (and CGSolverVAR with a vector preconditioner) on ctx uses the
        resident-operator kernel where the system fits (the default) or always the streaming
        kernel; returns the previous setting."""
        ctx = ctx or default_context()
        return bool(lib().hb_cg_set_resident(ctx.handle, 1 if enable else 0))

    @staticmethod
    def set_layout(rows_per_thread: int, ctx: Context | None = None) -> int:
        """The streaming CG kernel's layout on ctx: 4 rows per thread (groups of four) or 1 (one
        row per thread); returns the previous setting."""
        ctx = ctx or default_context()
        prev = lib().hb_cg_set_layout(ctx.handle, int(rows_per_thread))
        if prev < 0:
            raise ValueError("rows_per_thread must be 1 or 4")
        return prev


class CGSolverVAR:
    """CGSolver<tags::GPU::CUDA, methods::VAR>::value (honei/math/cg.hh:140-219): CG with the
    preconditioner container P -- a CUDA vector (z = P r elementwise, e.g. Jacobi
    0.7 / diag(A)) or a SparseMatrixELL (z = P r, e.g. SPAI / SAINV).

    ``value(A, P, b, x, max_iters, eps_relative=1e-8)`` solves in place into x (x holds x0) and
    returns used_iters; ``last_defect`` holds ||r|| at exit.
    """

    last_defect = None

    @staticmethod
    def value(A: SparseMatrixELL, P, b: torch.Tensor, x: torch.Tensor, max_iters: int,
              eps_relative: float = 1e-8, ctx: Context | None = None) -> int:
        if b.numel() != A.rows():
            raise VectorSizeDoesNotMatch(b.numel(), A.rows())
        if x.numel() != A.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A.columns())
        ctx = ctx or default_context()
        if isinstance(A, OrderedMatrixELL):
            return CGSolver._value_ordered(A, b, x, max_iters, eps_relative, ctx)
        used = C.c_int64(0)
        d = C.c_double() if A.dtype == torch.float64 else C.c_float()
        if isinstance(P, SparseMatrixELL):
            if P.rows() != A.rows() or P.columns() != A.columns():
                raise VectorSizeDoesNotMatch(P.rows(), A.rows())
            fn = getattr(lib(), f"hb_cg_var_ell_{_SUF[A.dtype]}")
            pa = C.byref(P.struct)
        else:
            if P.numel() != A.rows():
                raise VectorSizeDoesNotMatch(P.numel(), A.rows())
            fn = getattr(lib(), f"hb_cg_var_diag_{_SUF[A.dtype]}")
            pa = _vec(P, A.dtype, "P")
        check(fn(ctx.handle, C.byref(A.struct), pa, _vec(b, A.dtype, "b"), _vec(x, A.dtype, "x"), int(max_iters),
                 eps_relative, C.byref(used), C.byref(d)), "CGSolver<VAR>", ctx.handle)
        CGSolverVAR.last_defect = d.value
        return used.value


class SPAI2:
    """SPAI2<tags::GPU::CUDA>::value(M, A) (honei/math/spai2.hh:294-298, hb_spai2_*): the sparse
    approximate inverse of the square matrix A on A's pattern, bit-identical to
    SPAI2<tags::CPU::SSE> (honei/math/spai2.hh:129-260).  The result is the matrix preconditioner
    CGSolverVAR takes.

    ``value(A)`` returns a new SparseMatrixELL M; ``value(A, M)`` fills a caller-provided M of
    A's layout and returns it.
    """

    @staticmethod
    def value(A: SparseMatrixELL, M: SparseMatrixELL | None = None, ctx: Context | None = None) -> SparseMatrixELL:
        if A.rows() != A.columns():
            raise MatrixRowsDoNotMatch(A.rows(), A.columns())
        ctx = ctx or default_context()
        if M is None:
            M = SparseMatrixELL(A.rows(), A.columns(), A.K, A.ld, torch.empty_like(A.Aj), torch.empty_like(A.Ax))
        elif (M.rows(), M.columns(), M.K, M.ld, M.dtype) != (A.rows(), A.columns(), A.K, A.ld, A.dtype):
            raise MatrixRowsDoNotMatch(M.rows(), A.rows())
        fn = getattr(lib(), f"hb_spai2_{_SUF[A.dtype]}")
        check(fn(ctx.handle, C.byref(A.struct), C.byref(M.struct)), "SPAI2", ctx.handle)
        return M


class MGData:
    """Device MG hierarchy (MGData + the V(n_pre, n_post) cycle; honei/math/mg.hh:57-243, 567-662).

    Levels are coarsest first (HONEI level 1 first); ``prol[l]`` maps level l to l+1 and
    ``res[l] = prol[l]^T``.  Smoother: damped Jacobi (RISmoother with the "jac"
    preconditioner); coarse solver: CG on level 1 with the MG eps.
    """

    def __init__(self, A, prol, res, max_iters=100, max_iters_coarse=1000, n_pre=2, n_post=2,
                 damping=0.7, eps=1e-8, ctx: Context | None = None, banded: bool = False):
        from ._lib import HbMGParams, HbQ1Band
        self.ctx = ctx or default_context()
        self.A, self.prol, self.res = list(A), list(prol), list(res)
        self.dtype = self.A[0].dtype
        L = len(self.A)
        self._A = (HbEll * L)(*[a.struct for a in self.A])
        self._P = (HbEll * max(L - 1, 1))(*[p.struct for p in self.prol])
        self._R = (HbEll * max(L - 1, 1))(*[r.struct for r in self.res])
        self.params = HbMGParams(max_iters, max_iters_coarse, n_pre, n_post, damping, eps)
        h = C.c_void_p()
        if banded:
            # banded copies of the levels; transfers become matrix-free (prol / res unused)
            self.bands = [BandedMatrixQ1.from_ell(a, ctx=self.ctx) for a in self.A]
            self._B = (HbQ1Band * L)(*[b.struct for b in self.bands])
            check(lib().hb_mg_create_banded(self.ctx.handle, L, self._A, self._B, C.byref(self.params), C.byref(h)),
                  "hb_mg_create_banded", self.ctx.handle)
        else:
            check(lib().hb_mg_create(self.ctx.handle, L, self._A, self._P, self._R, C.byref(self.params),
                                     C.byref(h)), "hb_mg_create", self.ctx.handle)
        self.handle = h
        self.used_iters = 0

    @classmethod
    def from_hierarchy(cls, H, dtype=np.float64, ctx: Context | None = None, **kw) -> "MGData":
        """From a host problems.MGHierarchy (reference-layout matrices)."""
        ctx = ctx or default_context()
        Hd = H if dtype == np.float64 else H.astype(dtype)
        up = lambda m: SparseMatrixELL.from_reference(m, ctx)  # noqa: E731
        return cls([up(a) for a in Hd.A], [up(p) for p in Hd.prol], [up(r) for r in Hd.res], ctx=ctx, **kw)

    def configure(self, **kw):
        """MGUtil::configure (honei/math/mg.hh:426-439)."""
        for k, v in kw.items():
            setattr(self.params, k, v)
        check(lib().hb_mg_set_params(self.handle, C.byref(self.params)), "hb_mg_set_params", self.ctx.handle)

    def close(self):
        if getattr(self, "handle", None):
            lib().hb_mg_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class MGSolver:
    """MGSolver<tags::GPU::CUDA, Norm<vnt_l_two, true>>::value(data, x, b) (honei/math/mg.hh:1093-1127).

    Returns (used_cycles, initial_norm, final_norm); x holds x0 on entry.
    """

    @staticmethod
    def value(data: MGData, b: torch.Tensor, x: torch.Tensor):
        n = data.A[-1].rows()
        if b.numel() != n:
            raise VectorSizeDoesNotMatch(b.numel(), n)
        if x.numel() != n:
            raise VectorSizeDoesNotMatch(x.numel(), n)
        data.ctx.bind_stream()
        used = C.c_int64(0)
        if data.dtype == torch.float64:
            rn = (C.c_double * 2)()
            st = lib().hb_mg_solve_f64(data.handle, _vec(b, data.dtype, "b"), _vec(x, data.dtype, "x"),
                                       C.byref(used), rn)
        else:
            rn = (C.c_float * 2)()
            st = lib().hb_mg_solve_f32(data.handle, _vec(b, data.dtype, "b"), _vec(x, data.dtype, "x"),
                                       C.byref(used), rn)
        check(st, "MGSolver", data.ctx.handle)
        data.used_iters = used.value
        return used.value, rn[0], rn[1]


class IRSolver:
    """IRSolver<Outer=double, Inner=float, Norm<l2, true>> (honei/math/ir.hh:30-78).

    ``value(A64, b, x, mg32, eps, max_iters, warm_start=True)`` with an FP32 MG inner solve, or
    ``value_cg(A64, A32, b, x, eps, inner_eps, inner_max_iters, max_iters)`` with FP32 CG.
    Both return (used_outer, initial_norm, final_norm[, inner_iterations]).
    """

    @staticmethod
    def value(A64: SparseMatrixELL, b: torch.Tensor, x: torch.Tensor, mg32: MGData, eps: float = 1e-10,
              max_iters: int = 100, warm_start: bool = True, ctx: Context | None = None):
        if b.numel() != A64.rows():
            raise VectorSizeDoesNotMatch(b.numel(), A64.rows())
        if x.numel() != A64.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A64.columns())
        ctx = ctx or default_context()
        used = C.c_int64(0)
        rn = (C.c_double * 2)()
        check(lib().hb_ir_mg_solve(ctx.handle, C.byref(A64.struct), mg32.handle, _vec(b, torch.float64, "b"),
                                   _vec(x, torch.float64, "x"), eps, max_iters, int(warm_start), C.byref(used), rn),
              "IRSolver", ctx.handle)
        return used.value, rn[0], rn[1]

    @staticmethod
    def value_cg(A64: SparseMatrixELL, A32: SparseMatrixELL, b: torch.Tensor, x: torch.Tensor, eps: float = 1e-10,
                 inner_eps: float = 1e-3, inner_max_iters: int = 100000, max_iters: int = 100,
                 ctx: Context | None = None):
        if b.numel() != A64.rows():
            raise VectorSizeDoesNotMatch(b.numel(), A64.rows())
        if x.numel() != A64.columns():
            raise VectorSizeDoesNotMatch(x.numel(), A64.columns())
        ctx = ctx or default_context()
        used, inner = C.c_int64(0), C.c_int64(0)
        rn = (C.c_double * 2)()
        check(lib().hb_ir_cg_solve(ctx.handle, C.byref(A64.struct), C.byref(A32.struct), _vec(b, torch.float64, "b"),
                                   _vec(x, torch.float64, "x"), eps, inner_eps, inner_max_iters, max_iters,
                                   C.byref(used), C.byref(inner), rn), "IRSolver", ctx.handle)
        return used.value, rn[0], rn[1], inner.value


class Q1System:
    """A served SPD Q1 system (hb_q1): FP64 matrix, FP32 copy and the device-built FP32 MG
    hierarchy (bilinear transfers, Galerkin levels) for a grid of any side.

        q = Q1System(M, coef)                        # coef: CUDA float64 (M-1)^2 or None
        info = q.solve(b, x, eps=1e-8)               # IR + FP32 MG-preconditioned CG
    """

    def __init__(self, M: int, coef: torch.Tensor | None = None, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.M = int(M)
        cptr = None
        if coef is not None:
            if coef.numel() != (M - 1) * (M - 1):
                raise VectorSizeDoesNotMatch(coef.numel(), (M - 1) * (M - 1))
            cptr = _vec(coef, torch.float64, "coef")
        h = C.c_void_p()
        check(lib().hb_q1_create(self.ctx.handle, self.M, cptr, C.byref(h)), "hb_q1_create", self.ctx.handle)
        self.handle = h
        nl = C.c_int(0)
        sides = (C.c_int64 * 64)()
        check(lib().hb_q1_levels(h, C.byref(nl), sides), "hb_q1_levels")
        self.sides = [sides[i] for i in range(nl.value)]

    def set_fused_tail(self, max_rows: int):
        """hb_q1_set_fused_tail: the levels of at most max_rows rows in one launch (0: per level)."""
        check(lib().hb_q1_set_fused_tail(self.handle, int(max_rows)), "hb_q1_set_fused_tail", self.ctx.handle)

    @staticmethod
    def solve_batch(systems, bs, xs, eps=1e-8, inner_eps=1e-3, max_outer=50, max_inner=1000, cluster=8,
                    threads=256, max_clusters=0, ctx: Context | None = None):
        """hb_q1_batch_solve: every system (distinct Q1System objects) solved in one launch, one
        thread-block cluster per system at a time; xs hold the initial guesses.  Returns one info
        dict per system."""
        from .batch import HbBatchConfig, HbBatchResult
        ctx = ctx or default_context()
        n = len(systems)
        if not (n == len(bs) == len(xs)):
            raise ValueError("one b and one x per system")
        for q, b, x in zip(systems, bs, xs):
            if b.numel() != q.M * q.M:
                raise VectorSizeDoesNotMatch(b.numel(), q.M * q.M)
            if x.numel() != q.M * q.M:
                raise VectorSizeDoesNotMatch(x.numel(), q.M * q.M)
        hs = (C.c_void_p * max(n, 1))(*[q.handle.value for q in systems])
        bp = (C.c_void_p * max(n, 1))(*[_vec(b, torch.float64, "b") for b in bs])
        xp = (C.c_void_p * max(n, 1))(*[_vec(x, torch.float64, "x") for x in xs])
        res = (HbBatchResult * max(n, 1))()
        cfg = HbBatchConfig(cluster, threads, max_clusters)
        ctx.bind_stream()
        check(lib().hb_q1_batch_solve(ctx.handle, hs, bp, xp, n, eps, inner_eps, max_outer, max_inner, C.byref(cfg),
                                      res), "hb_q1_batch_solve", ctx.handle)
        return [{"iterations": r.iterations, "outer": r.outer, "defect0": r.defect0, "defect": r.defect,
                 "true_relres": r.true_relres, "status": r.status} for r in res[:n]]

    def level(self, l: int):
        """(A64, A32, P32, R32) device views of level l (P/R None on the finest level)."""
        e = [HbEll() for _ in range(4)]
        check(lib().hb_q1_level(self.handle, l, *[C.byref(x) for x in e]), "hb_q1_level")
        A64, A32 = SparseMatrixELL.from_struct(e[0]), SparseMatrixELL.from_struct(e[1])
        if l + 1 < len(self.sides):
            return A64, A32, SparseMatrixELL.from_struct(e[2]), SparseMatrixELL.from_struct(e[3])
        return A64, A32, None, None

    @property
    def A(self) -> SparseMatrixELL:
        return self.level(len(self.sides) - 1)[0]

    def solve(self, b: torch.Tensor, x: torch.Tensor, eps=1e-8, inner_eps=1e-3, max_outer=50, max_inner=1000):
        n = self.M * self.M
        if b.numel() != n:
            raise VectorSizeDoesNotMatch(b.numel(), n)
        if x.numel() != n:
            raise VectorSizeDoesNotMatch(x.numel(), n)
        from .batch import HbBatchResult
        info = HbBatchResult()
        self.ctx.bind_stream()
        check(lib().hb_q1_solve(self.handle, _vec(b, torch.float64, "b"), _vec(x, torch.float64, "x"), eps,
                                inner_eps, max_outer, max_inner, C.byref(info)), "hb_q1_solve", self.ctx.handle)
        return dict(iterations=info.iterations, outer=info.outer, defect0=info.defect0, defect=info.defect,
                    true_relres=info.true_relres, status=info.status)

    def close(self):
        if getattr(self, "handle", None):
            lib().hb_q1_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
