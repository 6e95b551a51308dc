"""Seeded problem generators for the HONEI sparse-solver path (host side, numpy).

Every matrix is produced in the reference's SparseMatrixELL layout
(honei/la/sparse_matrix_ell-impl.hh:75-122): entry k of row r at
``(k % T) + r*T + (k // T)*stride``, ``stride = 32 * ceil(rows*T / 32)``,
``Arl[r] = ceil(nnz_r / T)``, 64-bit column indices, columns ascending per row, explicit
zeros dropped.  These arrays are exactly what HONEI's ``SparseMatrixELL`` holds, so they feed
both the reference CPU path and the device import (``hb_ell_import_*``).

Q1 Poisson with Dirichlet rows set to identity follows
``FillMatrix<Tag, POISSON, DIRICHLET_0>`` (honei/math/fill_matrix.hh:37-77): interior rows
carry the 9-point stencil 8/3 and -1/3 and keep their couplings to boundary nodes.  The
variable-coefficient form assembles the bilinear element matrix
``K_e = k_c/6 * [[4,-1,-2,-1],[-1,4,-1,-2],[-2,-1,4,-1],[-1,-2,-1,4]]`` per cell; with
``k == 1`` it reproduces the constant stencil bit for bit (the sums are formed as
``4*(k1+k2+k3+k4)/6``, ``-(ka+kb)/6`` and ``-2*kc/6``).

MG transfer matrices follow ``Prolongation<Tag, methods::NONE>`` + ``ApplyDirichletBoundaries``
(honei/math/prolongation.hh:42-139): bilinear interpolation, fine Dirichlet rows zeroed;
the restriction is the transpose (``Transposition``, honei/math/transposition.hh:30-50).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


def ell_stride(rows: int, threads: int = 1) -> int:
    """Row stride of the reference ELL layout (sparse_matrix_ell-impl.hh:97-98)."""
    return 32 * ((rows * threads + 31) // 32)


@dataclasses.dataclass
class EllMatrix:
    """A sparse matrix in the reference's SparseMatrixELL layout (host arrays)."""

    rows: int
    cols: int
    stride: int
    ncpr: int
    threads: int
    Aj: np.ndarray   # uint64[ncpr*stride]
    Ax: np.ndarray   # float64 or float32 [ncpr*stride]
    Arl: np.ndarray  # uint64[rows]
    nnz: int = 0

    @property
    def dtype(self):
        return self.Ax.dtype

    def astype(self, dtype) -> "EllMatrix":
        """Same pattern with values cast (the reference fills FP32 matrices from FP64 values)."""
        return dataclasses.replace(self, Ax=self.Ax.astype(dtype))

    def info(self) -> list[int]:
        return [self.rows, self.cols, self.stride, self.ncpr, self.threads]

    def to_csr(self):
        """(indptr, indices, data) of the stored entries, per-row slot order."""
        T, stride = self.threads, self.stride
        counts = self.Arl.astype(np.int64) * T
        indptr = np.zeros(self.rows + 1, np.int64)
        np.cumsum(counts, out=indptr[1:])
        row = np.repeat(np.arange(self.rows, dtype=np.int64), counts)
        k = np.arange(indptr[-1], dtype=np.int64) - indptr[row]
        pos = (k % T) + row * T + (k // T) * stride
        return indptr, self.Aj[pos].astype(np.int64), self.Ax[pos]


def ell_from_csr(rows: int, cols: int, indptr, indices, data, threads: int = 1,
                 dtype=np.float64) -> EllMatrix:
    """Packs a CSR matrix (ascending columns per row) into the reference ELL layout.

    Zero values are dropped before packing, as the reference constructor does
    (sparse_matrix_ell-impl.hh:108-119).
    """
    indptr = np.asarray(indptr, np.int64)
    indices = np.asarray(indices, np.int64)
    data = np.asarray(data)
    keep = data != 0
    row_of = np.repeat(np.arange(rows, dtype=np.int64), np.diff(indptr))
    row_of, indices, data = row_of[keep], indices[keep], data[keep]
    counts = np.bincount(row_of, minlength=rows).astype(np.int64)
    T = int(threads)
    maxc = int(counts.max()) if rows else 0
    ncpr = max(1, maxc)
    ncpr = int(math.ceil(ncpr / T))
    stride = ell_stride(rows, T)
    start = np.zeros(rows + 1, np.int64)
    np.cumsum(counts, out=start[1:])
    k = np.arange(len(indices), dtype=np.int64) - start[row_of]
    pos = (k % T) + row_of * T + (k // T) * stride
    Aj = np.zeros(ncpr * stride, np.uint64)
    Ax = np.zeros(ncpr * stride, dtype)
    Aj[pos] = indices.astype(np.uint64)
    Ax[pos] = data.astype(dtype)
    Arl = ((counts + T - 1) // T).astype(np.uint64)
    return EllMatrix(rows, cols, stride, ncpr, T, Aj, Ax, Arl, int(len(indices)))


@dataclasses.dataclass
class CsrMatrix:
    """A sparse matrix in the reference's SparseMatrixCSR layout (host arrays,
    honei/la/sparse_matrix_csr.hh): ``Ar[rows + 1]`` block offsets, ``Aj[nblocks]`` the first
    column of each block, ``Ax[nblocks * blocksize]`` (csr::blocksize values per block; lanes
    without an entry hold zero)."""

    rows: int
    cols: int
    blocksize: int
    Ar: np.ndarray   # uint64[rows + 1]
    Aj: np.ndarray   # uint64[nblocks]
    Ax: np.ndarray   # float64 or float32 [nblocks * blocksize]
    used: int = 0    # stored entries (used_elements)

    @property
    def dtype(self):
        return self.Ax.dtype

    @property
    def nblocks(self) -> int:
        return int(self.Ar[-1]) if len(self.Ar) else 0

    def astype(self, dtype) -> "CsrMatrix":
        return dataclasses.replace(self, Ax=self.Ax.astype(dtype))

    def to_dense(self) -> np.ndarray:
        """Dense copy (small matrices, for tests): lanes at or beyond cols are dropped."""
        D = np.zeros((self.rows, self.cols), self.Ax.dtype)
        bs = self.blocksize
        for r in range(self.rows):
            for i in range(int(self.Ar[r]), int(self.Ar[r + 1])):
                for k in range(bs):
                    c = int(self.Aj[i]) + k
                    if c < self.cols:
                        D[r, c] += self.Ax[i * bs + k]
        return D


def csr_blocked(rows: int, cols: int, indptr, indices, data, blocksize: int = 1, dtype=np.float64) -> CsrMatrix:
    """The reference's SparseMatrixCSR(SparseMatrix) conversion with csr::blocksize = blocksize
    (honei/la/sparse_matrix_csr-impl.hh:98-136): per row, walking the stored entries in column
    order, a block starts at the entry's column rounded down to a multiple of blocksize and
    takes the following entries that fall on its lanes; lanes without an entry hold zero.
    ``indices`` strictly ascending per row; every stored entry is kept, zero values included."""
    bs = int(blocksize)
    if bs < 1:
        raise ValueError("blocksize must be >= 1")
    indptr = np.asarray(indptr, np.int64)
    indices = np.asarray(indices, np.int64)
    data = np.asarray(data)
    n = int(indptr[-1]) if rows else 0
    row_of = np.repeat(np.arange(rows, dtype=np.int64), np.diff(indptr))
    if n and not np.all((np.diff(indices[:n]) > 0) | (np.diff(row_of) != 0)):
        raise ValueError("column indices must ascend strictly within each row (a SparseMatrix's rows do)")
    # a block is a run of entries sharing (row, column // blocksize): the blocks the
    # reference's entry walk forms on strictly ascending columns
    blk = indices[:n] // bs
    new = np.ones(n, bool)
    new[1:] = (row_of[1:] != row_of[:-1]) | (blk[1:] != blk[:-1])
    bid = np.cumsum(new) - 1
    nb = int(bid[-1]) + 1 if n else 0
    Ax = np.zeros(nb * bs, dtype)
    Ax[bid * bs + indices[:n] % bs] = data[:n]
    Ar = np.zeros(rows + 1, np.uint64)
    np.cumsum(np.bincount(row_of[new], minlength=rows), out=Ar[1:])
    return CsrMatrix(rows, cols, bs, Ar, (blk[new] * bs).astype(np.uint64), Ax, n)


def csr_from_ell(A: "EllMatrix", blocksize: int = 1) -> CsrMatrix:
    """SparseMatrixCSR(SparseMatrixELL) (sparse_matrix_csr-impl.hh:84-96): through the
    matrix's stored entries, ascending columns per row."""
    ip, ix, dv = A.to_csr()
    order = np.lexsort((ix, np.repeat(np.arange(A.rows), np.diff(ip))))
    return csr_blocked(A.rows, A.cols, ip, ix[order], dv[order], blocksize, A.Ax.dtype)


def csr_product_test_matrix(size: int, dtype=np.float64):
    """The matrix of the reference's CSR product test (honei/la/product_TEST.cc:936-941): size x
    (size + 3), element with flat index i = r * (size + 3) + c set to i / 1.234 when i % 5 == 0
    (the element at index 0 stores 0), and its x: 4 everywhere, x[0] = 1, x[1] = 2.  Returns
    (indptr, indices, data, x)."""
    cols = size + 3
    flat = np.arange(0, size * cols, 5, dtype=np.int64)
    r, c = flat // cols, flat % cols
    data = (flat.astype(np.float64) / 1.234).astype(dtype)
    indptr = np.zeros(size + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=size), out=indptr[1:])
    x = np.full(cols, 4, dtype)
    x[0], x[1] = 1, 2
    return indptr, c, data, x


def q1_poisson_csr(M: int, coef=None, symmetric: bool = False):
    """CSR of the Q1 Poisson matrix on an M x M node grid, Dirichlet rows = identity.

    ``coef`` is None (unit coefficient) or an (M-1, M-1) array of per-cell coefficients.
    Node r = i*M + j (lexicographic), as FillMatrix numbers them.  ``symmetric`` drops the
    interior rows' couplings to boundary nodes (Dirichlet values eliminated into the right-hand
    side), which makes the matrix SPD; the default keeps them, as FillMatrix does.
    """
    M = int(M)
    N = M * M
    if coef is None:
        coef = np.ones((max(M - 1, 0), max(M - 1, 0)), np.float64)
    coef = np.asarray(coef, np.float64)
    ii, jj = np.divmod(np.arange(N, dtype=np.int64), M)
    bnd = (ii == 0) | (ii == M - 1) | (jj == 0) | (jj == M - 1)
    inner = np.nonzero(~bnd)[0]
    counts = np.where(bnd, 1, 9).astype(np.int64)
    indptr = np.zeros(N + 1, np.int64)
    np.cumsum(counts, out=indptr[1:])
    indices = np.empty(indptr[-1], np.int64)
    data = np.empty(indptr[-1], np.float64)
    b_rows = np.nonzero(bnd)[0]
    indices[indptr[b_rows]] = b_rows
    data[indptr[b_rows]] = 1.0
    if len(inner):
        i, j = ii[inner], jj[inner]
        k_nw, k_ne = coef[i - 1, j - 1], coef[i - 1, j]
        k_sw, k_se = coef[i, j - 1], coef[i, j]
        six = 6.0
        vals = [
            -(2.0 * k_nw) / six,            # (i-1, j-1)
            -(k_nw + k_ne) / six,           # (i-1, j)
            -(2.0 * k_ne) / six,            # (i-1, j+1)
            -(k_nw + k_sw) / six,           # (i,   j-1)
            (4.0 * (((k_nw + k_ne) + k_sw) + k_se)) / six,  # diagonal
            -(k_ne + k_se) / six,           # (i,   j+1)
            -(2.0 * k_sw) / six,            # (i+1, j-1)
            -(k_sw + k_se) / six,           # (i+1, j)
            -(2.0 * k_se) / six,            # (i+1, j+1)
        ]
        offs = [-M - 1, -M, -M + 1, -1, 0, 1, M - 1, M, M + 1]
        base = indptr[inner]
        for s, (o, v) in enumerate(zip(offs, vals)):
            indices[base + s] = inner + o
            data[base + s] = v
        if symmetric:
            keep = np.ones(len(indices), bool)
            row_of = np.repeat(np.arange(N, dtype=np.int64), counts)
            keep[(~bnd[row_of]) & bnd[indices]] = False
            new_counts = np.bincount(row_of[keep], minlength=N).astype(np.int64)
            indptr = np.zeros(N + 1, np.int64)
            np.cumsum(new_counts, out=indptr[1:])
            indices, data = indices[keep], data[keep]
    return indptr, indices, data


def q1_poisson(M: int, coef=None, threads: int = 1, dtype=np.float64, symmetric: bool = False) -> EllMatrix:
    """Q1 Poisson ELL matrix (see module docstring); FP32 values are the FP64 values cast."""
    indptr, indices, data = q1_poisson_csr(M, coef, symmetric)
    A = ell_from_csr(M * M, M * M, indptr, indices, data, threads, np.float64)
    return A if dtype == np.float64 else A.astype(dtype)


def log_uniform_coef(M: int, lo: float, hi: float, seed: int) -> np.ndarray:
    """Per-cell coefficient 10**U(log10 lo, log10 hi) on the (M-1)^2 cells, seeded."""
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(math.log10(lo), math.log10(hi), size=(M - 1, M - 1))


def coarsen_coef(coef: np.ndarray) -> np.ndarray:
    """Cell coefficients of the next coarser grid: mean of the 2x2 children."""
    c = np.asarray(coef, np.float64)
    return ((c[0::2, 0::2] + c[0::2, 1::2]) + (c[1::2, 0::2] + c[1::2, 1::2])) / 4.0


def uniform_vector(n: int, seed: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    """Seeded U[lo, hi] vector (x_true, SpMV inputs)."""
    return np.random.default_rng(seed).uniform(lo, hi, size=n)


def permute_csr(n: int, indptr, indices, data, perm):
    """A'[perm[i], perm[j]] = A[i, j], columns re-sorted ascending per row."""
    perm = np.asarray(perm, np.int64)
    indptr = np.asarray(indptr, np.int64)
    counts = np.diff(indptr)
    row = np.repeat(np.arange(n, dtype=np.int64), counts)
    new_row = perm[row]
    new_col = perm[np.asarray(indices, np.int64)]
    order = np.lexsort((new_col, new_row))
    new_counts = np.bincount(new_row, minlength=n)
    new_indptr = np.zeros(n + 1, np.int64)
    np.cumsum(new_counts, out=new_indptr[1:])
    return new_indptr, new_col[order], np.asarray(data)[order]


def random_permutation(n: int, seed: int) -> np.ndarray:
    """Seeded Fisher-Yates permutation."""
    return np.random.default_rng(seed).permutation(n)


def q1_poisson_permuted(M: int, seed: int, coef=None, threads: int = 1, dtype=np.float64):
    """(A', perm) with A'[perm[i], perm[j]] = A[i, j]; permute vectors with v'[perm] = v."""
    indptr, indices, data = q1_poisson_csr(M, coef)
    perm = random_permutation(M * M, seed)
    p_indptr, p_indices, p_data = permute_csr(M * M, indptr, indices, data, perm)
    A = ell_from_csr(M * M, M * M, p_indptr, p_indices, p_data, threads, np.float64)
    return (A if dtype == np.float64 else A.astype(dtype)), perm


def coarse_side(M: int) -> int:
    """Side of the next coarser grid: the fine nodes with even index, plus the last node when
    M is even (then the last coarse interval spans one fine interval)."""
    return int(M) // 2 + 1


def _interp_1d(i: int, Mf: int):
    """1-D bilinear interpolation of fine coordinate i: list of (coarse index, weight)."""
    Mc = coarse_side(Mf)
    ci = lambda k: Mc - 1 if k == Mf - 1 else k // 2  # noqa: E731
    if i % 2 == 0 or i == Mf - 1:
        return [(ci(i), 1.0)]
    return [(ci(i - 1), 0.5), (ci(i + 1), 0.5)]


def prolongation_csr(Mc: int = None, Mf: int = None):
    """Bilinear Q1 prolongation to an Mf x Mf grid from its coarse grid (coarse_side(Mf)), fine
    Dirichlet rows zero.  Pass Mc (odd grids, Mf = 2 Mc - 1) or Mf (any side >= 3)."""
    if Mf is None:
        Mf = 2 * int(Mc) - 1
    Mf = int(Mf)
    Mc = coarse_side(Mf)
    tab = [_interp_1d(i, Mf) for i in range(Mf)]
    rows, cols, vals = [], [], []
    for I in range(1, Mf - 1):
        for J in range(1, Mf - 1):
            f = I * Mf + J
            for ca, wa in tab[I]:
                for cb, wb in tab[J]:
                    rows.append(f)
                    cols.append(ca * Mc + cb)
                    vals.append(wa * wb)
    Nf, Nc = Mf * Mf, Mc * Mc
    r = np.asarray(rows, np.int64)
    c = np.asarray(cols, np.int64)
    v = np.asarray(vals, np.float64)
    order = np.lexsort((c, r))
    r, c, v = r[order], c[order], v[order]
    indptr = np.zeros(Nf + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=Nf), out=indptr[1:])
    return Nf, Nc, indptr, c, v


def transpose_csr(rows: int, cols: int, indptr, indices, data):
    """CSR transpose with ascending columns per row (what Transposition produces)."""
    indptr = np.asarray(indptr, np.int64)
    r = np.repeat(np.arange(rows, dtype=np.int64), np.diff(indptr))
    c = np.asarray(indices, np.int64)
    order = np.lexsort((r, c))
    t_indptr = np.zeros(cols + 1, np.int64)
    np.cumsum(np.bincount(c, minlength=cols), out=t_indptr[1:])
    return t_indptr, r[order], np.asarray(data)[order]


@dataclasses.dataclass
class MGHierarchy:
    """Levels coarsest first (HONEI level 1 == index 0), as MGData stores them."""

    A: list      # EllMatrix per level
    prol: list   # EllMatrix, prol[l]: level l -> l+1
    res: list    # EllMatrix, res[l] = prol[l]^T
    sides: list  # grid side per level

    def astype(self, dtype) -> "MGHierarchy":
        return MGHierarchy([a.astype(dtype) for a in self.A], [p.astype(dtype) for p in self.prol],
                           [r.astype(dtype) for r in self.res], list(self.sides))


def galerkin_csr(A: EllMatrix, prol: EllMatrix, res: EllMatrix):
    """CSR of the Galerkin coarse operator R A P (columns ascending, zeros dropped)."""
    import scipy.sparse as sp

    def csr(m):
        ip, ix, dv = m.to_csr()
        return sp.csr_matrix((dv, ix, ip), shape=(m.rows, m.cols))

    Ac = (csr(res) @ csr(A) @ csr(prol)).tocsr()
    Ac.eliminate_zeros()
    # coarse nodes no fine interior node interpolates from (the last line of an even-sided
    # grid) have empty rows and columns: they get identity rows (their correction is zero)
    dead = np.nonzero(np.diff(Ac.indptr) == 0)[0]
    if len(dead):
        Ac = (Ac + sp.csr_matrix((np.ones(len(dead)), (dead, dead)), shape=Ac.shape)).tocsr()
    Ac.sort_indices()
    return Ac.shape[0], Ac.indptr.astype(np.int64), Ac.indices.astype(np.int64), Ac.data


def mg_hierarchy(M: int, coarsest: int = 9, coef=None, threads: int = 1, coarse: str = "auto",
                 symmetric: bool = False) -> MGHierarchy:
    """Q1 Poisson hierarchy on sides M, (M+1)/2, ..., coarsest (all of the form 2^k + 1).

    coarse = "rediscretize": every level is the Q1 matrix of its own grid (coarser cell
    coefficients = 2x2 means).  coarse = "galerkin": A_{l-1} = R_l A_l P_l from the finest
    matrix down (robust for jumping coefficients, where rediscretisation diverges).
    "auto" = rediscretize for the unit coefficient, galerkin for a coefficient field.
    """
    if coarse == "auto":
        coarse = "rediscretize" if coef is None else "galerkin"
    if coarse not in ("rediscretize", "galerkin"):
        raise ValueError(coarse)
    sides = [int(M)]
    while sides[-1] > coarsest:
        sides.append(coarse_side(sides[-1]))
    sides = sides[::-1]
    coefs = [None] * len(sides)
    if coef is not None:
        if coarse == "rediscretize" and any((s - 1) % 2 for s in sides[1:]):
            raise ValueError("rediscretised coefficient levels need sides 2^k + 1")
        coefs[-1] = np.asarray(coef, np.float64)
        for l in range(len(sides) - 2, -1, -1):
            coefs[l] = coarsen_coef(coefs[l + 1]) if coarse == "rediscretize" else None
    prol, res = [], []
    for l in range(len(sides) - 1):
        nf, nc, ip, ix, dv = prolongation_csr(Mf=sides[l + 1])
        prol.append(ell_from_csr(nf, nc, ip, ix, dv, threads))
        t_ip, t_ix, t_dv = transpose_csr(nf, nc, ip, ix, dv)
        res.append(ell_from_csr(nc, nf, t_ip, t_ix, t_dv, threads))
    if coarse == "rediscretize":
        A = [q1_poisson(s, coefs[l], threads, symmetric=symmetric) for l, s in enumerate(sides)]
    else:
        A = [None] * len(sides)
        A[-1] = q1_poisson(sides[-1], coefs[-1], threads, symmetric=symmetric)
        for l in range(len(sides) - 1, 0, -1):
            n, ip, ix, dv = galerkin_csr(A[l], prol[l - 1], res[l - 1])
            A[l - 1] = ell_from_csr(n, n, ip, ix, dv, threads)
    return MGHierarchy(A, prol, res, sides)


# ---------------------------------------------------------------------------------------------
# HONEI file formats (honei/math/matrix_io.hh:433-582, honei/math/vector_io.hh:52-115)
# ---------------------------------------------------------------------------------------------
def write_ell(path: str, A: EllMatrix) -> None:
    """Binary ELL file: u64 {size, rows, cols, stride, ncpr}, u64 Aj[size], f64 Ax[size]
    (MatrixIO<io_formats::ELL>::write_matrix; FP64, one lane per row)."""
    if A.threads != 1:
        raise ValueError("the ELL file format stores one-lane layouts only")
    size = A.ncpr * A.stride
    with open(path, "wb") as f:
        np.array([size, A.rows, A.cols, A.stride, A.ncpr], np.uint64).tofile(f)
        np.asarray(A.Aj, np.uint64).tofile(f)
        np.asarray(A.Ax, np.float64).tofile(f)


def read_ell(path: str) -> EllMatrix:
    """Reads a binary ELL file (MatrixIO<io_formats::ELL>::read_matrix); Arl is recomputed from
    the first zero value of every row, as the reference's raw-array constructor does."""
    with open(path, "rb") as f:
        size, rows, cols, stride, ncpr = (int(v) for v in np.fromfile(f, np.uint64, 5))
        Aj = np.fromfile(f, np.uint64, size)
        Ax = np.fromfile(f, np.float64, size)
    nz = (Ax.reshape(ncpr, stride)[:, :rows] != 0)
    # row length = number of leading non-zero slots
    first_zero = np.where(nz.all(axis=0), ncpr, np.argmin(nz, axis=0))
    Arl = first_zero.astype(np.uint64)
    return EllMatrix(rows, cols, stride, ncpr, 1, Aj, Ax, Arl, int(Arl.sum()))


def write_exp(path: str, v) -> None:
    """EXP vector file: a '#' header line, then one value per line (VectorIO<io_formats::EXP>)."""
    with open(path, "w") as f:
        f.write("# honei_b200 vector\n")
        for x in np.asarray(v, np.float64):
            f.write(repr(float(x)) + "\n")
