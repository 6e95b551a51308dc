"""Matrix file converters of HONEI's clients/io_tools, for feeding external matrices to the
device path:

    python -m honei_b200.io_tools mtxtoell  matrix.mtx  matrix.ell   # clients/io_tools/mtxtoell.cc
    python -m honei_b200.io_tools elltomtx  matrix.ell  matrix.mtx   # clients/io_tools/elltomtx.cc
    python -m honei_b200.io_tools ellinfo   matrix.ell               # clients/io_tools/ellinfo.cc
    python -m honei_b200.io_tools elltospai matrix.ell  spai.ell     # clients/io_tools/elltospai.cc

MatrixMarket reading follows MatrixIO<io_formats::MTX>::read_matrix
(honei/math/matrix_io.hh:234-338): any line containing '%' is a comment (one that also contains
"symmetric" marks the file symmetric); the first other line gives "rows columns"; every further
line "row column value" (1-based; a missing value reads as 0); a symmetric file gets the mirror of
every off-diagonal entry; a later entry of the same position overwrites an earlier one
(SparseMatrix::operator()); a last line without a line break is not read, as the reference's
getline/eof loop skips it.  Entries of value 0 are dropped when the ELL matrix is built, as
SparseMatrixELL(SparseMatrix) does.  Writing follows write_matrix (matrix_io.hh:400-430): a
"coordinate real general" header, "rows columns nnz", then "row column value" with the value
printed as a C++ stream prints a double (six significant digits).  elltospai reads the file
straight to the device, builds SPAI2 there (bit-identical to the reference's
SPAI2<tags::CPU::MultiCore::SSE>, which computes what SPAI2<tags::CPU::SSE> does) and writes M in
the same one-lane layout; it needs a GPU.
"""
from __future__ import annotations

import sys

import numpy as np

from . import problems as P


def read_mtx(path: str):
    """(rows, cols, indptr, indices, data): the CSR of a MatrixMarket file, ascending columns."""
    with open(path, "r") as f:
        text = f.read()
    lines = text.split("\n")
    # the final piece is what follows the last line break: the reference never processes it
    lines = lines[:-1]
    symmetric = False
    rows = cols = None
    entries = {}
    for line in lines:
        if "%" in line:
            if "symmetric" in line:
                symmetric = True
            continue
        tok = line.split()
        if rows is None:
            rows, cols = int(tok[0]), int(tok[1])
            continue
        if len(tok) < 2:
            continue
        r, c = int(tok[0]) - 1, int(tok[1]) - 1
        v = float(tok[2]) if len(tok) > 2 else 0.0
        entries[(r, c)] = v
    if rows is None:
        raise ValueError(f"{path}: no size line")
    if symmetric:
        for (r, c), v in list(entries.items()):
            if r != c:
                entries[(c, r)] = v
    if entries:
        keys = sorted(entries)
        rr = np.array([k[0] for k in keys], np.int64)
        cc = np.array([k[1] for k in keys], np.int64)
        vv = np.array([entries[k] for k in keys], np.float64)
    else:
        rr = cc = np.zeros(0, np.int64)
        vv = np.zeros(0)
    indptr = np.zeros(rows + 1, np.int64)
    np.add.at(indptr, rr + 1, 1)
    np.cumsum(indptr, out=indptr)
    return rows, cols, indptr, cc, vv


def write_mtx(path: str, rows: int, cols: int, indptr, indices, data) -> None:
    indptr, indices, data = np.asarray(indptr), np.asarray(indices), np.asarray(data, np.float64)
    keep = data != 0
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{rows} {cols} {int(keep.sum())}\n")
        for r in range(rows):
            for k in range(indptr[r], indptr[r + 1]):
                if data[k] != 0:
                    f.write(f"{r + 1} {int(indices[k]) + 1} {data[k]:.6g}\n")


def mtxtoell(mtx: str, ell: str) -> P.EllMatrix:
    rows, cols, ip, ix, dv = read_mtx(mtx)
    A = P.ell_from_csr(rows, cols, ip, ix, dv, 1, np.float64)
    P.write_ell(ell, A)
    return A


def elltomtx(ell: str, mtx: str) -> None:
    A = P.read_ell(ell)
    write_mtx(mtx, A.rows, A.cols, *A.to_csr())


def ellinfo(ell: str) -> str:
    A = P.read_ell(ell)
    used = int(np.count_nonzero(A.Ax))
    return (f"ELL Matrix info for {ell}\nRows: {A.rows}\nColumns: {A.cols}\nNon Zero Elements: {used}\n"
            f"NumColsPerRow: {A.ncpr}, Stride: {A.stride}, Threads: {A.threads}\n")


def elltospai(ell: str, spai: str) -> None:
    """clients/io_tools/elltospai.cc: SPAI2 of the file's matrix (pattern of A), written as an
    ELL file (FP64)."""
    from . import la
    A = la.SparseMatrixELL.read_file(ell)
    la.SPAI2.value(A).write_file(spai)


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    usage = ("usage: python -m honei_b200.io_tools {mtxtoell MTX ELL | elltomtx ELL MTX | ellinfo ELL | "
             "elltospai ELL SPAI_ELL}")
    if not argv:
        print(usage)
        return 1
    cmd, args = argv[0], argv[1:]
    if cmd == "mtxtoell" and len(args) == 2:
        mtxtoell(*args)
    elif cmd == "elltomtx" and len(args) == 2:
        elltomtx(*args)
    elif cmd == "ellinfo" and len(args) == 1:
        sys.stdout.write(ellinfo(args[0]))
    elif cmd == "elltospai" and len(args) == 2:
        elltospai(*args)
    else:
        print(usage)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
