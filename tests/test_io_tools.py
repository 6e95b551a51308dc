"""The matrix file converters (honei_b200.io_tools): MatrixMarket -> ELL against the reference's
own MatrixIO<MTX> -> SparseMatrixELL path, ELL -> MatrixMarket and ellinfo round trips."""
import numpy as np

from honei_b200 import io_tools as T
from honei_b200 import problems as P


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)


def _random_mtx(path, n, seed, symmetric=False, with_zero=True):
    rng = np.random.default_rng(seed)
    lines = ["%%MatrixMarket matrix coordinate real " + ("symmetric" if symmetric else "general"),
             "% a comment line", f"{n} {n} 0"]
    for _ in range(4 * n):
        r, c = rng.integers(1, n + 1, 2)
        if symmetric and c > r:
            r, c = c, r
        lines.append(f"{r} {c} {rng.uniform(-2, 2):.17g}")
    if with_zero:
        lines.append(f"1 1 0")            # an explicit zero (dropped by the ELL constructor)
    lines.append(f"{n} {n} 3.5")
    _write(path, "\n".join(lines) + "\n")


def test_mtxtoell_matches_reference(tmp_path, reference):
    for k, sym in enumerate((False, True)):
        src = str(tmp_path / f"m{k}.mtx")
        _random_mtx(src, 37, k, symmetric=sym)
        A = T.mtxtoell(src, str(tmp_path / f"m{k}.ell"))
        R = reference.read_mtx(src)
        assert (A.rows, A.cols, A.stride, A.ncpr) == (R.rows, R.cols, R.stride, R.ncpr)
        assert np.array_equal(A.Aj, R.Aj) and np.array_equal(A.Ax, R.Ax)
        # the written file reads back through the reference's ELL reader unchanged
        B = reference.read_ell(str(tmp_path / f"m{k}.ell"))
        assert np.array_equal(B.Ax, R.Ax) and np.array_equal(B.Aj, R.Aj)


def test_mtx_quirks(tmp_path):
    src = str(tmp_path / "q.mtx")
    # duplicate positions: the later entry wins; a missing value reads as 0; a last line without
    # a line break is not read
    _write(src, "%%MatrixMarket matrix coordinate real general\n3 3 4\n1 1 2\n1 1 5\n2 2\n3 3 7")
    rows, cols, ip, ix, dv = T.read_mtx(src)
    assert (rows, cols) == (3, 3)
    d = {(r, int(ix[k])): dv[k] for r in range(rows) for k in range(ip[r], ip[r + 1])}
    assert d == {(0, 0): 5.0, (1, 1): 0.0}


def test_elltomtx_and_ellinfo_round_trip(tmp_path):
    A = P.q1_poisson(9, P.log_uniform_coef(9, 1e-1, 1e1, 1))
    ell = str(tmp_path / "a.ell")
    P.write_ell(ell, A)
    mtx = str(tmp_path / "a.mtx")
    T.elltomtx(ell, mtx)
    rows, cols, ip, ix, dv = T.read_mtx(mtx)
    ia, ja, va = A.to_csr()
    assert np.array_equal(ip, ia) and np.array_equal(ix, ja)
    assert np.allclose(dv, va, rtol=1e-5)          # six significant digits, as the reference prints
    info = T.ellinfo(ell)
    assert f"Rows: {A.rows}" in info and f"Non Zero Elements: {A.nnz}" in info
    assert T.main(["ellinfo", ell]) == 0 and T.main(["bogus"]) == 1
    assert T.main(["elltospai", ell]) == 1          # usage error, before any device work
