"""HONEI ELL files straight to and from the device (hb_ell_file_info, hb_ell_read_file_*,
hb_ell_write_file): the device import equals the import of the same arrays read on the host
(problems.read_ell follows the reference reader, pinned in test_oracle_pin), and what the device
writes reads back as the reference's own layout of the matrix."""
import numpy as np
import pytest

from conftest import golden_matrix, load_golden
from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


def same(a, b):
    return (a.rows(), a.columns(), a.K, a.ld) == (b.rows(), b.columns(), b.K, b.ld) and \
        torch.equal(a.Aj, b.Aj) and torch.equal(a.Ax, b.Ax)


@pytest.mark.parametrize("make", [lambda: P.q1_poisson(65, P.log_uniform_coef(65, 1e-2, 1e2, 2)),
                                  lambda: golden_matrix(load_golden("featflow_pa4"), "A_4"),
                                  lambda: P.q1_poisson_permuted(33, 5)[0]])
def test_read_file_matches_host_import(hb, tmp_path, make):
    A = make()
    path = str(tmp_path / "a.ell")
    P.write_ell(path, A)
    H = P.read_ell(path)
    d64 = hb.SparseMatrixELL.read_file(path)
    assert same(d64, hb.SparseMatrixELL.from_reference(H))
    d32 = hb.SparseMatrixELL.read_file(path, torch.float32)
    assert same(d32, hb.SparseMatrixELL.from_reference(H.astype(np.float32)))


def test_row_ends_at_first_zero_value(hb, tmp_path):
    """A zero value inside a row ends it, as the reference's raw-array constructor counts."""
    A = P.q1_poisson(9)
    Ax = A.Ax.copy().reshape(A.ncpr, A.stride)
    Ax[3, 40] = 0.0                       # row 40 keeps its first three slots only
    B = P.EllMatrix(A.rows, A.cols, A.stride, A.ncpr, 1, A.Aj, Ax.ravel(), A.Arl, A.nnz)
    path = str(tmp_path / "z.ell")
    P.write_ell(path, B)
    H = P.read_ell(path)
    assert int(H.Arl[40]) == 3
    assert same(hb.SparseMatrixELL.read_file(path), hb.SparseMatrixELL.from_reference(H))


@pytest.mark.parametrize("M", [9, 64, 257])
def test_write_file_is_the_reference_layout(hb, tmp_path, M):
    coef = P.log_uniform_coef(M, 1e-1, 1e1, M)
    D = hb.SparseMatrixELL.q1_poisson(M, torch.from_numpy(coef.ravel()).cuda())
    path = str(tmp_path / "w.ell")
    D.write_file(path)
    H = P.read_ell(path)
    R = P.q1_poisson(M, coef)             # the reference construction's own layout
    assert (H.rows, H.cols, H.stride, H.ncpr) == (R.rows, R.cols, R.stride, R.ncpr)
    assert np.array_equal(H.Aj, R.Aj) and np.array_equal(H.Ax, R.Ax) and np.array_equal(H.Arl, R.Arl)
    # and back to the device unchanged
    assert same(hb.SparseMatrixELL.read_file(path), D)


def test_file_errors(hb, tmp_path):
    from honei_b200._lib import HBError
    with pytest.raises(HBError) as e:
        hb.SparseMatrixELL.read_file(str(tmp_path / "missing.ell"))
    assert e.value.status == 8
    A = P.q1_poisson(9)
    path = str(tmp_path / "t.ell")
    P.write_ell(path, A)
    with open(path, "rb") as f:
        data = f.read()
    with open(str(tmp_path / "short.ell"), "wb") as f:
        f.write(data[:-100])
    with pytest.raises(HBError) as e:
        hb.SparseMatrixELL.read_file(str(tmp_path / "short.ell"))
    assert e.value.status == 1
    bad = P.EllMatrix(A.rows, 10, A.stride, A.ncpr, 1, A.Aj, A.Ax, A.Arl, A.nnz)   # columns past 10
    P.write_ell(str(tmp_path / "bad.ell"), bad)
    with pytest.raises(HBError) as e:
        hb.SparseMatrixELL.read_file(str(tmp_path / "bad.ell"))
    assert e.value.status == 1
