"""BandedMatrixQx<Q1Type> on the device (hb_q1band_*): product, defect, Poisson fill and the
conversion from ELL, bit for bit against the oracle (itself pinned to the reference's
Product<tags::CPU>, Defect<tags::CPU>, FillMatrix and BandedMatrixQx(SparseMatrixELL &))."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, q1band_test_data, q1band_used_mask
from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TDT = {np.float64: torch.float64, np.float32: torch.float32}


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


def dev(a, dt=None):
    return torch.from_numpy(np.ascontiguousarray(a if dt is None else a.astype(dt))).cuda()


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_product_on_the_reference_test_data(hb, oracle, dt):
    """Q1MatrixDenseVectorProductTest's data (levels 1..8) and its golden results."""
    g = load_golden("q1band")
    name = "f64" if dt == np.float64 else "f32"
    for level in range(1, 9):
        size = (2 ** level + 1) ** 2
        bands, x = q1band_test_data(size, dt)
        A = hb.BandedMatrixQ1.from_bands(bands, TDT[dt])
        y = torch.empty(size, dtype=TDT[dt], device="cuda")
        hb.Product.value(y, A, dev(x))
        yg = y.cpu().numpy()
        assert np.array_equal(yg, oracle.q1band_spmv(bands, x)), level
        if level in (2, 5):
            assert np.array_equal(yg, g[f"test_L{level}_{name}_y"])


def _unaligned(hb, bands, dt):
    """A BandedMatrixQ1 whose bands start one element past a 16-byte boundary (scalar path)."""
    n = len(bands[0])
    t = torch.zeros((9, n + 1), dtype=TDT[dt], device="cuda")
    for k, b in enumerate(bands):
        t[k, 1:] = dev(b)
    A = hb.BandedMatrixQ1(n, t)
    for k in range(9):
        A.struct.band[k] = t[k, 1:].data_ptr()
    A._keep = t
    return A


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 9, 49, 50, 1000, 4225, 66049])
def test_product_and_defect_random(hb, oracle, dt, n):
    rng = np.random.default_rng(n)
    bands = [rng.uniform(-1, 1, n).astype(dt) for _ in range(9)]
    x = rng.uniform(-1, 1, n).astype(dt)
    b = rng.uniform(-1, 1, n).astype(dt)
    y_o = oracle.q1band_spmv(bands, x)
    r_o = oracle.q1band_defect(bands, b, x)
    for A in (hb.BandedMatrixQ1.from_bands(bands, TDT[dt]), _unaligned(hb, bands, dt)):
        y = torch.empty(n, dtype=TDT[dt], device="cuda")
        r = torch.empty_like(y)
        hb.Product.value(y, A, dev(x))
        hb.Defect.value(r, dev(b), A, dev(x))
        assert np.array_equal(y.cpu().numpy(), y_o)
        assert np.array_equal(r.cpu().numpy(), r_o)
    # unaligned vectors too (views one element in)
    A = hb.BandedMatrixQ1.from_bands(bands, TDT[dt])
    buf = torch.zeros(3 * (n + 1), dtype=TDT[dt], device="cuda")
    xv, bv, yv = buf[1:n + 1], buf[n + 2:2 * n + 2], buf[2 * n + 3:3 * n + 3]
    xv.copy_(dev(x))
    bv.copy_(dev(b))
    hb.Defect.value(yv, bv, A, xv)
    assert np.array_equal(yv.cpu().numpy(), r_o)


def test_defect_golden(hb):
    g = load_golden("q1band")
    A = hb.BandedMatrixQ1.from_bands(list(g["var_bands"]))
    r = torch.empty(A.rows(), dtype=torch.float64, device="cuda")
    hb.Defect.value(r, dev(g["var_b"]), A, dev(g["var_x"]))
    assert np.array_equal(r.cpu().numpy(), g["var_r64"])
    y = torch.empty_like(r)
    hb.Product.value(y, A, dev(g["var_x"]))
    assert np.array_equal(y.cpu().numpy(), g["var_y64"])


@pytest.mark.parametrize("M", [1, 2, 3, 9, 33, 100])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_fill_poisson(hb, oracle, M, dt):
    A = hb.BandedMatrixQ1.poisson(M, TDT[dt])
    assert A.root == M
    want = np.stack(oracle.q1band_poisson(M)).astype(dt)
    got = A.bands[:, : M * M].cpu().numpy()
    assert np.array_equal(got, want)
    if M == 33 and dt == np.float64:
        assert np.array_equal(got, load_golden("q1band")["poisson_bands"])


@pytest.mark.parametrize("M,coef", [(33, True), (65, False), (40, True)])
def test_from_ell(hb, oracle, M, coef):
    """Band k of row i = A(i, i + offset_k): checked against the reference's conversion (the
    golden bands at 33^2) and, for every size, against the CSR of the same matrix."""
    c = P.log_uniform_coef(M, 1e-2, 1e2, 4) if coef else None
    E = P.q1_poisson(M, c)
    A = hb.BandedMatrixQ1.from_ell(hb.SparseMatrixELL.from_reference(E))
    n = M * M
    got = A.bands[:, :n].cpu().numpy()
    ip, ix, dv = E.to_csr()
    offs = [-M - 1, -M, -M + 1, -1, 0, 1, M - 1, M, M + 1]
    want = np.zeros((9, n))
    for r in range(n):
        for j, v in zip(ix[ip[r]:ip[r + 1]], dv[ip[r]:ip[r + 1]]):
            d = int(j) - r
            if d in offs:
                want[offs.index(d), r] = v
    assert np.array_equal(got, want)
    if M == 33 and coef:
        mask = q1band_used_mask(n)
        assert np.array_equal(got[mask], load_golden("q1band")["var_bands"][mask])
    # the banded product of the converted matrix: the oracle's banded product
    x = P.uniform_vector(n, 1)
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    hb.Product.value(y, A, dev(x))
    assert np.array_equal(y.cpu().numpy(), oracle.q1band_spmv(list(want), x))


def test_errors(hb):
    from honei_b200._lib import HBError, lib
    A = hb.BandedMatrixQ1.poisson(9)
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(torch.empty(81, dtype=torch.float64, device="cuda"), A,
                         torch.empty(80, dtype=torch.float64, device="cuda"))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Defect.value(torch.empty(81, dtype=torch.float64, device="cuda"),
                        torch.empty(82, dtype=torch.float64, device="cuda"), A,
                        torch.empty(81, dtype=torch.float64, device="cuda"))
    with pytest.raises(TypeError):
        hb.Product.value(torch.empty(81, dtype=torch.float32, device="cuda"), A,
                         torch.empty(81, dtype=torch.float32, device="cuda"))
    # ELL with a non-square row count cannot become a Q1 banded matrix
    E = hb.SparseMatrixELL.from_reference(P.ell_from_csr(10, 10, np.arange(11), np.arange(10), np.ones(10)))
    with pytest.raises(HBError) as e:
        hb.BandedMatrixQ1.from_ell(E)
    assert e.value.status == 6
    # a wrong root is refused before any launch
    A.struct.root = 8
    st = lib().hb_q1band_spmv_f64(hb.default_context().handle, C.byref(A.struct),
                                  torch.zeros(81, dtype=torch.float64, device="cuda").data_ptr(),
                                  torch.zeros(81, dtype=torch.float64, device="cuda").data_ptr())
    assert st == 1


def test_full_size_2049(hb, oracle):
    """2049^2 Poisson: device fill + product bit for bit against the oracle, and against the
    ELL product of the same matrix to rounding (the two sum in different orders)."""
    M = 2049
    n = M * M
    A = hb.BandedMatrixQ1.poisson(M)
    x = P.uniform_vector(n, 3)
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    xd = dev(x)
    hb.Product.value(y, A, xd)
    yo = oracle.q1band_spmv(oracle.q1band_poisson(M), x)
    assert np.array_equal(y.cpu().numpy(), yo)
    E = hb.SparseMatrixELL.q1_poisson(M)
    ye = torch.empty_like(y)
    hb.Product.value(ye, E, xd)
    assert float((ye - y).abs().max()) <= 1e-14 * float(y.abs().max())
