"""GPU parity of the SparseMatrixCSR product and defect (Product / Defect<tags::GPU::CUDA> on
SparseMatrixCSR, honei/la/product.hh:1762-1764, honei/math/defect.hh:673-676) against the
oracle, which restates tags::CPU (honei/la/product.hh:209-242, honei/math/defect.hh:386-419).

Bar: bit-exact.  Every row is summed by one thread in the reference's order (blocks, then the
csr::blocksize lanes of each block, lanes whose column is not below cols skipped), FP32 and
FP64 alike.  At the full 2049^2 size the size-independent property is used instead of the
oracle: the blocksize-1 CSR of a matrix sums each row in the same (ascending column) order as
its ELL form, so the two products agree bit for bit.
"""
import numpy as np
import pytest

from conftest import golden_csr, load_golden
from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_spmv(hb, A, x):
    Ad = hb.SparseMatrixCSR.from_reference(A)
    y = torch.full((A.rows,), float("nan"), dtype=Ad.dtype, device="cuda")
    hb.Product.value(y, Ad, dev(x.astype(A.dtype)))
    return y.cpu().numpy()


def gpu_defect(hb, A, b, x):
    Ad = hb.SparseMatrixCSR.from_reference(A)
    r = torch.full((A.rows,), float("nan"), dtype=Ad.dtype, device="cuda")
    hb.Defect.value(r, dev(b.astype(A.dtype)), Ad, dev(x.astype(A.dtype)))
    return r.cpu().numpy()


def random_csr(rng, rows, cols, fill, bs, dtype=np.float64, empty_frac=0.2):
    mask = rng.random((rows, cols)) < fill
    if rows > 4:
        mask[rng.choice(rows, int(rows * empty_frac), replace=False)] = False
    ri, ci = np.nonzero(mask)
    ip = np.zeros(rows + 1, np.int64)
    np.cumsum(np.bincount(ri, minlength=rows), out=ip[1:])
    return P.csr_blocked(rows, cols, ip, ci, rng.uniform(-1, 1, len(ci)), bs, dtype)


def test_csr_matches_reference_fixture(hb):
    """The reference's own CSR product test cases (csr::blocksize 1..8, size x (size + 3)), the
    Q1 33^2 ELL -> CSR conversion with product and defect, and a random rectangular pattern."""
    g = load_golden("csr")
    for bs in (1, 2, 4, 8):
        for size in (11, 44, 176):
            k = f"t{bs}_{size}"
            assert np.array_equal(gpu_spmv(hb, golden_csr(g, k), g[k + "_x"]), g[k + "_y"]), k
    for bs in (1, 4):
        k = f"q1_{bs}"
        A = golden_csr(g, k)
        assert np.array_equal(gpu_spmv(hb, A, g[k + "_x"]), g[k + "_y"]), k
        assert np.array_equal(gpu_defect(hb, A, g[k + "_b"], g[k + "_x"]), g[k + "_r"]), k
    for bs in (1, 3, 8):
        k = f"rand_{bs}"
        A = golden_csr(g, k)
        assert np.array_equal(gpu_spmv(hb, A, g[k + "_x"]), g[k + "_y"]), k
        assert np.array_equal(gpu_spmv(hb, A.astype(np.float32), g[k + "_x"].astype(np.float32)), g[k + "_y32"])


@pytest.mark.parametrize("bs", [1, 2, 3, 5, 8, 16, 64, 256, 300])
def test_csr_random_patterns_bitwise(hb, oracle, bs):
    """Square and rectangular, sparse and dense rows, empty rows, rows % 32 != 0; blocksizes up
    to the staged limit (256) and beyond it (the one-thread-per-row path)."""
    rng = np.random.default_rng(bs)
    for rows, cols, fill in ((1, 1, 1.0), (31, 700, 0.3), (33, 33, 0.5), (1000, 517, 0.01), (4097, 4097, 0.002)):
        for dt in (np.float64, np.float32):
            A = random_csr(rng, rows, cols, fill, bs, dt)
            x = rng.uniform(-1, 1, cols).astype(dt)
            b = rng.uniform(-1, 1, rows).astype(dt)
            assert np.array_equal(gpu_spmv(hb, A, x), oracle.csr_spmv(A, x)), (rows, cols, bs, dt)
            assert np.array_equal(gpu_defect(hb, A, b, x), oracle.csr_defect(A, b, x)), (rows, cols, bs, dt)


def test_csr_edge_cases(hb, oracle):
    rng = np.random.default_rng(7)
    # a row far longer than a staging chunk, surrounded by short rows
    rows, cols = 70, 20000
    ip = np.zeros(rows + 1, np.int64)
    lens = np.full(rows, 3)
    lens[33] = 9000
    np.cumsum(lens, out=ip[1:])
    ci = np.concatenate([np.sort(rng.choice(cols, n, replace=False)) for n in lens])
    for bs in (1, 4):
        A = P.csr_blocked(rows, cols, ip, ci, rng.uniform(-1, 1, len(ci)), bs)
        x = rng.uniform(-1, 1, cols)
        assert np.array_equal(gpu_spmv(hb, A, x), oracle.csr_spmv(A, x)), bs
    # no stored entry at all: y = 0; a matrix with rows but no columns
    A = P.csr_blocked(40, 10, np.zeros(41, np.int64), np.zeros(0, np.int64), np.zeros(0), 2)
    assert np.array_equal(gpu_spmv(hb, A, np.ones(10)), np.zeros(40))
    A = P.csr_blocked(5, 0, np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0), 1)
    assert np.array_equal(gpu_spmv(hb, A, np.zeros(0)), np.zeros(5))
    # a block that starts at or beyond cols (its lanes all skipped) and one that straddles cols
    A = P.CsrMatrix(3, 10, 4, np.array([0, 2, 3, 4], np.uint64), np.array([8, 12, 4, 1 << 40], np.uint64),
                    rng.uniform(-1, 1, 16), 9)
    x = rng.uniform(-1, 1, 10)
    assert np.array_equal(gpu_spmv(hb, A, x), oracle.csr_spmv(A, x))
    # an offset array that is not one is refused at import (checked on the device)
    from honei_b200._lib import HBError
    bad = P.CsrMatrix(3, 3, 1, np.array([0, 2, 1, 3], np.uint64), np.array([0, 1, 2], np.uint64), np.ones(3), 3)
    with pytest.raises(HBError):
        hb.SparseMatrixCSR.from_reference(bad)
    # size checks before any launch
    Ad = hb.SparseMatrixCSR.from_reference(random_csr(rng, 8, 6, 0.5, 1))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(torch.zeros(8, dtype=torch.float64, device="cuda"), Ad,
                         torch.zeros(8, dtype=torch.float64, device="cuda"))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Defect.value(torch.zeros(8, dtype=torch.float64, device="cuda"),
                        torch.zeros(6, dtype=torch.float64, device="cuda"), Ad,
                        torch.zeros(6, dtype=torch.float64, device="cuda"))


def test_csr_2049_equals_ell_product(hb):
    """Full size (Q1 2049^2, 4.2M rows, 37.7M entries), FP64 and FP32: the blocksize-1 CSR
    product equals the ELL product of the same matrix bit for bit."""
    E = P.q1_poisson(2049)
    C = P.csr_from_ell(E, 1)
    x = P.uniform_vector(E.rows, 3)
    for dt in (np.float64, np.float32):
        Ed = hb.SparseMatrixELL.from_reference(E.astype(dt))
        Cd = hb.SparseMatrixCSR.from_reference(C.astype(dt))
        xd = dev(x.astype(dt))
        y1 = torch.empty_like(xd)
        y2 = torch.empty_like(xd)
        hb.Product.value(y1, Ed, xd)
        hb.Product.value(y2, Cd, xd)
        assert torch.equal(y1, y2), dt
        del Ed, Cd
        torch.cuda.empty_cache()
