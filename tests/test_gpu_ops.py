"""GPU parity of the operators against the oracle (bit-exact where the reference is per-row or
elementwise; fixed-order tree reductions within 1e-13 / 1e-5 relative of the sequential
reference sum).  All calls go through libhonei_b200.so's C ABI."""
import numpy as np
import pytest

from conftest import golden_matrix, load_golden
from honei_b200 import problems as P

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return la


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def spmv_gpu(hb, A, x):
    Ad = hb.SparseMatrixELL.from_reference(A)
    y = torch.full((A.rows,), np.nan, dtype=Ad.dtype, device="cuda")
    hb.Product.value(y, Ad, dev(x))
    return host(y)


CASES = [
    ("q1_33", lambda: P.q1_poisson(33)),
    ("q1_5_ragged", lambda: P.q1_poisson(5)),
    ("q1_7_ragged", lambda: P.q1_poisson(7)),
    ("q1_257", lambda: P.q1_poisson(257)),
    ("q1_257_varcoef", lambda: P.q1_poisson(257, P.log_uniform_coef(257, 1e-2, 1e2, 5))),
    ("q1_257_permuted", lambda: P.q1_poisson_permuted(257, 11)[0]),
    ("q1_65_threads2", lambda: P.ell_from_csr(4225, 4225, *P.q1_poisson_csr(65), threads=2)),
    ("q1_65_threads3", lambda: P.ell_from_csr(4225, 4225, *P.q1_poisson_csr(65), threads=3)),
    ("q1_65_threads16", lambda: P.ell_from_csr(4225, 4225, *P.q1_poisson_csr(65), threads=16)),
    ("prolongation_33", lambda: P.mg_hierarchy(33).prol[-1]),
    ("restriction_33", lambda: P.mg_hierarchy(33).res[-1]),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_spmv_bit_exact(hb, oracle, name, make, dtype):
    A = make().astype(dtype)
    x = P.uniform_vector(A.cols, 17).astype(dtype)
    assert np.array_equal(spmv_gpu(hb, A, x), oracle.spmv(A, x))


def test_spmv_featflow_matrices_bit_exact(hb, oracle, featflow):
    """Unstructured FEATFLOW2 matrices (up to 11 entries per row: runtime-K kernel path)."""
    H, d = featflow
    for A in H.A + H.prol + H.res:
        x = P.uniform_vector(A.cols, A.rows)
        assert np.array_equal(spmv_gpu(hb, A, x), oracle.spmv(A, x))
    A4 = H.A[-1]
    assert np.array_equal(spmv_gpu(hb, A4, d["spmv_x"]), d["spmv_y"])   # the reference's own output


def test_defect_bit_exact(hb, oracle, featflow):
    H, d = featflow
    A4 = H.A[-1]
    Ad = hb.SparseMatrixELL.from_reference(A4)
    r = torch.empty(A4.rows, dtype=torch.float64, device="cuda")
    hb.Defect.value(r, dev(d["rhs_4"]), Ad, dev(d["spmv_x"]))
    assert np.array_equal(host(r), d["defect_r"])
    d5 = load_golden("defect_5pt")
    A5 = golden_matrix(d5, "A")
    Ad5 = hb.SparseMatrixELL.from_reference(A5)
    r = torch.empty(A5.rows, dtype=torch.float64, device="cuda")
    hb.Defect.value(r, dev(d5["b"]), Ad5, dev(d5["x"]))
    assert np.array_equal(host(r), d5["r"])
    for dtype in (np.float64, np.float32):
        A = P.q1_poisson(129, P.log_uniform_coef(129, 1e-2, 1e2, 2)).astype(dtype)
        b = P.uniform_vector(A.rows, 3).astype(dtype)
        x = P.uniform_vector(A.rows, 4).astype(dtype)
        Ad = hb.SparseMatrixELL.from_reference(A)
        r = torch.empty(A.rows, dtype=Ad.dtype, device="cuda")
        hb.Defect.value(r, dev(b), Ad, dev(x))
        assert np.array_equal(host(r), oracle.defect(A, b, x))


def test_spmv_unaligned_output_and_size_errors(hb, oracle):
    A = P.q1_poisson(33)
    x = P.uniform_vector(A.rows, 1)
    Ad = hb.SparseMatrixELL.from_reference(A)
    buf = torch.zeros(A.rows + 1, dtype=torch.float64, device="cuda")
    y = buf[1:]                      # 8-byte aligned only: scalar store path
    hb.Product.value(y, Ad, dev(x))
    assert np.array_equal(host(y), oracle.spmv(A, x))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(torch.zeros(A.rows - 1, dtype=torch.float64, device="cuda"), Ad, dev(x))
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(buf, Ad, dev(x))
    with pytest.raises(TypeError):
        hb.Product.value(torch.zeros(A.rows, dtype=torch.float32, device="cuda"), Ad, dev(x))


def test_empty_matrix(hb):
    A = P.ell_from_csr(0, 0, np.zeros(1, np.int64), np.zeros(0, np.int64), np.zeros(0))
    Ad = hb.SparseMatrixELL.from_reference(A)
    y = torch.zeros(0, dtype=torch.float64, device="cuda")
    hb.Product.value(y, Ad, y)
    assert hb.DotProduct.value(y, y) == 0.0


def test_import_rejects_out_of_range_columns(hb):
    A = P.q1_poisson(9)
    A.Aj[5] = A.cols + 3
    with pytest.raises(Exception) as ei:
        hb.SparseMatrixELL.from_reference(A)
    assert getattr(ei.value, "status", None) == 1


@pytest.mark.parametrize("symmetric", [False, True])
def test_device_q1_assembly_matches_host_generator(hb, oracle, symmetric):
    for M, coef in ((3, None), (33, None), (257, P.log_uniform_coef(257, 1e-2, 1e2, 9))):
        Ah = P.q1_poisson(M, coef, symmetric=symmetric)
        Ad = hb.SparseMatrixELL.q1_poisson(M, None if coef is None else dev(coef.ravel()), symmetric=symmetric)
        Ai = hb.SparseMatrixELL.from_reference(Ah)
        # the device kernel always lays out K = 9 slots; the host packing may need fewer
        K = Ai.K
        assert Ad.ld == Ai.ld and K <= Ad.K
        assert torch.equal(Ad.Aj[: K * Ad.ld], Ai.Aj) and torch.equal(Ad.Ax[: K * Ad.ld], Ai.Ax)
        assert bool((Ad.Aj[K * Ad.ld:] == -1).all()) and bool((Ad.Ax[K * Ad.ld:] == 0).all())
        x = P.uniform_vector(M * M, 2)
        y = torch.empty(M * M, dtype=torch.float64, device="cuda")
        hb.Product.value(y, Ad, dev(x))
        assert np.array_equal(host(y), oracle.spmv(Ah, x))


def test_spmv_full_size_2049_bit_exact(hb, oracle):
    """The bench workload itself (2049^2, 37.7M nonzeros), FP64 and FP32, natural and permuted."""
    M = 2049
    Ad = hb.SparseMatrixELL.q1_poisson(M)
    A = P.q1_poisson(M)
    x = P.uniform_vector(A.rows, 5)
    y = torch.empty(A.rows, dtype=torch.float64, device="cuda")
    hb.Product.value(y, Ad, dev(x))
    assert np.array_equal(host(y), oracle.spmv(A, x))
    A32d = Ad.to_float()
    y32 = torch.empty(A.rows, dtype=torch.float32, device="cuda")
    x32 = x.astype(np.float32)
    hb.Product.value(y32, A32d, dev(x32))
    assert np.array_equal(host(y32), oracle.spmv(A.astype(np.float32), x32))


def test_dot_norm_tolerance(hb, oracle):
    import math
    for n in (1, 3, 1000, 66049, 4198401):
        x = P.uniform_vector(n, 1)
        y = P.uniform_vector(n, 2)
        exact = math.fsum(x * y)       # products are exact enough here; reference is sequential
        g = hb.DotProduct.value(dev(x), dev(y))
        ref = oracle.dot(x, y)
        scale = math.fsum(np.abs(x * y))
        assert abs(g - ref) <= 1e-13 * scale + 1e-300, (n, g, ref, exact)
        nn = hb.Norm.value(dev(x), root=False)
        assert abs(nn - oracle.dot(x, x)) <= 1e-13 * oracle.dot(x, x)
        assert abs(hb.Norm.value(dev(x), root=True) - math.sqrt(oracle.dot(x, x))) <= 1e-13 * math.sqrt(oracle.dot(x, x))
        x32, y32 = x.astype(np.float32), y.astype(np.float32)
        g32 = hb.DotProduct.value(dev(x32), dev(y32))
        s32 = math.fsum(np.abs(x32.astype(np.float64) * y32))
        e32 = math.fsum(x32.astype(np.float64) * y32)
        assert abs(g32 - e32) <= 1e-5 * s32 + 1e-30


def test_dot_deterministic(hb):
    x = dev(P.uniform_vector(1_000_003, 8))
    vals = {hb.DotProduct.value(x, x) for _ in range(5)}
    assert len(vals) == 1


def test_elementwise_bit_exact(hb, oracle):
    n = 100_003
    for dtype in (np.float64, np.float32):
        x = P.uniform_vector(n, 1).astype(dtype)
        y = P.uniform_vector(n, 2).astype(dtype)
        b = dtype(0.37)
        tx = dev(x.copy())
        hb.ScaledSum.value(tx, dev(y), float(b))
        assert np.array_equal(host(tx), x + b * y)
        r = torch.empty(n, dtype=tx.dtype, device="cuda")
        hb.ScaledSum.value(r, dev(x), dev(y), float(b))
        assert np.array_equal(host(r), b * y + x)
        tx = dev(x.copy())
        hb.Scale.value(tx, float(b))
        assert np.array_equal(host(tx), x * b)
        tx = dev(x.copy())
        hb.Sum.value(tx, dev(y))
        assert np.array_equal(host(tx), x + y)
        hb.Difference.value(r, dev(x), dev(y))
        assert np.array_equal(host(r), x - y)
        hb.ElementProduct.value(r, dev(x), dev(y))
        assert np.array_equal(host(r), x * y)
    x = P.uniform_vector(n, 3)
    f = torch.empty(n, dtype=torch.float32, device="cuda")
    hb.convert(f, dev(x))
    assert np.array_equal(host(f), x.astype(np.float32))
    d = torch.empty(n, dtype=torch.float64, device="cuda")
    hb.convert(d, f)
    assert np.array_equal(host(d), x.astype(np.float32).astype(np.float64))
