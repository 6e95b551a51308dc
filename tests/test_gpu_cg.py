"""GPU parity of CGSolver<GPU, NONE> against the oracle (honei/math/cg.hh:63-133).

Tolerance (the solver bar): the iteration count within +-1 of the oracle's, the final true
relative residual ||b - A x|| / ||b|| within 1e-10 of the oracle's (both ~1e-8), and the
solutions equal to within the accuracy the stopping rule guarantees.  FP32 solves use the
FP32 bar: iterations within 2% + 1, residual matching to 1e-5 relative of ||b||.
The dot products are fixed-order trees on the GPU and sequential sums on tags::CPU, so the
iterates differ at round-off level; everything elementwise is bit-identical.
"""
import numpy as np
import pytest

from conftest import load_golden
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


def relres(oracle, A, b, x):
    r = oracle.defect(A, b, x)
    return np.linalg.norm(r) / np.linalg.norm(b)


def run_cg(hb, A, b, eps, max_iters=20000, x0=None):
    Ad = hb.SparseMatrixELL.from_reference(A)
    x = dev(np.zeros(A.rows, A.dtype) if x0 is None else x0.astype(A.dtype))
    used = hb.CGSolver.value(Ad, None, dev(b.astype(A.dtype)), x, max_iters, eps)
    torch.cuda.synchronize()
    return x.cpu().numpy(), used


CASES64 = [
    ("q1_33", lambda: P.q1_poisson(33)),
    ("q1_257", lambda: P.q1_poisson(257)),
    ("q1_129_varcoef", lambda: P.q1_poisson(129, P.log_uniform_coef(129, 1e-2, 1e2, 5))),
    ("q1_129_permuted", lambda: P.q1_poisson_permuted(129, 3)[0]),
    ("q1_65_threads4", lambda: P.ell_from_csr(4225, 4225, *P.q1_poisson_csr(65), threads=4)),
]


@pytest.mark.parametrize("name,make", CASES64, ids=[c[0] for c in CASES64])
def test_cg_f64_parity(hb, oracle, name, make):
    A = make()
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=20000)
    x_g, u_g = run_cg(hb, A, b, 1e-8)
    assert abs(u_g - u_o) <= 1, (u_g, u_o)
    rg, ro = relres(oracle, A, b, x_g), relres(oracle, A, b, x_o)
    assert abs(rg - ro) <= 1e-10, (rg, ro)
    assert np.linalg.norm(x_g - x_o) <= 1e-6 * np.linalg.norm(x_o)


def test_cg_257_matches_reference_fixture(hb, oracle):
    """The plain FP64 CG workload (257^2 Q1, x_true U[-1,1], x0 = 0, 1e-8): the reference's
    own iteration count from the golden fixture."""
    d = load_golden("q1_small")
    A = P.q1_poisson(257)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    x_g, u_g = run_cg(hb, A, b, 1e-8)
    assert abs(u_g - int(d["cg257_used"])) <= 1
    assert relres(oracle, A, b, x_g) < 1.2e-8


def test_cg_f32_parity(hb, oracle):
    """FP32 CG against the oracle's FP32 CG (tags::CPU order): iterations within +-1 (measured on
    B200: equal at 33^2, 65^2, 129^2 and 257^2, as are the reference's own tags::CPU::SSE and
    MultiCore::SSE); the final true residual, evaluated in FP64 from the FP32 iterates, within
    2 % of the oracle's -- the FP32 iterates themselves differ at FP32 rounding."""
    for M in (33, 129):
        A = P.q1_poisson(M).astype(np.float32)
        b = oracle.spmv(A, P.uniform_vector(A.rows, 1).astype(np.float32))
        x_o, u_o = oracle.cg(A, b, eps=1e-5, max_iters=20000)
        x_g, u_g = run_cg(hb, A, b, 1e-5)
        assert abs(u_g - u_o) <= 1, (u_g, u_o)
        r_o = relres(oracle, A.astype(np.float64), b.astype(np.float64), x_o.astype(np.float64))
        r_g = relres(oracle, A.astype(np.float64), b.astype(np.float64), x_g.astype(np.float64))
        print(M, u_g, u_o, r_g, r_o)
        assert abs(r_g - r_o) <= 0.02 * r_o, (r_g, r_o)


def test_cg_edge_cases(hb, oracle):
    A = P.q1_poisson(17)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 2))
    # max_iters bounds the loop and is reported as used
    x_g, u_g = run_cg(hb, A, b, 1e-12, max_iters=7)
    x_o, u_o = oracle.cg(A, b, eps=1e-12, max_iters=7)
    assert u_g == u_o == 7
    assert np.linalg.norm(x_g - x_o) <= 1e-12 * np.linalg.norm(x_o)
    # zero right-hand side: the absolute test fires after one iteration, x stays 0
    x_g, u_g = run_cg(hb, A, np.zeros(A.rows), 1e-8)
    x_o, u_o = oracle.cg(A, np.zeros(A.rows), eps=1e-8)
    assert u_g == u_o and np.array_equal(x_g, x_o)
    # max_iters = 0: no iteration, x unchanged
    x0 = P.uniform_vector(A.rows, 3)
    x_g, u_g = run_cg(hb, A, b, 1e-8, max_iters=0, x0=x0)
    assert u_g == 0 and np.array_equal(x_g, x0)
    # non-zero start vector
    x_g, u_g = run_cg(hb, A, b, 1e-8, x0=x0)
    x_o, u_o = oracle.cg(A, b, x0=x0, eps=1e-8)
    assert abs(u_g - u_o) <= 1
    # tiny systems (one block, ragged row count)
    for M in (2, 3, 5):
        A = P.q1_poisson(M)
        b = oracle.spmv(A, P.uniform_vector(A.rows, M))
        x_g, u_g = run_cg(hb, A, b, 1e-8, max_iters=2000)
        x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=2000)
        assert abs(u_g - u_o) <= 1 and np.allclose(x_g, x_o, rtol=0, atol=1e-12)
    # an inconsistent right-hand side on the non-symmetric 5x5 system stagnates: both stop at
    # max_iters and report it
    A = P.q1_poisson(5)
    b = P.uniform_vector(A.rows, 5)
    assert run_cg(hb, A, b, 1e-8, max_iters=300)[1] == oracle.cg(A, b, eps=1e-8, max_iters=300)[1] == 300


def test_cg_deterministic(hb, oracle):
    A = P.q1_poisson(129)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    xs = [run_cg(hb, A, b, 1e-8) for _ in range(3)]
    assert all(np.array_equal(xs[0][0], x) and xs[0][1] == u for x, u in xs)


def test_cg_size_mismatch_raises(hb):
    A = hb.SparseMatrixELL.q1_poisson(9)
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.CGSolver.value(A, None, torch.zeros(80, dtype=torch.float64, device="cuda"),
                          torch.zeros(81, dtype=torch.float64, device="cuda"), 10)


def test_cg_full_size_1025_property(hb):
    """At 1025^2 (configs' CG size) the oracle takes minutes: check size-independent properties
    instead -- convergence to the stated relative residual, measured with the GPU's own
    (bit-exact) defect, and reproducibility."""
    M = 1025
    Ad = hb.SparseMatrixELL.q1_poisson(M)
    xt = dev(P.uniform_vector(M * M, 1))
    b = torch.empty_like(xt)
    hb.Product.value(b, Ad, xt)
    x = torch.zeros_like(xt)
    used = hb.CGSolver.value(Ad, None, b, x, 20000, 1e-8)
    r = torch.empty_like(xt)
    hb.Defect.value(r, b, Ad, x)
    rel = hb.Norm.value(r, root=True) / hb.Norm.value(b, root=True)
    assert used < 20000 and rel < 1.5e-8
    x2 = torch.zeros_like(xt)
    assert hb.CGSolver.value(Ad, None, b, x2, 20000, 1e-8) == used and torch.equal(x, x2)


@pytest.mark.parametrize("M,coef", [(3, False), (9, False), (17, True), (31, True)])
def test_cg_small_systems_bitwise_equal_to_cooperative_kernel(hb, oracle, M, coef):
    """Systems of at most 1024 rows run in the one-block kernel; the cooperative kernel (the
    allocation-free entry point always uses it) must give the same iterates bit for bit,
    also on the non-symmetric 9^2 coarse matrix whose CG runs to the iteration cap."""
    import ctypes as C
    from honei_b200._lib import lib
    A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, M) if coef else None)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 2))
    Ad = hb.SparseMatrixELL.from_reference(A)
    bd = dev(b)
    x1, x2 = torch.zeros_like(bd), torch.zeros_like(bd)
    u1 = hb.CGSolver.value(Ad, None, bd, x1, 1000, 1e-8)
    d1 = hb.CGSolver.last_defect
    u2, d2 = C.c_int64(0), C.c_double(0)
    st = lib().hb_cg_f64_noalloc(C.byref(Ad.struct), bd.data_ptr(), x2.data_ptr(), 1000, 1e-8, C.byref(u2),
                                 C.byref(d2), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == 0 and u1 == u2.value and d1 == d2.value
    assert torch.equal(x1, x2)
    x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=1000)
    assert abs(u1 - u_o) <= 1


RESIDENT_CASES = [
    ("q1_257", lambda: P.q1_poisson(257)),
    ("q1_129_varcoef", lambda: P.q1_poisson(129, P.log_uniform_coef(129, 1e-2, 1e2, 5))),
    # a random permutation spreads each block's columns past its window: the out-of-window path
    ("q1_257_permuted", lambda: P.q1_poisson_permuted(257, 4)[0]),
    ("q1_65_threads4", lambda: P.ell_from_csr(4225, 4225, *P.q1_poisson_csr(65), threads=4)),
]


@pytest.mark.parametrize("name,make", RESIDENT_CASES, ids=[c[0] for c in RESIDENT_CASES])
def test_cg_resident_kernel_matches_streaming_kernel(hb, oracle, name, make):
    """Systems that fit run in the resident-operator kernel by default; the streaming kernel
    solves the same system to the same bar (iterations within 1, the true residual within
    1e-10), and each kernel is deterministic."""
    A = make()
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    x_r, u_r = run_cg(hb, A, b, 1e-8)
    x_r2, u_r2 = run_cg(hb, A, b, 1e-8)
    assert u_r == u_r2 and np.array_equal(x_r, x_r2)
    prev = hb.CGSolver.set_resident(False)
    try:
        x_s, u_s = run_cg(hb, A, b, 1e-8)
    finally:
        hb.CGSolver.set_resident(prev)
    assert prev is True
    assert abs(u_r - u_s) <= 1, (u_r, u_s)
    assert abs(relres(oracle, A, b, x_r) - relres(oracle, A, b, x_s)) <= 1e-10
    assert np.linalg.norm(x_r - x_s) <= 1e-6 * np.linalg.norm(x_s)


def test_cg_resident_kernel_edge_cases(hb, oracle):
    """The resident kernel (65^2: 34 blocks of 125 rows) on the loop's edges: max_iters = 0,
    a cap that stops the loop, a zero right-hand side, a non-zero start vector, FP32."""
    A = P.q1_poisson(65)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 2))
    x0 = P.uniform_vector(A.rows, 3)
    x_g, u_g = run_cg(hb, A, b, 1e-8, max_iters=0, x0=x0)
    assert u_g == 0 and np.array_equal(x_g, x0)
    x_g, u_g = run_cg(hb, A, b, 1e-12, max_iters=7)
    x_o, u_o = oracle.cg(A, b, eps=1e-12, max_iters=7)
    assert u_g == u_o == 7 and np.linalg.norm(x_g - x_o) <= 1e-12 * np.linalg.norm(x_o)
    x_g, u_g = run_cg(hb, A, np.zeros(A.rows), 1e-8)
    x_o, u_o = oracle.cg(A, np.zeros(A.rows), eps=1e-8)
    assert u_g == u_o and np.array_equal(x_g, x_o)
    x_g, u_g = run_cg(hb, A, b, 1e-8, x0=x0)
    x_o, u_o = oracle.cg(A, b, x0=x0, eps=1e-8)
    assert abs(u_g - u_o) <= 1 and abs(relres(oracle, A, b, x_g) - relres(oracle, A, b, x_o)) <= 1e-10
    A32 = P.q1_poisson(257).astype(np.float32)
    b32 = oracle.spmv(A32, P.uniform_vector(A32.rows, 1).astype(np.float32))
    x_o, u_o = oracle.cg(A32, b32, eps=1e-5, max_iters=20000)
    x_g, u_g = run_cg(hb, A32, b32, 1e-5)
    assert abs(u_g - u_o) <= 1, (u_g, u_o)
    r_o = relres(oracle, A32.astype(np.float64), b32.astype(np.float64), x_o.astype(np.float64))
    r_g = relres(oracle, A32.astype(np.float64), b32.astype(np.float64), x_g.astype(np.float64))
    print(u_g, u_o, r_g, r_o)
    assert abs(r_g - r_o) <= 0.02 * r_o, (r_g, r_o)


def test_cg_concurrent_solves_on_separate_contexts(hb):
    """Four host threads, each with its own context and stream, solve systems of different sizes
    (and so different resident-kernel plans) at the same time.  Every solve succeeds and is
    bit-identical to the same solve run alone; no failure leaks into the caller's CUDA state."""
    import threading
    sizes = (257, 129, 257, 513)

    def solve(M, seed, ctx=None, stream=None):
        A = hb.SparseMatrixELL.q1_poisson(M, ctx=ctx)
        xt = dev(P.uniform_vector(M * M, seed))
        b = torch.empty_like(xt)
        hb.Product.value(b, A, xt, ctx=ctx)
        x = torch.zeros_like(xt)
        used = hb.CGSolver.value(A, None, b, x, 100000, 1e-8, ctx=ctx)
        (stream or torch.cuda.current_stream()).synchronize()
        return used, x.cpu().numpy()

    alone = [solve(M, k + 1) for k, M in enumerate(sizes)]
    results, errors = {}, []

    def worker(k, M):
        try:
            ctx = hb.Context(0)
            s = torch.cuda.Stream()
            ctx.bind_stream(s)
            with torch.cuda.stream(s):
                results[k] = [solve(M, k + 1, ctx, s) for _ in range(3)]
        except Exception as e:    # reported below, in the test's thread
            errors.append((k, repr(e)))

    threads = [threading.Thread(target=worker, args=(k, M)) for k, M in enumerate(sizes)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    torch.cuda.synchronize()
    for k in range(len(sizes)):
        for used, x in results[k]:
            assert used == alone[k][0] and np.array_equal(x, alone[k][1]), k


@pytest.mark.parametrize("name,make", RESIDENT_CASES[:2] + [("q1_513", lambda: P.q1_poisson(513))],
                         ids=[c[0] for c in RESIDENT_CASES[:2]] + ["q1_513"])
def test_cg_row_layout_matches_group_layout(hb, oracle, name, make):
    """The streaming kernel with one row per thread solves the same systems to the CG bar
    (iterations within 1 of the four-row layout's and of the oracle's, true residual within
    1e-10), deterministically."""
    A = make()
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    prev_res = hb.CGSolver.set_resident(False)
    try:
        prev = hb.CGSolver.set_layout(4)
        x4, u4 = run_cg(hb, A, b, 1e-8)
        hb.CGSolver.set_layout(1)
        x1, u1 = run_cg(hb, A, b, 1e-8)
        x1b, u1b = run_cg(hb, A, b, 1e-8)
        hb.CGSolver.set_layout(prev)
    finally:
        hb.CGSolver.set_resident(prev_res)
    assert u1 == u1b and np.array_equal(x1, x1b)
    assert abs(u1 - u4) <= 1, (u1, u4)
    assert abs(relres(oracle, A, b, x1) - relres(oracle, A, b, x4)) <= 1e-10
    if A.rows <= 129 * 129:
        x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=20000)
        assert abs(u1 - u_o) <= 1 and abs(relres(oracle, A, b, x1) - relres(oracle, A, b, x_o)) <= 1e-10
    with pytest.raises(ValueError):
        hb.CGSolver.set_layout(3)
