"""GPU parity of the MG V-cycle (MGSolver + RISmoother + PROLMAT transfers + CG coarse solve)
and of mixed-precision iterative refinement (IRSolver) against the oracle.

Bar: cycle / outer-step counts within +-1 of the oracle's; final relative residual matching
the oracle's (FP64: to 1e-10 of ||b||; FP32: to 1e-5); the FEATFLOW2 fixture solved to the
reference test's own tolerance against FEATFLOW's solution (8e-3, honei/math/mg_TEST.cc).
The smoother, defect, transfers and updates are bit-exact; only the norms and the coarse CG's
dot products are summed in a different (fixed) order.
"""
import numpy as np
import pytest

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


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def mg_gpu(hb, H, b, x0=None, dtype=np.float64, **kw):
    data = hb.MGData.from_hierarchy(H, dtype=dtype, **kw)
    n = H.A[-1].rows
    x = dev(np.zeros(n, dtype) if x0 is None else np.asarray(x0, dtype))
    used, r0, r1 = hb.MGSolver.value(data, dev(np.asarray(b, dtype)), x)
    out = host(x)
    data.close()
    return out, used, r0, r1


@pytest.mark.parametrize("M,coef_seed", [(17, None), (33, None), (129, None), (65, 4), (129, 6)])
def test_mg_f64_parity(hb, oracle, M, coef_seed):
    """Unit coefficient: rediscretised levels; cell coefficients 10^U(-1,1): Galerkin levels."""
    coef = None if coef_seed is None else P.log_uniform_coef(M, 1e-1, 1e1, coef_seed)
    H = P.mg_hierarchy(M, coef=coef)
    A = H.A[-1]
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    x_o, u_o, h_o = oracle.mg(H, b, eps=1e-8, history=True)
    x_g, u_g, r0, r1 = mg_gpu(hb, H, b, eps=1e-8)
    assert abs(u_g - u_o) <= 1, (u_g, u_o)
    nb = np.linalg.norm(b)
    rg = np.linalg.norm(oracle.defect(A, b, x_g)) / nb
    ro = np.linalg.norm(oracle.defect(A, b, x_o)) / nb
    assert abs(rg - ro) <= 1e-10, (rg, ro)
    assert abs(r0 - h_o[0]) <= 1e-13 * h_o[0]


def test_mg_one_cycle_bit_exact_with_exact_coarse(hb, oracle):
    """With a single level the V-cycle is the coarse CG; with two levels and no coarse
    iterations it is smoother + transfers only, which must be bit-exact."""
    H = P.mg_hierarchy(33)
    A = H.A[-1]
    b = oracle.spmv(A, P.uniform_vector(A.rows, 2))
    x_o, u_o = oracle.mg(H, b, eps=1e-30, max_iters=1, max_iters_coarse=0)
    x_g, u_g, _, _ = mg_gpu(hb, H, b, eps=1e-30, max_iters=1, max_iters_coarse=0)
    assert u_o == u_g == 1
    assert np.array_equal(x_g, x_o)
    x_o, _ = oracle.mg(H, b, eps=1e-30, max_iters=3, max_iters_coarse=0, n_pre=3, n_post=1)
    x_g, _, _, _ = mg_gpu(hb, H, b, eps=1e-30, max_iters=3, max_iters_coarse=0, n_pre=3, n_post=1)
    assert np.array_equal(x_g, x_o)


def test_mg_f32_parity(hb, oracle):
    H = P.mg_hierarchy(129)
    A = H.A[-1]
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    H32 = H.astype(np.float32)
    b32 = b.astype(np.float32)
    x_o, u_o = oracle.mg(H32, b32, eps=1e-5)
    x_g, u_g, _, _ = mg_gpu(hb, H, b32, dtype=np.float32, eps=1e-5)
    assert abs(u_g - u_o) <= 1
    nb = np.linalg.norm(b)
    rg = np.linalg.norm(oracle.defect(A, b, x_g.astype(np.float64))) / nb
    ro = np.linalg.norm(oracle.defect(A, b, x_o.astype(np.float64))) / nb
    assert abs(rg - ro) <= 1e-5


def test_mg_featflow_fixture(hb, featflow):
    """MGSolverTest data (unstructured FEATFLOW2 matrices, 11 entries per row): the reference
    needs 59 cycles with this smoother; the solution matches sol_4 to the test's 8e-3."""
    H, d = featflow
    x_g, u_g, _, _ = mg_gpu(hb, H, d["rhs_4"], d["init_4"], eps=1e-8, max_iters=100)
    assert abs(u_g - int(d["mg_used"])) <= 1
    assert np.max(np.abs(x_g - d["sol_4"])) < 8e-3
    assert np.max(np.abs(x_g - d["mg_x"])) < 1e-8


def test_ir_mg_parity(hb, oracle):
    """Cell coefficients 10^U(-2,2) (Galerkin levels): reference loop (warm start) and the
    scaled mode; both reach a relative FP64 residual of 1e-10 with FP32 V-cycles to 1e-3."""
    for M, warm in ((33, True), (65, True), (65, False)):
        coef = P.log_uniform_coef(M, 1e-2, 1e2, M)
        H = P.mg_hierarchy(M, coef=coef)
        A = H.A[-1]
        b = oracle.spmv(A, P.uniform_vector(A.rows, 3))
        H32 = H.astype(np.float32)
        x_o, u_o, h_o = oracle.ir_mg(A, H32, b, eps=1e-10, inner_eps=1e-3, warm_start=warm)
        A64 = hb.SparseMatrixELL.from_reference(A)
        mg32 = hb.MGData.from_hierarchy(H, dtype=np.float32, eps=1e-3, max_iters=100)
        x = torch.zeros(A.rows, dtype=torch.float64, device="cuda")
        u_g, r0, r1 = hb.IRSolver.value(A64, dev(b), x, mg32, eps=1e-10, max_iters=100, warm_start=warm)
        x_g = host(x)
        assert abs(u_g - u_o) <= 1, (M, warm, u_g, u_o)
        # x0 = 0, so the outer stopping rule |r| < eps |r0| is a relative residual of 1e-10
        rel = np.linalg.norm(oracle.defect(A, b, x_g)) / np.linalg.norm(b)
        assert rel < 1e-10 and r1 < 1e-10 * r0
        mg32.close()


def test_ir_cg_parity(hb, oracle):
    M = 65
    A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, 8))
    b = oracle.spmv(A, P.uniform_vector(A.rows, 5))
    x_o, u_o, inner_o, _ = oracle.ir_cg(A, A.astype(np.float32), b, eps=1e-10, inner_eps=1e-3)
    A64 = hb.SparseMatrixELL.from_reference(A)
    A32 = A64.to_float()
    x = torch.zeros(A.rows, dtype=torch.float64, device="cuda")
    u_g, r0, r1, inner_g = hb.IRSolver.value_cg(A64, A32, dev(b), x, eps=1e-10, inner_eps=1e-3)
    assert abs(u_g - u_o) <= 1
    assert r1 < 1e-10 * r0
    assert abs(inner_g - inner_o) <= 0.05 * inner_o + u_o
    rel = np.linalg.norm(oracle.defect(A, b, host(x))) / np.linalg.norm(b)
    assert rel < 1e-10


def test_mg_full_size_2049_property(hb):
    """2049^2 (9 levels, 4.2M rows): the oracle would take minutes, so check properties --
    convergence to 1e-8 relative, the defect of the result measured with the bit-exact
    GPU defect, and the mixed-precision IR reaching 1e-10 relative with FP32 cycles."""
    M = 2049
    H = P.mg_hierarchy(M)
    data = hb.MGData.from_hierarchy(H, eps=1e-8, max_iters=60)
    A = data.A[-1]
    xt = dev(P.uniform_vector(M * M, 1))
    b = torch.empty_like(xt)
    hb.Product.value(b, A, xt)
    x = torch.zeros_like(b)
    used, r0, r1 = hb.MGSolver.value(data, b, x)
    assert used < 60 and r1 < 1e-8 * r0
    r = torch.empty_like(b)
    hb.Defect.value(r, b, A, x)
    assert abs(hb.Norm.value(r, root=True) - r1) <= 1e-12 * r0
    mg32 = hb.MGData.from_hierarchy(H, dtype=np.float32, eps=1e-3, max_iters=50)
    x2 = torch.zeros_like(b)
    u, s0, s1 = hb.IRSolver.value(A, b, x2, mg32, eps=1e-10, max_iters=50, warm_start=False)
    assert s1 < 1e-10 * s0
    assert ((x2 - xt).norm() / xt.norm()).item() < 1e-6


@pytest.mark.parametrize("M,coarse,coef", [(33, "rediscretize", False), (129, "rediscretize", False),
                                           (65, "rediscretize", True), (65, "galerkin", True), (257, "galerkin", True)])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_banded_matrix_free_mg_bitwise_equal_to_ell_mg(hb, M, coarse, coef, dt):
    """The banded cycle (banded smoother / defect, matrix-free PROLMAT-order transfers) rounds
    exactly as the ELL cycle on the same matrices: same cycles, same x bit for bit."""
    c = P.log_uniform_coef(M, 1e-1, 1e1, M) if coef else None
    H = P.mg_hierarchy(M, coef=c, coarse=coarse)
    eps = 1e-8 if dt == np.float64 else 1e-5
    tdt = torch.float64 if dt == np.float64 else torch.float32
    b = torch.from_numpy(P.uniform_vector(M * M, 4).astype(dt)).cuda()
    out = []
    for banded in (False, True):
        data = hb.MGData.from_hierarchy(H, dt, eps=eps, max_iters=50, banded=banded)
        x = torch.zeros(M * M, dtype=tdt, device="cuda")
        used, r0, r1 = hb.MGSolver.value(data, b, x)
        out.append((used, r0, r1, x.cpu().numpy()))
        data.close()
    assert out[0][:3] == out[1][:3]
    assert np.array_equal(out[0][3], out[1][3])


def test_banded_conversion_refuses_off_band_entries(hb):
    from honei_b200._lib import HBError
    A = P.q1_poisson(9)
    ip, ix, dv = A.to_csr()
    # add an entry two columns right of the diagonal in row 40 (not a Q1 band)
    rows = []
    for r in range(A.rows):
        cols, vals = list(ix[ip[r]:ip[r + 1]]), list(dv[ip[r]:ip[r + 1]])
        if r == 40:
            cols.append(42); vals.append(-0.125)
            order = np.argsort(cols); cols = list(np.array(cols)[order]); vals = list(np.array(vals)[order])
        rows.append((cols, vals))
    ip2 = np.cumsum([0] + [len(c) for c, _ in rows])
    B = P.ell_from_csr(A.rows, A.cols, ip2, np.concatenate([c for c, _ in rows]), np.concatenate([v for _, v in rows]))
    with pytest.raises(HBError) as e:
        hb.BandedMatrixQ1.from_ell(hb.SparseMatrixELL.from_reference(B))
    assert e.value.status == 6


@pytest.mark.parametrize("M", [64, 100, 130])
def test_banded_mg_general_sides_bitwise(hb, M):
    """Even and other non-(2^k + 1) sides (coarse side = side / 2 + 1, the served systems'
    coarsening): the banded, matrix-free cycle equals the ELL cycle bit for bit (FP32, SPD
    Galerkin hierarchy, dense coarse solve replaced by the coarse CG here)."""
    c = P.log_uniform_coef(M, 1e-2, 1e2, M)
    H = P.mg_hierarchy(M, coef=c, coarse="galerkin", symmetric=True).astype(np.float32)
    b = torch.from_numpy(P.uniform_vector(M * M, 2).astype(np.float32)).cuda()
    out = []
    for banded in (False, True):
        data = hb.MGData.from_hierarchy(H, np.float32, eps=1e-5, max_iters=30, banded=banded)
        x = torch.zeros(M * M, dtype=torch.float32, device="cuda")
        used, r0, r1 = hb.MGSolver.value(data, b, x)
        out.append((used, r0, r1, x.cpu().numpy()))
        data.close()
    assert out[0][:3] == out[1][:3]
    assert np.array_equal(out[0][3], out[1][3])


def test_mg_cycle_graph_recapture_and_parameter_changes(hb, oracle):
    """A solve replays its cycle as a captured CUDA graph: solving into another x buffer or with
    another b re-captures it (same results as the first buffers), and changing the parameters
    drops it (the new coarse iteration cap takes effect; the old one back gives the old x)."""
    M = 65
    H = P.mg_hierarchy(M)
    A = H.A[-1]
    b = oracle.spmv(A, P.uniform_vector(A.rows, 2))
    data = hb.MGData.from_hierarchy(H, eps=1e-8)
    bd = dev(b)
    xs = []
    for _ in range(2):                       # x1, x2, then x1 again
        for k in range(2):
            x = dev(np.zeros(A.rows))
            used, _, _ = hb.MGSolver.value(data, bd, x)
            xs.append((host(x), used))
    assert all(np.array_equal(xs[0][0], x) and xs[0][1] == u for x, u in xs)
    bd2 = dev(b * 2.0)
    x = dev(np.zeros(A.rows))
    hb.MGSolver.value(data, bd2, x)
    assert np.allclose(host(x), 2.0 * xs[0][0], rtol=0, atol=1e-7 * np.abs(xs[0][0]).max())
    x_o, u_o = oracle.mg(H, b, eps=1e-8, max_iters_coarse=1)
    data.configure(max_iters_coarse=1)
    x = dev(np.zeros(A.rows))
    used1, _, _ = hb.MGSolver.value(data, bd, x)
    assert abs(used1 - u_o) <= 1
    assert not np.array_equal(host(x), xs[0][0])
    data.configure(max_iters_coarse=1000)
    x = dev(np.zeros(A.rows))
    hb.MGSolver.value(data, bd, x)
    assert np.array_equal(host(x), xs[0][0])
    data.close()
