"""Device-built multigrid for Q1 grids of any side (hb_q1_*): transfers and Galerkin levels
against the host generators, and the served mixed-precision solve (FP64 refinement around FP32
MG-preconditioned CG) against the oracle's restatement of the same algorithm."""
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


def csr_equal(A, B, rtol=0.0):
    ia, ja, va = A.to_csr()
    ib, jb, vb = B.to_csr()
    if not (np.array_equal(ia, ib) and np.array_equal(ja, jb)):
        return False
    if rtol == 0.0:
        return np.array_equal(va, vb)
    return np.allclose(va, vb, rtol=rtol, atol=rtol * np.abs(vb).max())


@pytest.mark.parametrize("Mf", [3, 4, 9, 10, 33, 64, 100])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_transfers_match_host(hb, Mf, dtype):
    import ctypes as C
    from honei_b200._lib import HbEll, lib
    Mc = Mf // 2 + 1
    assert lib().hb_q1_coarse_side(Mf) == Mc == P.coarse_side(Mf)
    Kp, ldp = hb.SparseMatrixELL.layout(Mf * Mf, 4)
    Kr, ldr = hb.SparseMatrixELL.layout(Mc * Mc, 9)
    tens = [torch.empty(Kp * ldp, dtype=torch.int32, device="cuda"), torch.empty(Kp * ldp, dtype=dtype, device="cuda"),
            torch.empty(Kr * ldr, dtype=torch.int32, device="cuda"), torch.empty(Kr * ldr, dtype=dtype, device="cuda")]
    dt = 0 if dtype == torch.float64 else 1
    Pd = HbEll(0, 0, Kp, ldp, tens[0].data_ptr(), tens[1].data_ptr(), dt, 0)
    Rd = HbEll(0, 0, Kr, ldr, tens[2].data_ptr(), tens[3].data_ptr(), dt, 0)
    assert lib().hb_q1_transfers(hb.default_context().handle, Mf, C.byref(Pd), C.byref(Rd)) == 0
    Pg = hb.SparseMatrixELL(Pd.rows, Pd.cols, Kp, ldp, tens[0], tens[1]).to_host()
    Rg = hb.SparseMatrixELL(Rd.rows, Rd.cols, Kr, ldr, tens[2], tens[3]).to_host()
    nf, nc, ip, ix, dv = P.prolongation_csr(Mf=Mf)
    npdt = np.float64 if dtype == torch.float64 else np.float32
    Ph = P.ell_from_csr(nf, nc, ip, ix, dv, 1, npdt)
    Rh = P.ell_from_csr(nc, nf, *P.transpose_csr(nf, nc, ip, ix, dv), 1, npdt)
    assert csr_equal(Pg, Ph) and csr_equal(Rg, Rh)


@pytest.mark.parametrize("M", [9, 10, 33, 64, 100, 257])
def test_galerkin_levels_match_host(hb, M):
    coef = P.log_uniform_coef(M, 1e-2, 1e2, M)
    q = hb.Q1System(M, torch.from_numpy(coef.ravel()).cuda())
    H = P.mg_hierarchy(M, coef=coef, symmetric=True, coarse="galerkin")
    assert q.sides == H.sides
    for l in range(len(q.sides)):
        A64, A32, Pd, Rd = q.level(l)
        assert csr_equal(A64.to_host(), H.A[l], rtol=1e-13), l
        if Pd is not None:
            assert csr_equal(Pd.to_host(), H.prol[l].astype(np.float32))
            assert csr_equal(Rd.to_host(), H.res[l].astype(np.float32))
    q.close()


@pytest.mark.parametrize("M", [17, 33, 64, 100])
def test_served_solve_matches_oracle(hb, oracle, M):
    coef = P.log_uniform_coef(M, 1e-2, 1e2, 7 + M)
    q = hb.Q1System(M, torch.from_numpy(coef.ravel()).cuda())
    # the oracle runs on the device-built matrices themselves
    L = len(q.sides)
    levels = [q.level(l) for l in range(L)]
    H32 = P.MGHierarchy([lv[1].to_host() for lv in levels], [lv[2].to_host() for lv in levels[:-1]],
                        [lv[3].to_host() for lv in levels[:-1]], list(q.sides))
    A64 = levels[-1][0].to_host()
    xt = P.uniform_vector(M * M, 3)
    b = oracle.spmv(A64, xt)
    x_o, outer_o, inner_o, hist = oracle.ir_pcg(A64, H32, b, eps=1e-8, inner_eps=1e-3)
    x = torch.zeros(M * M, dtype=torch.float64, device="cuda")
    info = q.solve(torch.from_numpy(b).cuda(), x, eps=1e-8, inner_eps=1e-3)
    xg = x.cpu().numpy()
    rel = np.linalg.norm(oracle.defect(A64, b, xg)) / np.linalg.norm(b)
    assert info["status"] == 0 and rel < 1e-8 and abs(info["true_relres"] - rel) <= 1e-12 + 1e-6 * rel
    assert abs(info["outer"] - outer_o) <= 1, (info, outer_o)
    assert abs(info["iterations"] - inner_o) <= 0.2 * inner_o + 2, (info, inner_o)
    assert np.linalg.norm(xg - xt) <= 1e-5 * np.linalg.norm(xt)
    q.close()


def test_served_solve_large_high_contrast(hb):
    """1025^2 nodes, cell coefficient 10^U(-2,2): the largest request of the serving stream."""
    M = 1025
    coef = torch.from_numpy(P.log_uniform_coef(M, 1e-2, 1e2, 1).ravel()).cuda()
    q = hb.Q1System(M, coef)
    xt = torch.from_numpy(P.uniform_vector(M * M, 2)).cuda()
    b = torch.empty_like(xt)
    hb.Product.value(b, q.A, xt)
    x = torch.zeros_like(b)
    info = q.solve(b, x, eps=1e-8)
    r = torch.empty_like(b)
    hb.Defect.value(r, b, q.A, x)
    rel = hb.Norm.value(r, root=True) / hb.Norm.value(b, root=True)
    assert rel < 1e-8 and info["outer"] <= 6 and info["iterations"] < 400, info
    q.close()
