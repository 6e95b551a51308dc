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


def _batch_case(hb, sides, seed0=0):
    systems, bs, xts = [], [], []
    for k, M in enumerate(sides):
        coef = torch.from_numpy(P.log_uniform_coef(M, 1e-2, 1e2, seed0 + k).ravel()).cuda()
        q = hb.Q1System(M, coef)
        xt = torch.from_numpy(P.uniform_vector(M * M, seed0 + k + 100)).cuda()
        b = torch.empty_like(xt)
        hb.Product.value(b, q.A, xt)
        systems.append(q)
        bs.append(b)
        xts.append(xt)
    return systems, bs, xts


@pytest.mark.parametrize("cluster,threads", [(8, 256), (4, 512), (1, 256), (16, 256)])
def test_batched_served_solve_matches_single(hb, cluster, threads):
    """hb_q1_batch_solve runs hb_q1_solve's algorithm per cluster: same outer steps, inner
    iterations within a few (only the dot products' summation order differs), FP64 target met."""
    sides = [17, 33, 40, 64, 100, 129, 257]
    systems, bs, xts = _batch_case(hb, sides)
    xs = [torch.zeros_like(b) for b in bs]
    infos = hb.Q1System.solve_batch(systems, bs, xs, eps=1e-8, cluster=cluster, threads=threads)
    for q, b, x, xt, info in zip(systems, bs, xs, xts, infos):
        x1 = torch.zeros_like(b)
        ref = q.solve(b, x1, eps=1e-8)
        r = torch.empty_like(b)
        hb.Defect.value(r, b, q.A, x)
        rel = hb.Norm.value(r, root=True) / hb.Norm.value(b, root=True)
        assert info["status"] == 0 and rel < 1e-8 and abs(info["true_relres"] - rel) <= 1e-6 * rel + 1e-15, (q.M, info)
        assert abs(info["outer"] - ref["outer"]) <= 1, (q.M, info, ref)
        assert abs(info["iterations"] - ref["iterations"]) <= 0.1 * ref["iterations"] + 3, (q.M, info, ref)
        assert float(torch.linalg.norm(x - x1) / torch.linalg.norm(x1)) < 1e-6
    for q in systems:
        q.close()


def test_batched_served_solve_matches_oracle(hb, oracle):
    M = 64
    systems, bs, _ = _batch_case(hb, [M], seed0=7)
    q = systems[0]
    L = len(q.sides)
    levels = [q.level(l) for l in range(L)]
    H32 = P.MGHierarchy([lv[1].to_host() for lv in levels], [lv[2].to_host() for lv in levels[:-1]],
                        [lv[3].to_host() for lv in levels[:-1]], list(q.sides))
    A64 = levels[-1][0].to_host()
    b = bs[0].cpu().numpy()
    x_o, outer_o, inner_o, hist = oracle.ir_pcg(A64, H32, b, eps=1e-8, inner_eps=1e-3)
    x = torch.zeros_like(bs[0])
    (info,) = hb.Q1System.solve_batch(systems, bs, [x], eps=1e-8)
    assert abs(info["outer"] - outer_o) <= 1 and abs(info["iterations"] - inner_o) <= 0.2 * inner_o + 2, (info, inner_o)
    assert np.linalg.norm(x.cpu().numpy() - x_o) <= 1e-6 * np.linalg.norm(x_o)
    q.close()


def test_batched_served_solve_alone_equals_in_the_mix(hb):
    sides = [33, 65, 129, 200]
    systems, bs, _ = _batch_case(hb, sides, seed0=3)
    mix = [torch.zeros_like(b) for b in bs]
    infos = hb.Q1System.solve_batch(systems, bs, mix, eps=1e-8, cluster=8, threads=256)
    for q, b, xm, im in zip(systems, bs, mix, infos):
        xa = torch.zeros_like(b)
        (ia,) = hb.Q1System.solve_batch([q], [b], [xa], eps=1e-8, cluster=8, threads=256)
        assert ia == im and torch.equal(xa, xm), q.M
    # the same handle twice in one batch is refused
    from honei_b200._lib import HBError
    with pytest.raises(HBError):
        hb.Q1System.solve_batch([systems[0], systems[0]], [bs[0], bs[0]], [mix[0], mix[0]])
    for q in systems:
        q.close()


@pytest.mark.parametrize("M", [9, 17, 100, 257, 300, 700])
def test_fused_coarse_cycle_same_iterates(hb, M):
    """The coarse levels of the served cycle in one single-cluster launch compute exactly what the
    per-level kernels compute: the same solve, bit for bit."""
    coef = torch.from_numpy(P.log_uniform_coef(M, 1e-2, 1e2, 3 + M).ravel()).cuda()
    q = hb.Q1System(M, coef)
    xt = torch.from_numpy(P.uniform_vector(M * M, 9)).cuda()
    b = torch.empty_like(xt)
    hb.Product.value(b, q.A, xt)
    x1 = torch.zeros_like(b)
    i1 = q.solve(b, x1, eps=1e-8)
    q.set_fused_tail(0)
    x0 = torch.zeros_like(b)
    i0 = q.solve(b, x0, eps=1e-8)
    assert i0 == i1 and torch.equal(x0, x1), (i0, i1)
    for rows in (289, 17000, 70000):
        q.set_fused_tail(rows)
        x2 = torch.zeros_like(b)
        i2 = q.solve(b, x2, eps=1e-8)
        assert i2 == i1 and torch.equal(x2, x1), (rows, i2, i1)
    q.close()
