"""Canary-padded buffers: every caller-visible vector an entry point writes or reads is handed to
it as a view into a larger allocation whose guard zones before and after carry a fixed bit
pattern (a signalling-NaN payload for floating point); after the call, each guard zone must still
hold that pattern bit for bit.  A kernel that stores past the end of a vector -- a tail group of
four rows written whole, a row range rounded up to the matrix's padded ld, a reduction slot
placed one past the end -- changes a guard and fails here, on sizes chosen so that the vectors
end inside a group of four and inside a 64-row block (33^2 = 1089 rows, 17^2 = 289, 65^2 = 4225).

These checks stand in for running under a memory checker, which is not available where these
tests run; they are the canary part of the debug checks (with hb_ell_validate for the matrices'
column bounds and the bounded device waits of test_gpu_failure.py)."""
import ctypes as C

import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

GUARD = 256                      # elements on each side (keeps the view 16-byte aligned)
PATTERN = {torch.float64: 0x7FF4DEADBEEFCAFE, torch.float32: 0x7FA5C0DE, torch.int32: 0x5A5A5A5A}
INT_VIEW = {torch.float64: torch.int64, torch.float32: torch.int32, torch.int32: torch.int32}
MASK = [2, 0, 2, 0, 2, 2, 0, 0]  # a Dirichlet mask with both kinds of sides


class Guarded:
    """A length-n vector inside guard zones; .v is the view handed to the library."""

    def __init__(self, n, dtype, values=None):
        self.n, self.dtype = n, dtype
        self.full = torch.empty(n + 2 * GUARD, dtype=dtype, device="cuda")
        bits = self.full.view(INT_VIEW[dtype])
        pat = PATTERN[dtype]
        if INT_VIEW[dtype] == torch.int32 and pat >= 2 ** 31:
            pat -= 2 ** 32
        bits.fill_(pat)
        self.v = self.full[GUARD:GUARD + n]
        if values is not None:
            self.v.copy_(torch.as_tensor(values, dtype=dtype))
        else:
            self.v.zero_()
        self._pat = pat

    def intact(self) -> bool:
        torch.cuda.synchronize()
        bits = self.full.view(INT_VIEW[self.dtype])
        return bool((bits[:GUARD] == self._pat).all() and (bits[GUARD + self.n:] == self._pat).all())


def guarded_like(values, dtype):
    return Guarded(len(values), dtype, values)


def diagonal(A):
    ip, ix, dv = A.to_csr()
    return np.array([dv[ip[r]:ip[r + 1]][ix[ip[r]:ip[r + 1]] == r][0] for r in range(A.rows)])


def check(*gs):
    bad = [i for i, g in enumerate(gs) if not g.intact()]
    assert not bad, f"guard zone overwritten on argument(s) {bad}"


@pytest.fixture(scope="module")
def la():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


TDT = {np.float64: torch.float64, np.float32: torch.float32}


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("M", [17, 33])
def test_products_and_defect_stay_inside_their_vectors(la, oracle, dt, M):
    A = P.q1_poisson(M).astype(dt)
    Ad = la.SparseMatrixELL.from_reference(A)
    td = TDT[dt]
    xh = P.uniform_vector(A.rows, 1).astype(dt)
    x, y = guarded_like(xh, td), Guarded(A.rows, td)
    la.Product.value(y.v, Ad, x.v)
    check(x, y)
    assert np.array_equal(y.v.cpu().numpy(), oracle.spmv(A, xh))
    b, r = guarded_like(P.uniform_vector(A.rows, 2).astype(dt), td), Guarded(A.rows, td)
    la.Defect.value(r.v, b.v, Ad, x.v)
    check(x, b, r)
    # the ordered copy's forms (rows, ranked, packed)
    for form in ({"columns": False}, {"columns": True, "packed": False}, {"columns": True, "packed": True}):
        y2 = Guarded(A.rows, td)
        la.Product.value(y2.v, Ad.ordered(**form), x.v)
        check(x, y2)
        assert torch.equal(y2.v, y.v)
    Ab = la.BandedMatrixQ1.from_ell(Ad)
    y3 = Guarded(A.rows, td)
    la.Product.value(y3.v, Ab, x.v)
    check(x, y3)
    # the banded product sums in the reference's banded order (diagonal first), not the ELL's
    assert np.array_equal(y3.v.cpu().numpy(), oracle.q1band_spmv(list(Ab.bands[:, :A.rows].cpu().numpy()), xh))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 5, 289, 1089, 4225])
def test_vector_kernels_stay_inside_their_vectors(la, dt, n):
    td = TDT[dt]
    x = guarded_like(P.uniform_vector(n, 1).astype(dt), td)
    y = guarded_like(P.uniform_vector(n, 2).astype(dt), td)
    r = Guarded(n, td)
    la.ScaledSum.value(x.v, y.v, 0.5)
    la.ScaledSum.value(r.v, x.v, y.v, -2.0)
    la.Scale.value(r.v, 3.0)
    la.Sum.value(r.v, y.v)
    la.Difference.value(r.v, x.v, y.v)
    la.ElementProduct.value(r.v, x.v, y.v)
    la.DotProduct.value(x.v, y.v)
    la.Norm.value(x.v, root=True)
    check(x, y, r)


def test_transfers_stay_inside_their_vectors(la):
    for Mc in (5, 9, 17):
        Mf = 2 * Mc - 1
        c = guarded_like(P.uniform_vector(Mc * Mc, 1), torch.float64)
        f = Guarded(Mf * Mf, torch.float64)
        la.Prolongation.value(f.v, c.v, MASK)
        c2 = Guarded(Mc * Mc, torch.float64)
        la.Restriction.value(c2.v, f.v, MASK)
        check(c, f, c2)


@pytest.mark.parametrize("resident", [True, False])
def test_solvers_stay_inside_their_vectors(la, oracle, resident):
    prev = la.CGSolver.set_resident(resident)
    try:
        for M in (17, 33):
            A = P.q1_poisson(M)
            Ad = la.SparseMatrixELL.from_reference(A)
            b = guarded_like(oracle.spmv(A, P.uniform_vector(A.rows, 1)), torch.float64)
            x = Guarded(A.rows, torch.float64)
            used = la.CGSolver.value(Ad, None, b.v, x.v, 10000, 1e-8)
            check(b, x)
            assert used > 0
            Pj = guarded_like(0.7 / diagonal(A), torch.float64)
            x2 = Guarded(A.rows, torch.float64)
            la.CGSolverVAR.value(Ad, Pj.v, b.v, x2.v, 10000, 1e-8)
            check(b, x2, Pj)
    finally:
        la.CGSolver.set_resident(prev)


def test_mg_and_refinement_stay_inside_their_vectors(la, oracle):
    H = P.mg_hierarchy(65)
    data = la.MGData.from_hierarchy(H, np.float64, eps=1e-8, max_iters=50, max_iters_coarse=100)
    A = H.A[-1]
    b = guarded_like(oracle.spmv(A, P.uniform_vector(A.rows, 3)), torch.float64)
    x = Guarded(A.rows, torch.float64)
    la.MGSolver.value(data, b.v, x.v)
    check(b, x)
    Ad = la.SparseMatrixELL.from_reference(A)
    x2 = Guarded(A.rows, torch.float64)
    la.IRSolver.value_cg(Ad, Ad.to_float(), b.v, x2.v, eps=1e-10, inner_eps=1e-3)
    check(b, x2)


@pytest.mark.parametrize("mode", ["cg64", "ir32"])
def test_batch_stays_inside_each_systems_vectors(la, mode):
    from honei_b200 import batch as B
    sides = [5, 17, 33, 9, 21]
    systems = B.q1_batch(sides, coef_range=(1e-1, 1e1), seed=7, mode=mode)
    guards = []
    for s in systems:
        gb = guarded_like(s.b.cpu().numpy(), torch.float64)
        gx = Guarded(s.n, torch.float64)
        s.b, s.x = gb.v, gx.v
        guards += [gb, gx]
    for shape in ((1, 256, 0, 4), (4, 256, 0, 1), (2, 512, 0, 4)):
        for s in systems:
            s.x.zero_()
        res = B.BatchSolver(systems).solve(B.HbBatchConfig(*shape))
        assert all(r["status"] == 0 for r in res)
        check(*guards)


def test_noalloc_cg_stays_inside_its_vectors(la, oracle):
    from honei_b200._lib import lib
    A = P.q1_poisson(33)
    Ad = la.SparseMatrixELL.from_reference(A)
    b = guarded_like(oracle.spmv(A, P.uniform_vector(A.rows, 1)), torch.float64)
    x = Guarded(A.rows, torch.float64)
    used, d = C.c_int64(0), C.c_double(0)
    st = lib().hb_cg_f64_noalloc(C.byref(Ad.struct), b.v.data_ptr(), x.v.data_ptr(), 10000, 1e-8, C.byref(used),
                                 C.byref(d), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0 and used.value > 0
    check(b, x)
