"""GPU parity of SPAI2<tags::GPU::CUDA>::value(M, A) (honei/math/spai2.hh:294-298) against
SPAI2<tags::CPU::SSE> (honei/math/spai2.hh:129-260): the reference's outputs stored in
tests/golden/spai2.npz and the oracle's restatement (oracle/ora_spai2.inc).

Bar: bit-exact.  Every column's normal equations are summed in the reference's order and its
LU runs the reference's operations in the reference's order, FP32 and FP64 alike.  At the full
Q1 2049^2 size the oracle is run on column ranges (its col_start / col_end arguments) and the
device result is compared there.
"""
import dataclasses

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


def gpu_spai2(hb, A):
    """(M's values, sorted by (row, column)) and the keys, from the device SPAI2 of A."""
    Ad = hb.SparseMatrixELL.from_reference(A)
    M = hb.SPAI2.value(Ad)
    return entries(M.to_host())


def entries(E, Ax=None):
    """(keys, values) of the entries of E (slots whose value in E is not 0), values taken from
    Ax (E's layout) when given, sorted by (row, column)."""
    ip, ix, dv = E.to_csr()
    vals = dv if Ax is None else dataclasses.replace(E, Ax=Ax).to_csr()[2]
    rows = np.repeat(np.arange(E.rows), np.diff(ip))
    keep = dv != 0
    order = np.lexsort((ix[keep], rows[keep]))
    return np.stack([rows[keep][order], ix[keep][order]]), vals[keep][order]


def oracle_spai2(oracle, A, lo=0, hi=0):
    return entries(A, oracle.spai2(A, lo, hi))


def same_bits(a, b):
    if a.shape != b.shape:
        return False
    nan = np.isnan(a)
    return np.array_equal(nan, np.isnan(b)) and np.array_equal(a[~nan].view(np.uint8), b[~nan].view(np.uint8))


def test_spai2_matches_reference_fixture(hb):
    """The reference's SPAI2<tags::CPU::SSE> of the FEATFLOW matrices (Q2 with 25 entries per row
    and Q1 levels) and of its Q1 33^2 construction, FP64 and FP32."""
    g, f = load_golden("spai2"), load_golden("featflow_pa4")
    cases = [("q2a2", golden_matrix(g, "q2a2")), ("pa_a4", golden_matrix(g, "pa_a4")),
             ("pa4_a4", golden_matrix(f, "A_4")), ("q1", golden_matrix(g, "q1"))]
    for name, A in cases:
        ip, ix, _ = A.to_csr()
        rows = np.repeat(np.arange(A.rows), np.diff(ip))
        order = np.lexsort((ix, rows))
        for dt, suf in ((np.float64, "64"), (np.float32, "32")):
            keys, vals = gpu_spai2(hb, A.astype(dt))
            assert np.array_equal(keys, np.stack([rows[order], ix[order]])), name
            assert same_bits(vals, g[f"{name}_M{suf}"][order]), (name, suf)


@pytest.mark.parametrize("name,make", [
    ("q1_65", lambda: P.q1_poisson(65)),
    ("q1_65_varcoef", lambda: P.q1_poisson(65, P.log_uniform_coef(65, 1e-2, 1e2, 4))),
    ("q1_65_permuted", lambda: P.q1_poisson_permuted(65, 5)[0]),
    ("q1_33_threads4", lambda: P.ell_from_csr(1089, 1089, *P.q1_poisson_csr(33), threads=4)),
    ("q1_33_spd", lambda: P.q1_poisson(33, symmetric=True)),
])
def test_spai2_bitwise_against_oracle(hb, oracle, name, make):
    A = make()
    for dt in (np.float64, np.float32):
        B = A.astype(dt)
        keys, vals = gpu_spai2(hb, B)
        okeys, ovals = oracle_spai2(oracle, B)
        assert np.array_equal(keys, okeys) and same_bits(vals, ovals), (name, dt)


def random_square(rng, n, fill, diag=True, dtype=np.float64):
    mask = rng.random((n, n)) < fill
    if diag:
        np.fill_diagonal(mask, True)
    ri, ci = np.nonzero(mask)
    ip = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(ri, minlength=n), out=ip[1:])
    vals = rng.uniform(-1, 1, len(ci)) + np.where(ri == ci, 4.0 + n * fill, 0.0)
    return P.ell_from_csr(n, n, ip, ci, vals, 1, dtype)


def test_spai2_random_patterns_and_wide_columns(hb, oracle):
    """Unsymmetric random patterns; columns of 40-70 entries (the column lists and the normal
    equations larger than a warp: several 32-row chunks of At and more than 32 unknowns)."""
    rng = np.random.default_rng(11)
    for n, fill in ((50, 0.1), (300, 0.02), (120, 0.45)):
        for dt in (np.float64, np.float32):
            A = random_square(rng, n, fill, dtype=dt)
            keys, vals = gpu_spai2(hb, A)
            okeys, ovals = oracle_spai2(oracle, A)
            assert np.array_equal(keys, okeys) and same_bits(vals, ovals), (n, fill, dt)


def test_spai2_edge_cases(hb, oracle):
    """An empty row and column, a column whose system is empty (n1 == 0: M keeps A's value), a
    1 x 1 matrix; a non-square matrix, a column system too large for shared memory and a column
    longer than any kernel solves are refused."""
    # column 0 holds row 1 only, and column 1 is empty: n1 == 0, M(1, 0) stays 5
    A = P.ell_from_csr(3, 3, np.array([0, 0, 1, 2]), np.array([0, 2]), np.array([5.0, 2.0]))
    keys, vals = gpu_spai2(hb, A)
    okeys, ovals = oracle_spai2(oracle, A)
    assert np.array_equal(keys, okeys) and same_bits(vals, ovals)
    assert vals[0] == 5.0 and vals[1] == 0.5
    A = P.ell_from_csr(1, 1, np.array([0, 1]), np.array([0]), np.array([4.0]))
    assert gpu_spai2(hb, A)[1][0] == 0.25
    from honei_b200._lib import HBError
    R = hb.SparseMatrixELL.from_reference(P.ell_from_csr(4, 6, np.array([0, 1, 2, 3, 4]), np.arange(4),
                                                         np.ones(4)))
    with pytest.raises(hb.MatrixRowsDoNotMatch):
        hb.SPAI2.value(R)
    dense = random_square(np.random.default_rng(3), 200, 1.0)
    with pytest.raises(HBError):
        hb.SPAI2.value(hb.SparseMatrixELL.from_reference(dense))
    # a column of 300 entries (every row couples to row 0): longer than any kernel solves, refused
    # after the column lists are built (and left unsorted)
    n = 300
    ip = np.concatenate([[0], np.arange(1, 2 * n, 2)])
    ix = np.concatenate([[0]] + [[0, r] for r in range(1, n)])
    vals = np.where(ix == 0, -1.0, 4.0)
    vals[0] = 4.0
    with pytest.raises(HBError):
        hb.SPAI2.value(hb.SparseMatrixELL.from_reference(P.ell_from_csr(n, n, ip, ix, vals)))


def test_spai2_2049_column_ranges(hb, oracle):
    """Full size (Q1 2049^2 FP64, 4.2M columns): the device result equals the oracle on column
    ranges at the start, in the middle (an interior grid line) and at the end."""
    A = P.q1_poisson(2049)
    Ad = hb.SparseMatrixELL.from_reference(A)
    Mh = hb.SPAI2.value(Ad).to_host()
    del Ad
    _, ix, _ = A.to_csr()
    got = Mh.to_csr()[2]
    for lo, hi in ((0, 3000), (2049 * 1024 - 1500, 2049 * 1024 + 1500), (A.rows - 3000, A.rows)):
        want = dataclasses.replace(A, Ax=oracle.spai2(A, lo, hi)).to_csr()[2]
        sel = (ix >= lo) & (ix < hi)
        assert same_bits(got[sel], want[sel]), (lo, hi)
    torch.cuda.empty_cache()


def test_spai2_preconditioned_cg(hb, oracle):
    """CGSolver<VAR> with the device-built SPAI2 of the FEATFLOW A_4 equals the solve with the
    reference's SPAI2 bit for bit (same preconditioner), and the reference's own SPAI2 test
    property holds: ||I - A M||_1 < ||I - A diag(A)^-1||_1 (honei/math/spai2_TEST.cc:47-77)."""
    f, g = load_golden("featflow_pa4"), load_golden("spai2")
    A = golden_matrix(f, "A_4")
    Ad = hb.SparseMatrixELL.from_reference(A)
    M = hb.SPAI2.value(Ad)
    Mref = hb.SparseMatrixELL.from_reference(
        P.ell_from_csr(A.rows, A.cols, *A.to_csr()[:2], g["pa4_a4_M64"]))
    xs = []
    for Pm in (M, Mref):
        x = torch.from_numpy(f["init_4"].copy()).cuda()
        used = hb.CGSolverVAR.value(Ad, Pm, torch.from_numpy(f["rhs_4"]).cuda(), x, 700, 1e-8)
        xs.append((used, x.cpu().numpy()))
    assert xs[0][0] == xs[1][0] and np.array_equal(xs[0][1], xs[1][1])
    xo, uo = oracle.cg_var(A, dataclasses.replace(A, Ax=oracle.spai2(A)), f["rhs_4"], x0=f["init_4"],
                           max_iters=700, eps=1e-8)
    assert abs(xs[0][0] - uo) <= 1
    B = golden_matrix(g, "q2a2")
    _, mv = gpu_spai2(hb, B)
    ip, ix, dv = B.to_csr()
    rows = np.repeat(np.arange(B.rows), np.diff(ip))
    Adn = np.zeros((B.rows, B.cols))
    Adn[rows, ix] = dv
    Mdn = np.zeros_like(Adn)
    order = np.lexsort((ix, rows))
    Mdn[rows[order], ix[order]] = mv
    eye = np.eye(B.rows)
    assert np.abs(eye - Adn @ Mdn).sum() < np.abs(eye - Adn @ np.diag(1 / np.diag(Adn))).sum()


def test_elltospai_client(hb, tmp_path):
    """clients/io_tools/elltospai.cc on the device: the file's SPAI2 written in the same one-lane
    ELL layout, values bit-identical to the reference's."""
    from honei_b200 import io_tools
    g = load_golden("spai2")
    A = golden_matrix(g, "pa_a4")
    P.write_ell(str(tmp_path / "A.ell"), A)
    assert io_tools.main(["elltospai", str(tmp_path / "A.ell"), str(tmp_path / "M.ell")]) == 0
    M = P.read_ell(str(tmp_path / "M.ell"))
    assert (M.rows, M.cols, M.stride, M.ncpr) == (A.rows, A.cols, A.stride, A.ncpr)
    assert np.array_equal(M.Aj, A.Aj)
    assert same_bits(M.to_csr()[2], g["pa_a4_M64"])
