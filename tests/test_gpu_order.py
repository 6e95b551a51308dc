"""Locality order (hb_ell_cm_order) and the product through a reordered copy (hb_ell_permute,
hb_spmv_rows, hb_gather; the sorted copy with hb_spmv_ranked; the packed form with
hb_ell_pack_offsets and hb_spmv_packed).

The order has no reference counterpart; the product through the reordered copy must equal the
product on the matrix as given (Product<tags::CPU>, honei/la/product.hh:148-204) bit for bit,
whichever numbering the matrix has.  The order itself is checked against a sequential
Cuthill-McKee written here from its definition.
"""
from collections import deque

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


def sequential_cm(A):
    """Cuthill-McKee as the device kernel defines it: start at the row with the fewest
    off-diagonal entries (lowest index on ties) among rows that have one; visit rows level by
    level, each row's unvisited columns in slot order; unreached rows last, ascending."""
    ip, ix, _ = A.to_csr()
    n = A.rows
    deg = np.array([np.count_nonzero(ix[ip[r]:ip[r + 1]] != r) for r in range(n)])
    cand = np.flatnonzero(deg > 0)
    order, seen = [], np.zeros(n, bool)
    if len(cand):
        start = cand[np.argmin(deg[cand])]
        q = deque([start])
        seen[start] = True
        while q:
            v = q.popleft()
            order.append(v)
            for c in ix[ip[v]:ip[v + 1]]:
                if c != v and not seen[c]:
                    seen[c] = True
                    q.append(c)
    order += [r for r in range(n) if not seen[r]]
    return np.array(order, np.int32)


def random_pattern(n, seed, max_per_row=7):
    """Rows of 0..max_per_row random columns (ascending, values U[-1,1]); a quarter of the rows
    empty, so parts of the graph are not reached from the start row."""
    rng = np.random.default_rng(seed)
    ip, ix, dv = [0], [], []
    for r in range(n):
        k = 0 if rng.random() < 0.25 else int(rng.integers(1, max_per_row + 1))
        cols = np.unique(rng.integers(0, n, size=k))
        ix.extend(cols.tolist())
        dv.extend(rng.uniform(-1, 1, size=len(cols)).tolist())
        ip.append(len(ix))
    dv = [v if v != 0.0 else 0.5 for v in dv]
    return P.ell_from_csr(n, n, np.array(ip), np.array(ix, np.int64), np.array(dv))


CASES = [
    ("q1_33", lambda: P.q1_poisson(33)),
    ("q1_33_permuted", lambda: P.q1_poisson_permuted(33, 2)[0]),
    ("q1_65_spd_varcoef", lambda: P.q1_poisson(65, P.log_uniform_coef(65, 1e-1, 1e1, 3), symmetric=True)),
    ("q1_17_threads3", lambda: P.ell_from_csr(289, 289, *P.q1_poisson_csr(17), threads=3)),
    ("random_pattern_500", lambda: random_pattern(500, 11)),
    # 4096 rows and more take the grid-wide kernel
    ("q1_129_permuted", lambda: P.q1_poisson_permuted(129, 6)[0]),
    ("random_pattern_6000", lambda: random_pattern(6000, 12)),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_cm_order_matches_sequential_definition(hb, name, make):
    A = make()
    Ad = hb.SparseMatrixELL.from_reference(A)
    order, pos, info = Ad.cm_order()
    o = order.cpu().numpy()
    assert np.array_equal(np.sort(o), np.arange(A.rows))
    assert np.array_equal(pos.cpu().numpy()[o], np.arange(A.rows))
    assert np.array_equal(o, sequential_cm(A))
    order2, _, info2 = Ad.cm_order()
    assert torch.equal(order, order2) and info == info2


FORMS = ["rows", "ranked", "packed"]


def ordered_form(Ad, form):
    """The ordered copy in one of its forms: rows (A's columns), ranked (renumbered, slots sorted
    by new column, 64-bit summation ranks) and packed (renumbered, slots in their order, 16-bit
    column offsets)."""
    B = Ad.ordered(columns=form != "rows", packed=form == "packed")
    if form == "packed":
        assert B.Bd is not None and B.Bd.dtype == torch.int16 and B.ranks is None
    else:
        assert B.Bd is None
    return B


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_product_through_ordered_copy_bit_exact(hb, oracle, name, make, form, dt):
    A = make().astype(dt)
    Ad = hb.SparseMatrixELL.from_reference(A)
    Bd = ordered_form(Ad, form)
    x = P.uniform_vector(A.cols, 5).astype(dt)
    y = torch.full((A.rows,), float("nan"), dtype=Ad.dtype, device="cuda")
    hb.Product.value(y, Bd, torch.from_numpy(x).cuda())
    assert np.array_equal(y.cpu().numpy(), oracle.spmv(A, x))


def test_packed_form_declined_falls_back_to_ranks(hb, oracle):
    """The packed form needs K <= 9 and every reordered column within +-32767 of its row: a
    random pattern over 120,000 rows (offsets up to n after ordering) and one with 12 entries per
    row fall back to the sorted, ranked form, and their products stay bit-exact."""
    for A in (random_pattern(120000, 7, max_per_row=3), random_pattern(800, 9, max_per_row=12)):
        Ad = hb.SparseMatrixELL.from_reference(A)
        B = Ad.ordered(columns=True, packed=True)
        assert B.Bd is None and B.ranks is not None
        x = P.uniform_vector(A.cols, 2)
        y = torch.empty(A.rows, dtype=torch.float64, device="cuda")
        hb.Product.value(y, B, torch.from_numpy(x).cuda())
        assert np.array_equal(y.cpu().numpy(), oracle.spmv(A, x))


def test_ordered_copy_of_permuted_grid_is_banded(hb):
    """A randomly numbered 129^2 grid has bandwidth near n; its Cuthill-McKee copy has the
    bandwidth of a grid ordering (a few grid lines)."""
    M = 129
    Ap, _ = P.q1_poisson_permuted(M, 4)
    Ad = hb.SparseMatrixELL.from_reference(Ap)
    assert Ad.bandwidth() > M * M // 2
    order, pos, (levels, reached, start) = Ad.cm_order()
    assert reached == M * M                  # every row: the boundary rows as leaves
    assert Ad.bandwidth(pos) <= 6 * M
    B = Ad.ordered(columns=True)
    assert B.B.bandwidth() == Ad.bandwidth(pos)


def test_product_through_ordered_copy_2049_permuted_bit_exact(hb, oracle):
    """The permuted 2049^2 workload: every form of the ordered copy gives the product on the
    permuted matrix bit for bit."""
    Ap, _ = P.q1_poisson_permuted(2049, 5)
    Ad = hb.SparseMatrixELL.from_reference(Ap)
    x = torch.from_numpy(P.uniform_vector(Ap.rows, 6)).cuda()
    y0 = torch.empty_like(x)
    hb.Product.value(y0, Ad, x)
    for form in FORMS:
        B = ordered_form(Ad, form)
        y = torch.full_like(x, float("nan"))
        hb.Product.value(y, B, x)
        assert torch.equal(y, y0), form
    # and the product on the permuted matrix against the oracle
    assert np.array_equal(y0.cpu().numpy(), oracle.spmv(Ap, x.cpu().numpy()))


def test_ordered_copy_edge_cases(hb, oracle):
    from honei_b200._lib import HBError
    # a diagonal matrix: no off-diagonal entries, the order is the identity
    A = P.q1_poisson(2)                       # 4 Dirichlet rows: identity
    Ad = hb.SparseMatrixELL.from_reference(A)
    order, pos, info = Ad.cm_order()
    assert order.cpu().tolist() == [0, 1, 2, 3] and info[0] == 0 and info[2] == -1
    x = torch.from_numpy(P.uniform_vector(4, 1)).cuda()
    y = torch.empty_like(x)
    hb.Product.value(y, Ad.ordered(), x)
    assert torch.equal(y, x)
    # ragged row counts (not a multiple of 4)
    for M in (3, 5, 7):
        A = P.q1_poisson_permuted(M, M)[0]
        Ad = hb.SparseMatrixELL.from_reference(A)
        xh = P.uniform_vector(A.rows, M)
        for form in FORMS:
            y = torch.empty(A.rows, dtype=torch.float64, device="cuda")
            hb.Product.value(y, ordered_form(Ad, form), torch.from_numpy(xh).cuda())
            assert np.array_equal(y.cpu().numpy(), oracle.spmv(A, xh)), (M, form)
    # a rectangular matrix (a prolongation) has no order
    nf, nc, ip, ix, dv = P.prolongation_csr(Mc=5)
    R = hb.SparseMatrixELL.from_reference(P.ell_from_csr(nf, nc, ip, ix, dv))
    with pytest.raises(HBError) as e:
        R.cm_order()
    assert e.value.status == 2


@pytest.mark.parametrize("M", [65, 257])
def test_cg_through_ordered_copy_matches_oracle_on_the_permuted_system(hb, oracle, M):
    """CGSolver on a randomly permuted Q1 system through its ordered copy (b and x permuted in
    once, the solve in the copy's numbering, x permuted back) against the oracle's CG on the
    permuted matrix: iterations within +-1, final true residual within 1e-10."""
    Ap, _ = P.q1_poisson_permuted(M, 3)
    b = oracle.spmv(Ap, P.uniform_vector(Ap.rows, 1))
    x_o, u_o = oracle.cg(Ap, b, eps=1e-8, max_iters=20000)
    O = hb.SparseMatrixELL.from_reference(Ap).ordered(columns=True)
    x = torch.zeros(Ap.rows, dtype=torch.float64, device="cuda")
    u = hb.CGSolver.value(O, None, torch.from_numpy(b).cuda(), x, 20000, 1e-8)
    xg = x.cpu().numpy()
    nb = np.linalg.norm(b)
    rg = np.linalg.norm(oracle.defect(Ap, b, xg)) / nb
    ro = np.linalg.norm(oracle.defect(Ap, b, x_o)) / nb
    print(M, u, u_o, rg, ro)
    assert abs(u - u_o) <= 1, (u, u_o)
    assert abs(rg - ro) <= 1e-10, (rg, ro)
    with pytest.raises(ValueError):
        hb.CGSolver.value(hb.SparseMatrixELL.from_reference(Ap).ordered(columns=False), None,
                          torch.from_numpy(b).cuda(), x, 10, 1e-8)
