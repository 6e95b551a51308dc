"""Host-side generator properties (no GPU)."""
import numpy as np

from honei_b200 import problems as P


def test_variable_coefficient_one_reproduces_constant_stencil():
    for M in (3, 17, 33):
        A1 = P.q1_poisson(M)
        A2 = P.q1_poisson(M, np.ones((M - 1, M - 1)))
        assert np.array_equal(A1.Ax, A2.Ax) and np.array_equal(A1.Aj, A2.Aj)


def test_q1_rows_sum_and_structure():
    M = 9
    A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-2, 1e2, 1))
    ip, ix, dv = A.to_csr()
    ii, jj = np.divmod(np.arange(M * M), M)
    bnd = (ii == 0) | (ii == M - 1) | (jj == 0) | (jj == M - 1)
    counts = np.diff(ip)
    assert np.all(counts[bnd] == 1) and np.all(counts[~bnd] == 9)
    rowsum = np.add.reduceat(dv, ip[:-1])
    assert np.allclose(rowsum[~bnd], 0.0, atol=1e-12 * np.abs(dv).max())
    for r in range(M * M):
        assert np.all(np.diff(ix[ip[r]:ip[r + 1]]) > 0)


def test_ell_layout_threads():
    ip, ix, dv = P.q1_poisson_csr(5)
    for T in (1, 2, 3, 4):
        A = P.ell_from_csr(25, 25, ip, ix, dv, T)
        assert A.stride == 32 * ((25 * T + 31) // 32)
        assert A.ncpr == -(-9 // T)
        ip2, ix2, dv2 = A.to_csr()
        # the packed rows round-trip (thread padding carries explicit zeros at column 0)
        for r in range(25):
            seg = slice(ip2[r], ip2[r + 1])
            keep = dv2[seg] != 0
            assert np.array_equal(ix2[seg][keep], ix[ip[r]:ip[r + 1]])


def test_permutation_is_similarity():
    M = 9
    ip, ix, dv = P.q1_poisson_csr(M)
    A, perm = P.q1_poisson_permuted(M, 3)
    dense = np.zeros((M * M, M * M))
    rows = np.repeat(np.arange(M * M), np.diff(ip))
    dense[rows, ix] = dv
    pd = np.zeros_like(dense)
    pip, pix, pdv = A.to_csr()
    pd[np.repeat(np.arange(M * M), np.diff(pip)), pix] = pdv
    assert np.array_equal(pd[np.ix_(perm, perm)], dense)


def test_prolongation_bilinear_and_restriction_transpose():
    Mc = 5
    nf, nc, ip, ix, dv = P.prolongation_csr(Mc)
    Mf = 2 * Mc - 1
    # interpolating a bilinear function is exact at interior fine nodes
    yc, xc = np.divmod(np.arange(nc), Mc)
    f = 2.0 * xc + 3.0 * yc + 1.0
    rows = np.repeat(np.arange(nf), np.diff(ip))
    fine = np.zeros(nf)
    np.add.at(fine, rows, dv * f[ix])
    yf, xf = np.divmod(np.arange(nf), Mf)
    expect = 2.0 * (xf / 2) + 3.0 * (yf / 2) + 1.0
    bnd = (yf == 0) | (yf == Mf - 1) | (xf == 0) | (xf == Mf - 1)
    assert np.allclose(fine[~bnd], expect[~bnd]) and np.all(fine[bnd] == 0)
    tip, tix, tdv = P.transpose_csr(nf, nc, ip, ix, dv)
    dense = np.zeros((nf, nc))
    dense[rows, ix] = dv
    dt = np.zeros((nc, nf))
    dt[np.repeat(np.arange(nc), np.diff(tip)), tix] = tdv
    assert np.array_equal(dt, dense.T)


def test_mg_hierarchy_sides():
    H = P.mg_hierarchy(65)
    assert H.sides == [9, 17, 33, 65]
    assert [a.rows for a in H.A] == [81, 289, 1089, 4225]
    assert [(p.rows, p.cols) for p in H.prol] == [(289, 81), (1089, 289), (4225, 1089)]


def test_symmetric_form_is_spd_and_consistent():
    import scipy.sparse as sp
    M = 9
    A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-2, 1e2, 2), symmetric=True)
    ip, ix, dv = A.to_csr()
    S = sp.csr_matrix((dv, ix, ip), shape=(A.rows, A.cols)).toarray()
    assert np.array_equal(S, S.T)
    assert np.linalg.eigvalsh(S).min() > 0
    full = P.q1_poisson(M, P.log_uniform_coef(M, 1e-2, 1e2, 2))
    fi, fx, fd = full.to_csr()
    F = sp.csr_matrix((fd, fx, fi), shape=(A.rows, A.cols)).toarray()
    ii, jj = np.divmod(np.arange(M * M), M)
    bnd = (ii == 0) | (ii == M - 1) | (jj == 0) | (jj == M - 1)
    assert np.array_equal(S[np.ix_(~bnd, ~bnd)], F[np.ix_(~bnd, ~bnd)])
    assert np.array_equal(S[bnd], F[bnd])
