"""Pins the plain-C oracle and the problem generators to the reference.

* Always (no HONEI tree needed): against the committed golden fixtures, which hold the
  reference's own outputs (tests/golden/make_golden.py).
* Where oracle/_ref/libhonei_ref.so exists: live, against the reference's CPU path.
Bit-exact comparisons throughout: the oracle restates tags::CPU's arithmetic order.
"""
import dataclasses
import os

import numpy as np
import pytest

from conftest import golden_matrix, load_golden
from honei_b200 import problems as P


def test_q1_generator_matches_reference_construction():
    d = load_golden("q1_small")
    A = P.q1_poisson(33)
    rows, cols, stride, ncpr, T, nnz = (int(v) for v in d["q1_info"])
    assert (A.rows, A.cols, A.stride, A.ncpr, A.threads, A.nnz) == (rows, cols, stride, ncpr, T, nnz)
    assert np.array_equal(A.Aj, d["q1_Aj"])
    assert np.array_equal(A.Ax, d["q1_Ax"])
    assert np.array_equal(A.Arl, d["q1_Arl"])


def test_oracle_spmv_cg_mg_ir_match_reference_q1():
    from oracle.bindings import Oracle
    O = Oracle()
    d = load_golden("q1_small")
    A = P.q1_poisson(33)
    assert np.array_equal(O.spmv(A, d["spmv_x"]), d["spmv_y64"])
    A32 = A.astype(np.float32)
    assert np.array_equal(O.spmv(A32, d["spmv_x"].astype(np.float32)), d["spmv_y32"])
    b = d["b"]
    x, used = O.cg(A, b, eps=1e-8)
    assert used == int(d["cg_used64"]) and np.array_equal(x, d["cg_x64"])
    x, used = O.cg(A32, b.astype(np.float32), eps=1e-5)
    assert used == int(d["cg_used32"]) and np.array_equal(x, d["cg_x32"])
    H = P.mg_hierarchy(33)
    x, used = O.mg(H, b, eps=1e-8)
    assert used == int(d["mg_used64"]) and np.array_equal(x, d["mg_x64"])
    H32 = H.astype(np.float32)
    x, used = O.mg(H32, b.astype(np.float32), eps=1e-5)
    assert used == int(d["mg_used32"]) and np.array_equal(x, d["mg_x32"])
    x, used, _ = O.ir_mg(H.A[-1], H32, b, eps=1e-10, inner_eps=1e-3, warm_start=True)
    assert used == int(d["ir_used"]) and np.array_equal(x, d["ir_x"])


def test_oracle_matches_reference_permuted_and_variable_coefficient():
    from oracle.bindings import Oracle
    O = Oracle()
    d = load_golden("q1_small")
    Ap, perm = P.q1_poisson_permuted(33, 7)
    assert np.array_equal(perm, d["perm"])
    assert np.array_equal(O.spmv(Ap, d["spmv_x"]), d["perm_spmv_y"])
    bp = np.empty_like(d["b"])
    bp[perm] = d["b"]
    x, used = O.cg(Ap, bp, eps=1e-8)
    assert used == int(d["perm_cg_used"]) and np.array_equal(x, d["perm_cg_x"])
    Av = P.q1_poisson(33, P.log_uniform_coef(33, 1e-2, 1e2, 5))
    x, used = O.cg(Av, d["var_b"], eps=1e-8)
    assert used == int(d["var_cg_used"]) and np.array_equal(x, d["var_cg_x"])


def test_oracle_cg_257_iteration_count_and_solution():
    """The plain FP64 CG workload on 257^2 (566-578 iterations with the reference)."""
    from oracle.bindings import Oracle
    O = Oracle()
    d = load_golden("q1_small")
    A = P.q1_poisson(257)
    b = O.spmv(A, P.uniform_vector(A.rows, 1))
    x, used = O.cg(A, b, eps=1e-8)
    assert used == int(d["cg257_used"])
    assert np.array_equal(x[::97], d["cg257_x_sample"])
    assert x.sum() == float(d["cg257_x_sum"])


def test_oracle_featflow_fixture(featflow):
    """MGSolverTest data (poisson_advanced4): reference MG/CG/SpMV/defect results, and the
    FEATFLOW2 solution sol_4 within the reference test's own tolerance (8e-3, mg_TEST.cc)."""
    from oracle.bindings import Oracle
    O = Oracle()
    H, d = featflow
    A4 = H.A[-1]
    assert np.array_equal(O.spmv(A4, d["spmv_x"]), d["spmv_y"])
    assert np.array_equal(O.defect(A4, d["rhs_4"], d["spmv_x"]), d["defect_r"])
    x, used = O.cg(A4, d["rhs_4"], d["init_4"], eps=1e-8)
    assert used == int(d["cg_used"]) and np.array_equal(x, d["cg_x"])
    x, used = O.mg(H, d["rhs_4"], d["init_4"], damping=0.7, eps=1e-8, max_iters=100)
    assert used == int(d["mg_used"]) and np.array_equal(x, d["mg_x"])
    assert np.max(np.abs(x - d["sol_4"])) < 8e-3


def test_oracle_defect_fixture():
    from oracle.bindings import Oracle
    O = Oracle()
    d = load_golden("defect_5pt")
    A = golden_matrix(d, "A")
    assert np.array_equal(O.spmv(A, d["x"]), d["y"])
    assert np.array_equal(O.defect(A, d["b"], d["x"]), d["r"])


def test_oracle_threads_layout_matches_reference(reference):
    """T > 1 lanes per row (ell::threads): the oracle's SpMV follows the reference order."""
    from oracle.bindings import Oracle
    O = Oracle()
    ip, ix, dv = P.q1_poisson_csr(17)
    for T in (1, 2, 3, 4, 16):
        A = P.ell_from_csr(289, 289, ip, ix, dv, T)
        x = P.uniform_vector(289, T)
        y_ref, _ = reference.spmv(A, x)
        assert np.array_equal(O.spmv(A, x), y_ref)


def test_oracle_live_against_reference(reference):
    from oracle.bindings import Oracle
    O = Oracle()
    for M in (3, 9, 65):
        Ar = reference.q1_poisson(M)
        A = P.q1_poisson(M)
        assert np.array_equal(A.Aj, Ar.Aj) and np.array_equal(A.Ax, Ar.Ax) and np.array_equal(A.Arl, Ar.Arl)
    A = P.q1_poisson(65, P.log_uniform_coef(65, 1e-1, 1e1, 3))
    b = O.spmv(A, P.uniform_vector(A.rows, 9))
    for dt, eps in ((np.float64, 1e-8), (np.float32, 1e-5)):
        Ad = A.astype(dt)
        bd = b.astype(dt)
        x1, u1 = O.cg(Ad, bd, eps=eps)
        x2, u2, _ = reference.cg(Ad, bd, eps=eps)
        assert u1 == u2 and np.array_equal(x1, x2)
        assert O.dot(bd, bd) == reference.dot(bd, bd)
    H = P.mg_hierarchy(65, coef=P.log_uniform_coef(65, 1e-1, 1e1, 3))
    x1, u1 = O.mg(H, b)
    x2, u2, _ = reference.mg(H, b)
    assert u1 == u2 and np.array_equal(x1, x2)


def test_oracle_multicore_tags_agree_on_iterations(reference):
    """The reference's own tags agree with tags::CPU on the CG iteration count (orientation
    for the +-1 iteration tolerance used against the GPU)."""
    A = P.q1_poisson(65)
    b, _ = reference.spmv(A, P.uniform_vector(A.rows, 1))
    counts = {tag: reference.cg(A, b, tag=tag)[1] for tag in ("cpu", "generic", "sse", "mc-sse")}
    assert max(counts.values()) - min(counts.values()) <= 1, counts


def test_oracle_multicore_mg_and_ir_agree_with_cpu_tag(reference):
    """MultiCore::SSE (the tag the full-size GPU comparisons use) takes tags::CPU's cycle and
    outer-step counts for MG and for IRSolver, and reaches the same residual."""
    reference.set_threads(os.cpu_count() or 1)
    H = P.mg_hierarchy(33, coef=P.log_uniform_coef(33, 1e-2, 1e2, 7))
    A = H.A[-1]
    b, _ = reference.spmv(A, P.uniform_vector(A.rows, 2))
    runs = {t: reference.mg(H, b, eps=1e-8, max_iters_coarse=100, tag=t) for t in ("cpu", "mc-sse")}
    assert runs["cpu"][1] == runs["mc-sse"][1]
    assert np.allclose(runs["cpu"][0], runs["mc-sse"][0], rtol=0, atol=1e-9 * np.abs(runs["cpu"][0]).max())
    H32 = H.astype(np.float32)
    irs = {t: reference.ir_mg(H, H32, b, eps=1e-10, inner_eps=1e-3, max_iters_coarse=100, tag=t)
           for t in ("cpu", "mc-sse")}
    assert abs(irs["cpu"][1] - irs["mc-sse"][1]) <= 1
    r = {t: np.linalg.norm(reference.defect(A, b, irs[t][0])) / np.linalg.norm(b) for t in irs}
    assert r["cpu"] < 1e-10 and r["mc-sse"] < 1e-10, r


def test_batch512_fixture_matches_oracle_and_reference():
    """The 512-system batch fixture (tests/golden/batch512.npz, CGSolver<tags::CPU> and
    <tags::CPU::SSE> counts): the oracle reproduces tags::CPU's count and residual on a sample of
    the systems, and, where the compiled reference is present, its SSE tag the stored SSE count."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.bindings import REF_SO, Oracle, Reference
    O = Oracle()
    g = load_golden("batch512")
    seed = 2024
    sides = np.random.default_rng(seed).integers(17, 258, size=512)
    assert np.array_equal(sides, g["sides"])
    sample = [int(i) for i in np.argsort(sides)[::37]]        # 14 systems across the size range

    def system(i):
        M = int(sides[i])
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, seed + i), symmetric=True)
        return A, O.spmv(A, P.uniform_vector(M * M, seed + i + 1))

    def run(i):
        A, b = system(i)
        x, u = O.cg(A, b, eps=1e-8, max_iters=100000)
        return u, np.linalg.norm(O.defect(A, b, x)) / np.linalg.norm(b)

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        out = list(ex.map(run, sample))
    for i, (u, r) in zip(sample, out):
        assert u == g["cpu_used"][i] and r == g["cpu_relres"][i], (i, u, g["cpu_used"][i])
    if os.path.exists(REF_SO):
        R = Reference()
        for i in sample[:4]:
            A, b = system(i)
            assert R.cg(A, b, eps=1e-8, max_iters=100000, tag="sse")[1] == g["sse_used"][i]


# ---- BandedMatrixQx<Q1Type> ----------------------------------------------------------------
def test_oracle_q1band_matches_reference_fixture(oracle):
    from conftest import q1band_test_data
    g = load_golden("q1band")
    for level in (2, 5):
        size = (2 ** level + 1) ** 2
        for name, dt in (("f64", np.float64), ("f32", np.float32)):
            bands, x = q1band_test_data(size, dt)
            assert np.array_equal(oracle.q1band_spmv(bands, x), g[f"test_L{level}_{name}_y"]), (level, name)
    assert np.array_equal(np.stack(oracle.q1band_poisson(33)), g["poisson_bands"])
    vb = list(g["var_bands"])
    assert np.array_equal(oracle.q1band_spmv(vb, g["var_x"]), g["var_y64"])
    assert np.array_equal(oracle.q1band_spmv([v.astype(np.float32) for v in vb], g["var_x"].astype(np.float32)),
                          g["var_y32"])
    assert np.array_equal(oracle.q1band_defect(vb, g["var_b"], g["var_x"]), g["var_r64"])


def test_oracle_q1band_live_against_reference(oracle, reference):
    """Random bands on square and non-square sizes: tags::CPU bit for bit; on the sizes the
    reference's own tests use, (2^L + 1)^2, its SSE and MultiCore::SSE tags agree to rounding
    (the SSE kernel does not handle a single row)."""
    from conftest import q1band_used_mask
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 9, 50, 289, 1000, 4225):
        for dt in (np.float64, np.float32):
            bands = [rng.uniform(-1, 1, n).astype(dt) for _ in range(9)]
            x = rng.uniform(-1, 1, n).astype(dt)
            y_o = oracle.q1band_spmv(bands, x)
            y_r, _ = reference.q1band_spmv(bands, x, tag="cpu")
            assert np.array_equal(y_o, y_r), (n, dt)
            tol = 1e-13 if dt == np.float64 else 1e-5
            for tag in (("sse", "mc-sse") if n in (9, 289, 4225) else ()):
                y_t, _ = reference.q1band_spmv(bands, x, tag=tag)
                assert np.allclose(y_t, y_r, rtol=tol, atol=tol), (n, dt, tag)
        b = rng.uniform(-1, 1, n)
        bands64 = [rng.uniform(-1, 1, n) for _ in range(9)]
        assert np.array_equal(oracle.q1band_defect(bands64, b, x.astype(np.float64)),
                              reference.q1band_defect(bands64, b, x.astype(np.float64)))
    # the conversion from ELL reproduces the banded Poisson fill on every entry the product reads
    conv = np.stack(reference.q1band_from_ell(P.q1_poisson(33)))
    fill = np.stack(oracle.q1band_poisson(33))
    mask = q1band_used_mask(33 * 33)
    assert np.array_equal(conv[mask], fill[mask])


# ---- CGSolver<methods::VAR> --------------------------------------------------------------
def _featflow_eps(digits=3, add=2, size=8):
    """The FEATFLOW comparison tolerance of honei/math/cg_TEST.cc:200-210 (3e-5 for double)."""
    base = 1 / 10 ** digits
    m = (base / 10 ** add - base) / 4
    return 3 * (m * size + base - 4 * m)


def test_oracle_cg_var_matches_reference_fixture(oracle):
    g = load_golden("pcg")
    A = golden_matrix(g, "q_A")
    x, used = oracle.cg_var(A, g["q_P"], g["q_rhs"], x0=g["q_init"], max_iters=700, eps=1e-8)
    assert used == int(g["q_used"]) and np.array_equal(x, g["q_x"])
    assert np.abs(x - g["q_sol"]).max() <= _featflow_eps()
    f = load_golden("featflow_pa4")
    A4 = golden_matrix(f, "A_4")
    for kind in ("sainv", "spai"):
        Pm = golden_matrix(g, f"a4_{kind}")
        x, used = oracle.cg_var(A4, Pm, f["rhs_4"], x0=f["init_4"], max_iters=700, eps=1e-8)
        assert used == int(g[f"a4_{kind}_used"]), kind
        assert np.array_equal(x, g[f"a4_{kind}_x"]), kind


def test_oracle_cg_var_live_against_reference(oracle, reference):
    for M, dt, eps in ((17, np.float64, 1e-8), (33, np.float64, 1e-8), (33, np.float32, 1e-5)):
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, M)).astype(dt)
        ip, ix, dv = A.to_csr()
        diag = np.array([dv[ip[i]:ip[i + 1]][ix[ip[i]:ip[i + 1]] == i][0] for i in range(A.rows)])
        Pd = (dt(0.7) / diag).astype(dt)
        b = oracle.spmv(A, P.uniform_vector(A.rows, 2).astype(dt))
        xo, uo = oracle.cg_var(A, Pd, b, max_iters=700, eps=eps)
        xr, ur, _ = reference.cg_var(A, Pd, b, max_iters=700, eps=eps)
        assert uo == ur and np.array_equal(xo, xr), (M, dt)
        Pm = P.ell_from_csr(A.rows, A.rows, np.arange(A.rows + 1), np.arange(A.rows), Pd, 1, dt)
        xo2, uo2 = oracle.cg_var(A, Pm, b, max_iters=700, eps=eps)
        xr2, ur2, _ = reference.cg_var(A, Pm, b, max_iters=700, eps=eps)
        assert uo2 == ur2 and np.array_equal(xo2, xr2) and np.array_equal(xo2, xo)


# ---- geometric transfers (Prolongation / Restriction<methods::NONE>) ---------------------
MASKS = [[2] * 8, [0] * 8, [2, 0, 2, 0, 2, 2, 0, 0], [0, 2, 0, 2, 0, 0, 2, 2]]


def test_oracle_geometric_transfers_match_reference(oracle, reference):
    rng = np.random.default_rng(8)
    for side in (3, 5, 9, 17, 33, 65):
        nf, nc = side * side, ((side - 1) // 2 + 1) ** 2
        for dt in (np.float64, np.float32):
            for mask in MASKS:
                c = rng.uniform(-1, 1, nc).astype(dt)
                f = rng.uniform(-1, 1, nf).astype(dt)
                assert np.array_equal(oracle.prolongate(c, mask, nf), reference.prolongate(c, mask, nf)), (side, dt)
                assert np.array_equal(oracle.restrict(f, mask), reference.restrict(f, mask)), (side, dt)


def test_geometric_transfers_are_the_bilinear_pair():
    """Away from the masked boundary the geometric prolongation is the bilinear interpolation of
    the PROLMAT matrices, and the restriction is its transpose."""
    from oracle.bindings import Oracle
    O = Oracle()
    side = 17
    nf, ncs = side * side, (side - 1) // 2 + 1
    nfp, ncp, ip, ix, dv = P.prolongation_csr(Mf=side)
    Pm = np.zeros((nfp, ncp))
    for r in range(nfp):
        Pm[r, ix[ip[r]:ip[r + 1]]] = dv[ip[r]:ip[r + 1]]
    c = P.uniform_vector(ncs * ncs, 1)
    f = P.uniform_vector(nf, 2)
    mask = [2] * 8
    assert np.allclose(O.prolongate(c, mask, nf), Pm @ c, rtol=0, atol=1e-15)
    interior = np.ones(ncs * ncs, bool)
    for k in range(ncs * ncs):
        i, j = divmod(k, ncs)
        interior[k] = 0 < i < ncs - 1 and 0 < j < ncs - 1
    fi = f.copy()
    fr = np.arange(nf)
    fi[(fr // side == 0) | (fr // side == side - 1) | (fr % side == 0) | (fr % side == side - 1)] = 0
    assert np.allclose(O.restrict(fi, mask)[interior], (Pm.T @ fi)[interior], rtol=0, atol=1e-14)


# ---- SparseMatrixCSR ------------------------------------------------------------------------
def test_oracle_csr_matches_reference_fixture(oracle):
    """The reference's CSR product test cases (csr::blocksize 1..8, size x (size + 3)), its
    ELL -> CSR conversion of Q1 33^2 with product and defect, and a random rectangular pattern
    with empty rows: the host converter rebuilds the reference's arrays, the oracle its
    results, bit for bit."""
    from conftest import golden_csr
    g = load_golden("csr")
    for bs in (1, 2, 4, 8):
        for size in (11, 44, 176):
            k = f"t{bs}_{size}"
            A = golden_csr(g, k)
            ip, ix, dv, x = P.csr_product_test_matrix(size)
            C = P.csr_blocked(size, size + 3, ip, ix, dv, bs)
            assert np.array_equal(C.Ar, A.Ar) and np.array_equal(C.Aj, A.Aj) and np.array_equal(C.Ax, A.Ax)
            assert C.used == A.used and np.array_equal(x, g[k + "_x"])
            assert np.array_equal(oracle.csr_spmv(A, x), g[k + "_y"]), k
    E = P.q1_poisson(33)
    for bs in (1, 4):
        k = f"q1_{bs}"
        A = golden_csr(g, k)
        C = P.csr_from_ell(E, bs)
        assert np.array_equal(C.Ar, A.Ar) and np.array_equal(C.Aj, A.Aj) and np.array_equal(C.Ax, A.Ax)
        assert np.array_equal(oracle.csr_spmv(A, g[k + "_x"]), g[k + "_y"])
        assert np.array_equal(oracle.csr_defect(A, g[k + "_b"], g[k + "_x"]), g[k + "_r"])
    for bs in (1, 3, 8):
        k = f"rand_{bs}"
        A = golden_csr(g, k)
        assert np.array_equal(oracle.csr_spmv(A, g[k + "_x"]), g[k + "_y"])
        A32 = A.astype(np.float32)
        assert np.array_equal(oracle.csr_spmv(A32, g[k + "_x"].astype(np.float32)), g[k + "_y32"])


def test_oracle_csr_live_against_reference(oracle, reference):
    """Random CSR patterns (block sizes 1, 2, 5, 8, square and rectangular, empty rows) and the
    ELL -> CSR conversion of Q1 grids: tags::CPU bit for bit.  The Generic and MultiCore::SSE
    tags agree to rounding where no block reaches past the last column; where one does, their
    loops read x beyond its end (only tags::CPU tests the column bound), so they are not
    compared there."""
    rng = np.random.default_rng(5)
    for rows, cols, fill in ((1, 1, 1.0), (37, 53, 0.1), (200, 200, 0.03), (513, 300, 0.02)):
        mask = rng.random((rows, cols)) < fill
        if rows > 5:
            mask[rng.choice(rows, rows // 5, replace=False)] = False
        ri, ci = np.nonzero(mask)
        ip = np.zeros(rows + 1, np.int64)
        np.cumsum(np.bincount(ri, minlength=rows), out=ip[1:])
        dv = rng.uniform(-1, 1, len(ci))
        for bs in (1, 2, 5, 8):
            for dt in (np.float64, np.float32):
                A = P.csr_blocked(rows, cols, ip, ci, dv, bs, dt)
                x = rng.uniform(-1, 1, cols).astype(dt)
                b = rng.uniform(-1, 1, rows).astype(dt)
                y_r, _ = reference.csr_spmv(A, x, tag="cpu")
                assert np.array_equal(oracle.csr_spmv(A, x), y_r), (rows, cols, bs, dt)
                assert np.array_equal(oracle.csr_defect(A, b, x), reference.csr_defect(A, b, x, tag="cpu"))
                tol = 1e-12 if dt == np.float64 else 1e-4
                for tag in (("generic", "mc-sse") if cols % bs == 0 else ()):
                    y_t, _ = reference.csr_spmv(A, x, tag=tag)
                    assert np.allclose(y_t, y_r, rtol=tol, atol=tol), (rows, cols, bs, dt, tag)
    for M in (9, 65):
        E = P.q1_poisson(M)
        for bs in (1, 2, 4):
            A = reference.csr_from_ell(E, bs)
            C = P.csr_from_ell(E, bs)
            assert np.array_equal(C.Ar, A.Ar) and np.array_equal(C.Aj, A.Aj) and np.array_equal(C.Ax, A.Ax)


# ---- SPAI2 (honei/math/spai2.hh:129-260) --------------------------------------------------
def spai2_cases():
    """(name, A, stored SPAI matrix of the reference's testdata or None) of spai2.npz."""
    g, f, p = load_golden("spai2"), load_golden("featflow_pa4"), load_golden("pcg")
    return g, [("q2a2", golden_matrix(g, "q2a2"), golden_matrix(g, "q2a2_file")),
               ("pa_a4", golden_matrix(g, "pa_a4"), golden_matrix(g, "pa_a4_file")),
               ("pa4_a4", golden_matrix(f, "A_4"), golden_matrix(p, "a4_spai")),
               ("q1", golden_matrix(g, "q1"), None)]


def test_oracle_spai2_matches_reference_fixture(oracle):
    """The restatement equals SPAI2<tags::CPU::SSE> bit for bit on the FEATFLOW matrices (Q2 with
    25 entries per row, Q1 levels) and Q1 33^2, FP64 and FP32; and the reference's own stored
    A_*_spai.ell files are SPAI2 of their matrices: same pattern, values within 1e-13."""
    g, cases = spai2_cases()
    for name, A, stored in cases:
        for dt, suf in ((np.float64, "64"), (np.float32, "32")):
            B = A.astype(dt)
            M = dataclasses.replace(B, Ax=oracle.spai2(B))
            assert np.array_equal(M.to_csr()[2], g[f"{name}_M{suf}"]), (name, suf)
        if stored is not None:
            ip, ix, dv = dataclasses.replace(A, Ax=oracle.spai2(A)).to_csr()
            sp, sx, sv = stored.to_csr()
            assert np.array_equal(ip, sp) and np.array_equal(ix, sx), name
            assert np.abs(dv - sv).max() <= 1e-13, name


def test_oracle_spai2_is_a_better_inverse_than_jacobi(oracle):
    """The reference's own SPAI2 test property (honei/math/spai2_TEST.cc:47-77):
    ||I - A M||_1 (entrywise) below ||I - A diag(A)^-1||_1, on its Q2 matrix."""
    _, cases = spai2_cases()
    A = cases[0][1]
    ip, ix, dv = A.to_csr()
    Ad = np.zeros((A.rows, A.cols))
    Ad[np.repeat(np.arange(A.rows), np.diff(ip)), ix] = dv
    _, mx, mv = dataclasses.replace(A, Ax=oracle.spai2(A)).to_csr()
    Md = np.zeros_like(Ad)
    Md[np.repeat(np.arange(A.rows), np.diff(ip)), mx] = mv
    eye = np.eye(A.rows)
    assert np.abs(eye - Ad @ Md).sum() < np.abs(eye - Ad @ np.diag(1 / np.diag(Ad))).sum()


def test_oracle_spai2_live_against_reference(oracle, reference):
    """Live, against the compiled reference: natural, permuted, variable-coefficient and
    threads = 4 layouts, FP64 and FP32, the SSE and MultiCore::SSE tags; and a column range
    (the col_start / col_end arguments) changes only its own columns."""
    cases = [P.q1_poisson(17), P.q1_poisson_permuted(17, 2)[0], P.q1_poisson(17, P.log_uniform_coef(17, 1e-2, 1e2, 3)),
             P.ell_from_csr(289, 289, *P.q1_poisson_csr(17), threads=4)]
    for A in cases:
        for dt in (np.float64, np.float32):
            B = A.astype(dt)
            Mr, _ = reference.spai2(B, "sse")
            assert np.array_equal(oracle.spai2(B), Mr)
    Mr, _ = reference.spai2(cases[1], "mc-sse")
    assert np.array_equal(oracle.spai2(cases[1]), Mr)
    # an empty row and column, a column whose system is empty (n1 == 0: M keeps A's value), 1 x 1
    for E in (P.ell_from_csr(3, 3, np.array([0, 0, 1, 2]), np.array([0, 2]), np.array([5.0, 2.0])),
              P.ell_from_csr(1, 1, np.array([0, 1]), np.array([0]), np.array([4.0]))):
        Mr, _ = reference.spai2(E, "sse")
        assert np.array_equal(oracle.spai2(E), Mr)
    A = cases[0]
    full = oracle.spai2(A)
    part = oracle.spai2(A, 40, 90)
    inside = np.isin(A.Aj.astype(np.int64), np.arange(40, 90)) & (A.Ax != 0)
    assert np.array_equal(part[inside], full[inside]) and np.array_equal(part[~inside], A.Ax[~inside])
    assert not np.array_equal(part[inside], A.Ax[inside])
