"""Generates the committed golden fixtures from the reference itself.

Run where the HONEI tree and oracle/_ref/libhonei_ref.so exist (``make -C oracle ref``):

    python tests/golden/make_golden.py [/path/to/honei-tree]

Outputs (all numbers come from the reference's own CPU path, tags::CPU, through
oracle/ref_shim.cc; the FEATFLOW2 matrices and vectors are read with the reference's own
readers, honei/math/matrix_io.hh and honei/math/vector_io.hh):

* featflow_pa4.npz -- the MGSolverTest fixture (honei/math/mg_TEST.cc:224-365, data
  honei/math/testdata/poisson_advanced4/sort_0): A_1..A_4, prol_2..prol_4, rhs_4, init_4,
  sol_4, stored as CSR; plus the reference's results on them: V(2,2) MG with the "jac"
  smoother (damping 0.7) and a CG coarse solver, CG on A_4, SpMV and defect of A_4.
* defect_5pt.npz -- honei/math/testdata/5pt_10x10.ell (defect_TEST.cc) with a seeded
  SpMV/defect evaluated by the reference.
* q1_small.npz -- the reference's own Q1 Poisson construction (FillMatrix -> SparseMatrix ->
  SparseMatrixELL) at 33^2, with SpMV/CG/MG/IR results, FP64 and FP32, natural, permuted and
  variable-coefficient variants, plus CG iteration counts at 257^2.
* q1band.npz -- BandedMatrixQx<Q1Type>: the data of the reference's banded product test
  (honei/la/product_TEST.cc:189-244, bands (i + k) % 311) at levels 2 and 5, FP32 and FP64,
  with Product<tags::CPU> results; the banded Poisson fill at 33^2
  (honei/math/fill_matrix.hh:41-77); the banded form of a variable-coefficient Q1 ELL matrix
  by the reference's conversion (banded_matrix_qx-impl.hh:111-167) with a seeded product and
  defect.

* pcg.npz -- CGSolver<tags::CPU, methods::VAR>: the Jacobi-preconditioned test of
  honei/math/cg_TEST.cc:359-440 (testdata/poisson A_6, rhs_6, init_6, P = 0.7 / diag(A),
  700 iterations, eps 1e-8) with FEATFLOW's sol_6, and the SAINV / SPAI preconditioned solves of
  poisson_advanced4/sort_0 A_4 (A_4_sainv.ell, A_4_spai.ell; rhs_4, init_4), each with the
  reference's solution and iteration count (A_4, rhs_4, init_4 live in featflow_pa4.npz).

* spai2.npz -- SPAI2<tags::CPU::SSE> (honei/math/spai2.hh:129-260, the tag the reference's
  spai2_TEST.cc runs) of poisson_advanced/q2_sort_0/A_2 (Q2, 25 entries per row),
  poisson_advanced/sort_0/A_4 and poisson_advanced4/sort_0/A_4 (matrix in featflow_pa4.npz),
  FP64 and FP32, each with the reference's stored A_*_spai.ell beside it (pcg.npz for the
  last), and of the reference's Q1 33^2 construction.

* batch512.npz -- the 512-system batch workload (SPD Q1 systems, side U{17..257} from seed 2024,
  cellwise coefficient 10^U(-1,1) with seed 2024 + i, x_true U[-1,1] with seed 2024 + i + 1,
  b = A x_true): for every system, the iteration count and final true relative residual of
  CGSolver<tags::CPU, NONE>, of CGSolver<tags::CPU::SSE, NONE> and of
  CGSolver<tags::CPU::MultiCore::SSE, NONE> on 4 and on 16 threads (eps 1e-8, x0 = 0).  The tags
  differ only in the summation order of their dot products; their spread is the measured
  sensitivity of these solves to that order.  Needs only oracle/_ref (no HONEI tree).  An
  existing file keeps the columns it has; missing ones are added.

    python tests/golden/make_golden.py [/path/to/honei-tree] [--only q1band|pcg|csr|spai2|batch512]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from honei_b200 import problems as P  # noqa: E402
from oracle.bindings import Reference  # noqa: E402


def csr_of(A):
    ip, ix, dv = A.to_csr()
    return ip.astype(np.int64), ix.astype(np.int32), dv.astype(np.float64)


def put_matrix(out, name, A):
    ip, ix, dv = csr_of(A)
    out[f"{name}_shape"] = np.array([A.rows, A.cols], np.int64)
    out[f"{name}_indptr"] = ip
    out[f"{name}_indices"] = ix
    out[f"{name}_data"] = dv


def product_test_bands(size: int, dtype):
    """The vectors of Q1MatrixDenseVectorProductTest (honei/la/product_TEST.cc:196-219): x and
    the bands (dv3, dv2, dv4, dv2, dv3, dv4, dv4, dv3, dv2), v_k[i] = (i + k) % 311."""
    i = np.arange(size)
    dv = {k: ((i + k) % 311).astype(dtype) for k in (1, 2, 7, 25)}
    dv1, dv2, dv3, dv4 = dv[2], dv[1], dv[25], dv[7]
    return [dv3, dv2, dv4, dv2, dv3, dv4, dv4, dv3, dv2], dv1


def banded(R) -> None:
    out = {}
    for level in (2, 5):
        size = (2 ** level + 1) ** 2
        for name, dt in (("f64", np.float64), ("f32", np.float32)):
            bands, x = product_test_bands(size, dt)
            y, _ = R.q1band_spmv(bands, x, tag="cpu")
            out[f"test_L{level}_{name}_y"] = y
    M = 33
    out["poisson_bands"] = np.stack(R.q1band_poisson(M))
    coef = P.log_uniform_coef(M, 1e-2, 1e2, 4)
    A = P.q1_poisson(M, coef)
    out["var_coef"] = coef
    bands = R.q1band_from_ell(A)
    # the conversion leaves band entries whose column lies outside [0, n) as allocated
    # (uninitialised); the product never reads them.  Zero them for a stable fixture.
    n, root = M * M, M
    offs = [-root - 1, -root, -root + 1, -1, 0, 1, root - 1, root, root + 1]
    r = np.arange(n)
    for k, o in enumerate(offs):
        bands[k][(r + o < 0) | (r + o >= n)] = 0.0
    out["var_bands"] = np.stack(bands)
    x = P.uniform_vector(M * M, 6)
    b = P.uniform_vector(M * M, 8)
    out["var_x"], out["var_b"] = x, b
    out["var_y64"], _ = R.q1band_spmv(bands, x, tag="cpu")
    out["var_y32"], _ = R.q1band_spmv([v.astype(np.float32) for v in bands], x.astype(np.float32), tag="cpu")
    out["var_r64"] = R.q1band_defect(bands, b, x)
    np.savez_compressed(os.path.join(HERE, "q1band.npz"), **out)


def pcg(R, tree: str) -> None:
    td = os.path.join(tree, "honei", "math", "testdata")
    out = {}
    base = os.path.join(td, "poisson") + "/"
    A = R.read_ell(base + "A_6.ell")
    put_matrix(out, "q_A", A)
    rhs, init, sol = (R.read_exp(base + f"{v}_6") for v in ("rhs", "init", "sol"))
    out["q_rhs"], out["q_init"], out["q_sol"] = rhs, init, sol
    ip, ix, dv = A.to_csr()
    diag = np.array([dv[ip[i]:ip[i + 1]][ix[ip[i]:ip[i + 1]] == i][0] for i in range(A.rows)])
    out["q_P"] = 0.7 / diag
    x, used, _ = R.cg_var(A, out["q_P"], rhs, x0=init, max_iters=700, eps=1e-8)
    out["q_x"], out["q_used"] = x, np.array(used)
    base = os.path.join(td, "poisson_advanced4", "sort_0") + "/"
    # A_4, rhs_4 and init_4 are in featflow_pa4.npz already
    A4 = R.read_ell(base + "A_4.ell")
    rhs4, init4 = R.read_exp(base + "rhs_4"), R.read_exp(base + "init_4")
    for kind in ("sainv", "spai"):
        Pm = R.read_ell(base + f"A_4_{kind}.ell")
        put_matrix(out, f"a4_{kind}", Pm)
        x, used, _ = R.cg_var(A4, Pm, rhs4, x0=init4, max_iters=700, eps=1e-8)
        out[f"a4_{kind}_x"], out[f"a4_{kind}_used"] = x, np.array(used)
    np.savez_compressed(os.path.join(HERE, "pcg.npz"), **out)


def spai2(R, tree: str) -> None:
    """SPAI2 of the FEATFLOW matrices and of Q1 33^2: M's values in the CSR order of A (M has
    A's pattern), FP64 and FP32, plus the reference's stored SPAI matrix of each file."""
    import dataclasses
    td = os.path.join(tree, "honei", "math", "testdata")
    out = {}
    for name, path in (("q2a2", "poisson_advanced/q2_sort_0/A_2"), ("pa_a4", "poisson_advanced/sort_0/A_4"),
                       ("pa4_a4", "poisson_advanced4/sort_0/A_4")):
        A = R.read_ell(os.path.join(td, path + ".ell"))
        if name != "pa4_a4":    # A_4 is in featflow_pa4.npz, its A_4_spai.ell in pcg.npz
            put_matrix(out, name, A)
            put_matrix(out, name + "_file", R.read_ell(os.path.join(td, path + "_spai.ell")))
        for dt, suf in ((np.float64, "64"), (np.float32, "32")):
            B = A.astype(dt)
            Mx, _ = R.spai2(B, "sse")
            out[f"{name}_M{suf}"] = dataclasses.replace(B, Ax=Mx).to_csr()[2]
    Aq = R.q1_poisson(33)
    put_matrix(out, "q1", Aq)
    for dt, suf in ((np.float64, "64"), (np.float32, "32")):
        B = Aq.astype(dt)
        Mx, _ = R.spai2(B, "sse")
        out[f"q1_M{suf}"] = dataclasses.replace(B, Ax=Mx).to_csr()[2]
    np.savez_compressed(os.path.join(HERE, "spai2.npz"), **out)


def csr(R) -> None:
    """SparseMatrixCSR: the reference's own CSR product test cases (product_TEST.cc:917-958,
    csr::blocksize 1, 2, 4, 8), the reference's ELL -> CSR conversion of Q1 33^2 with its
    product and defect, and a rectangular random pattern with empty rows and a ragged last
    block, each with tags::CPU results."""
    out = {}
    for bs in (1, 2, 4, 8):
        for size in (11, 44, 176):
            A, x, y = R.csr_product_test(size, bs)
            k = f"t{bs}_{size}"
            out[k + "_Ar"], out[k + "_Aj"], out[k + "_Ax"] = A.Ar, A.Aj, A.Ax
            out[k + "_info"] = np.array([A.rows, A.cols, A.blocksize, A.used], np.uint64)
            out[k + "_x"], out[k + "_y"] = x, y
    E = R.q1_poisson(33)
    for bs in (1, 4):
        A = R.csr_from_ell(E, bs)
        x = P.uniform_vector(A.cols, 7)
        b = P.uniform_vector(A.rows, 8)
        k = f"q1_{bs}"
        out[k + "_Ar"], out[k + "_Aj"], out[k + "_Ax"] = A.Ar, A.Aj, A.Ax
        out[k + "_info"] = np.array([A.rows, A.cols, A.blocksize, A.used], np.uint64)
        out[k + "_x"], out[k + "_b"] = x, b
        out[k + "_y"] = R.csr_spmv(A, x)[0]
        out[k + "_r"] = R.csr_defect(A, b, x)
    rng = np.random.default_rng(11)
    rows, cols = 300, 257
    mask = rng.random((rows, cols)) < 0.05
    mask[rng.choice(rows, 20, replace=False)] = False          # empty rows
    mask[:, cols - 1] |= rng.random(rows) < 0.3                # last column: ragged last blocks
    ri, ci = np.nonzero(mask)
    ip = np.zeros(rows + 1, np.int64)
    np.cumsum(np.bincount(ri, minlength=rows), out=ip[1:])
    dv = rng.uniform(-1, 1, len(ci))
    for bs in (1, 3, 8):
        A = P.csr_blocked(rows, cols, ip, ci, dv, bs)
        x = rng.uniform(-1, 1, cols)
        k = f"rand_{bs}"
        out[k + "_Ar"], out[k + "_Aj"], out[k + "_Ax"] = A.Ar, A.Aj, A.Ax
        out[k + "_info"] = np.array([A.rows, A.cols, A.blocksize, A.used], np.uint64)
        out[k + "_x"] = x
        out[k + "_y"] = R.csr_spmv(A, x)[0]
        out[k + "_y32"] = R.csr_spmv(A.astype(np.float32), x.astype(np.float32))[0]
    np.savez_compressed(os.path.join(HERE, "csr.npz"), **out)


def main(tree: str, only: str | None = None) -> None:
    R = Reference()
    if only is not None:
        {"q1band": lambda R: banded(R), "pcg": lambda R: pcg(R, tree), "csr": lambda R: csr(R),
         "spai2": lambda R: spai2(R, tree), "batch512": lambda R: batch512(R)}[only](R)
        print("golden fixture", only, "written to", HERE)
        return
    td = os.path.join(tree, "honei", "math", "testdata")

    # ---- FEATFLOW2 MG fixture --------------------------------------------------------
    base = os.path.join(td, "poisson_advanced4", "sort_0") + "/"
    out = {}
    A = [R.read_ell(base + f"A_{l}.ell") for l in range(1, 5)]
    prol = [R.read_ell(base + f"prol_{l}.ell") for l in range(2, 5)]
    for l, a in enumerate(A, 1):
        put_matrix(out, f"A_{l}", a)
    for l, p in enumerate(prol, 2):
        put_matrix(out, f"prol_{l}", p)
    for v in ("rhs_4", "init_4", "sol_4"):
        out[v] = R.read_exp(base + v)
    res = [P.ell_from_csr(p.cols, p.rows, *P.transpose_csr(p.rows, p.cols, *p.to_csr())) for p in prol]
    H = P.MGHierarchy(A, prol, res, [0] * 4)
    x, used, _ = R.mg(H, out["rhs_4"], out["init_4"], damping=0.7, eps=1e-8, max_iters=100,
                      max_iters_coarse=1000, n_pre=2, n_post=2)
    out["mg_x"], out["mg_used"] = x, np.array(used)
    x, used, _ = R.cg(A[3], out["rhs_4"], out["init_4"], max_iters=10000, eps=1e-8)
    out["cg_x"], out["cg_used"] = x, np.array(used)
    xs = P.uniform_vector(A[3].rows, 11)
    out["spmv_x"] = xs
    out["spmv_y"], _ = R.spmv(A[3], xs)
    out["defect_r"] = R.defect(A[3], out["rhs_4"], xs)
    np.savez_compressed(os.path.join(HERE, "featflow_pa4.npz"), **out)

    # ---- 5pt defect fixture -----------------------------------------------------------
    out = {}
    A5 = R.read_ell(os.path.join(td, "5pt_10x10.ell"))
    put_matrix(out, "A", A5)
    x = P.uniform_vector(A5.cols, 3)
    b = P.uniform_vector(A5.rows, 4)
    out["x"], out["b"] = x, b
    out["y"], _ = R.spmv(A5, x)
    out["r"] = R.defect(A5, b, x)
    np.savez_compressed(os.path.join(HERE, "defect_5pt.npz"), **out)

    # ---- Q1 Poisson (reference construction) -----------------------------------------
    out = {}
    M = 33
    Aq = R.q1_poisson(M)
    out["q1_Aj"], out["q1_Ax"], out["q1_Arl"] = Aq.Aj, Aq.Ax, Aq.Arl
    out["q1_info"] = np.array(Aq.info() + [Aq.nnz], np.int64)
    x = P.uniform_vector(Aq.rows, 2)
    out["spmv_x"] = x
    out["spmv_y64"], _ = R.spmv(Aq, x)
    A32 = Aq.astype(np.float32)
    out["spmv_y32"], _ = R.spmv(A32, x.astype(np.float32))
    xt = P.uniform_vector(Aq.rows, 1)
    b, _ = R.spmv(Aq, xt)
    out["b"] = b
    x64, u64, _ = R.cg(Aq, b, eps=1e-8)
    out["cg_x64"], out["cg_used64"] = x64, np.array(u64)
    x32, u32, _ = R.cg(A32, b.astype(np.float32), eps=1e-5)
    out["cg_x32"], out["cg_used32"] = x32, np.array(u32)
    H = P.mg_hierarchy(M)
    xm, um, _ = R.mg(H, b, eps=1e-8)
    out["mg_x64"], out["mg_used64"] = xm, np.array(um)
    H32 = H.astype(np.float32)
    xm, um, _ = R.mg(H32, b.astype(np.float32), eps=1e-5)
    out["mg_x32"], out["mg_used32"] = xm, np.array(um)
    xi, ui, _ = R.ir_mg(H, H32, b, eps=1e-10, inner_eps=1e-3)
    out["ir_x"], out["ir_used"] = xi, np.array(ui)
    # permuted variant (seed 7) and variable coefficient (seed 5, log-uniform [1e-2, 1e2])
    Ap, perm = P.q1_poisson_permuted(M, 7)
    bp = np.empty_like(b)
    bp[perm] = b
    out["perm"] = perm
    out["perm_spmv_y"], _ = R.spmv(Ap, x)
    xp, up, _ = R.cg(Ap, bp, eps=1e-8)
    out["perm_cg_x"], out["perm_cg_used"] = xp, np.array(up)
    coef = P.log_uniform_coef(M, 1e-2, 1e2, 5)
    Av = P.q1_poisson(M, coef)
    bv, _ = R.spmv(Av, xt)
    out["var_b"] = bv
    xv, uv, _ = R.cg(Av, bv, eps=1e-8)
    out["var_cg_x"], out["var_cg_used"] = xv, np.array(uv)
    # 257^2, plain FP64 CG (the CG-latency workload); iteration count and checksums only
    A257 = R.q1_poisson(257)
    xt257 = P.uniform_vector(A257.rows, 1)
    b257, _ = R.spmv(A257, xt257)
    x257, u257, _ = R.cg(A257, b257, eps=1e-8)
    out["cg257_used"] = np.array(u257)
    out["cg257_x_sample"] = x257[::97].copy()
    out["cg257_x_sum"] = np.array(x257.sum())
    np.savez_compressed(os.path.join(HERE, "q1_small.npz"), **out)
    banded(R)
    pcg(R, tree)
    csr(R)
    spai2(R, tree)
    print("golden fixtures written to", HERE)


BATCH_SEED = 2024


def batch512(R):
    """CG on every system of the 512-system batch with the reference's tags::CPU and
    tags::CPU::SSE, one host thread per system (the reference's containers are independent)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.bindings import Oracle
    O = Oracle()
    R.set_threads(1)
    sides = np.random.default_rng(BATCH_SEED).integers(17, 258, size=512)

    def one(i):
        M = int(sides[i])
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, BATCH_SEED + i), symmetric=True)
        b, _ = R.spmv(A, P.uniform_vector(M * M, BATCH_SEED + i + 1))
        nb = np.linalg.norm(b)
        row = []
        for tag in ("cpu", "sse"):
            x, u, _ = R.cg(A, b, eps=1e-8, max_iters=100000, tag=tag)
            row += [u, np.linalg.norm(O.defect(A, b, x)) / nb]
        return row

    path = os.path.join(HERE, "batch512.npz")
    out = dict(np.load(path)) if os.path.exists(path) else {}
    if "cpu_used" not in out:
        with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
            r = np.array(list(ex.map(one, range(len(sides)))))
        out.update(sides=sides, cpu_used=r[:, 0].astype(np.int64), cpu_relres=r[:, 1],
                   sse_used=r[:, 2].astype(np.int64), sse_relres=r[:, 3])
    # the MultiCore tag runs its own thread pool: one system at a time, on 4 threads (the
    # honeirc default) and on 16; every dot product is split into that many partial sums
    for threads in (4, 16):
        if f"mc{threads}_used" in out:
            continue
        R.set_threads(threads)
        used, rel = [], []
        for i in range(len(sides)):
            M = int(sides[i])
            A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, BATCH_SEED + i), symmetric=True)
            b, _ = R.spmv(A, P.uniform_vector(M * M, BATCH_SEED + i + 1))
            x, u, _ = R.cg(A, b, eps=1e-8, max_iters=100000, tag="mc-sse")
            used.append(u)
            rel.append(np.linalg.norm(O.defect(A, b, x)) / np.linalg.norm(b))
        out[f"mc{threads}_used"] = np.array(used, np.int64)
        out[f"mc{threads}_relres"] = np.array(rel)
        np.savez_compressed(path, **out)
    np.savez_compressed(path, **out)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only")]
    only = None
    if "--only" in sys.argv:
        only = sys.argv[sys.argv.index("--only") + 1]
        args = [a for a in args if a != only]
    tree = args[0] if args else os.environ.get("HONEI_REF")
    if not tree:
        sys.exit("usage: make_golden.py <HONEI source tree> [--only NAME]  (or set HONEI_REF)")
    main(tree, only)
