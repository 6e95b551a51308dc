"""Parity at the workloads' own sizes, against the reference compiled from its sources.

The small-size tests pin every solver against the oracle; these run the same comparisons on
the systems the benchmark quotes its figures on:

- plain FP64 CG on the Q1 Poisson grids of 1025^2 and 2049^2 (x0 = 0, relative residual 1e-8);
- V(2,2) MG on the 2049^2 grid, FP64 and FP32 (coarse CG capped at 100 iterations);
- FP64 iterative refinement around FP32 V-cycles on the 2049^2 grid with a cellwise
  coefficient 10^U(-2,2) (contrast 10^4, Galerkin coarse levels), to 1e-10;
- every system of the 512-system batch (side U{17..257}, coefficient 10^U(-1,1)), FP64 CG and
  FP32-inner refinement.

The reference side is HONEI's own solver templates (honei/math/cg.hh:68-132,
honei/math/mg.hh:1098-1126, honei/math/ir.hh:30-78) on tags::CPU::MultiCore::SSE over all host
cores (tests/test_oracle_pin.py pins that tag's iteration counts to tags::CPU's); the batch
systems go through the plain-C oracle, one host thread per system.

Bar: iterations / cycles / outer steps within +-1 of the reference's, and the
final true relative residual ||b - A x|| / ||b|| within 1e-10 of the reference's.  Where the
counts differ by one, the residuals differ by one step's contraction, which is stated and
checked per case (FP32 solves: the FP32 bar of the test).  The batch's FP64 CG is held to the
reference's own spread between its tags on the same systems (the test says why).
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CORES = os.cpu_count() or 1


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


@pytest.fixture(scope="module")
def ref(reference):
    reference.set_threads(CORES)
    return reference


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def relres(oracle, A, b, x):
    return float(np.linalg.norm(oracle.defect(A, b, np.asarray(x, A.dtype))) / np.linalg.norm(b))


def contraction(hist_len, rel):
    """Mean residual reduction per step of a solve that reached `rel` in `hist_len` steps."""
    return rel ** (1.0 / max(hist_len, 1))


@pytest.mark.parametrize("M", [1025, 2049])
def test_cg_f64_at_size_matches_reference(hb, oracle, ref, M):
    A = P.q1_poisson(M)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    x_r, u_r, _ = ref.cg(A, b, eps=1e-8, max_iters=100000, tag="mc-sse")
    Ad = hb.SparseMatrixELL.from_reference(A)
    x = torch.zeros(A.rows, dtype=torch.float64, device="cuda")
    u_g = hb.CGSolver.value(Ad, None, dev(b), x, 100000, 1e-8)
    x_g = host(x)
    rg, rr = relres(oracle, A, b, x_g), relres(oracle, A, b, x_r)
    print(f"CG {M}^2: GPU {u_g} iterations, relres {rg:.6e}; reference {u_r}, {rr:.6e}")
    assert abs(u_g - u_r) <= 1, (M, u_g, u_r)
    if u_g == u_r:
        assert abs(rg - rr) <= 1e-10, (M, rg, rr)
    else:
        # one CG step apart: the residuals differ by about one step's reduction
        q = contraction(u_r, rr)
        assert abs(rg - rr) <= 2 * (1 - q) * rr + 1e-10, (M, rg, rr, q)
    assert np.linalg.norm(x_g - x_r) <= 1e-5 * np.linalg.norm(x_r)


def test_cg_f64_permuted_2049_matches_reference(hb, oracle, ref):
    """Config 2's CG on the randomly permuted 2049^2 matrix, against the reference's CG on the
    same permuted matrix: the GPU as given (its product on the permuted ELL) and through the
    Cuthill-McKee ordered copy (CGSolver on an OrderedMatrixELL), each within +-1 iteration and
    1e-10 of the reference's final true residual."""
    Ap, _ = P.q1_poisson_permuted(2049, 5)
    b = oracle.spmv(Ap, P.uniform_vector(Ap.rows, 1))
    x_r, u_r, _ = ref.cg(Ap, b, eps=1e-8, max_iters=100000, tag="mc-sse")
    rr = relres(oracle, Ap, b, x_r)
    Ad = hb.SparseMatrixELL.from_reference(Ap)
    for name, A in (("as given", Ad), ("ordered copy", Ad.ordered(columns=True))):
        x = torch.zeros(Ap.rows, dtype=torch.float64, device="cuda")
        u_g = hb.CGSolver.value(A, None, dev(b), x, 100000, 1e-8)
        rg = relres(oracle, Ap, b, host(x))
        print(f"CG permuted 2049^2 {name}: GPU {u_g} iterations, relres {rg:.6e}; reference {u_r}, {rr:.6e}")
        assert abs(u_g - u_r) <= 1, (name, u_g, u_r)
        tol = 1e-10 if u_g == u_r else 2 * (1 - contraction(u_r, rr)) * rr + 1e-10
        assert abs(rg - rr) <= tol, (name, rg, rr)


def test_cg_f32_1025_matches_reference(hb, oracle, ref):
    """Config 2's CG in FP32 at 1025^2 (to 1e-5, where FP32 CG still converges steadily) against
    the reference's FP32 CGSolver: iterations within +-1, the final true residual (in FP64 from
    the FP32 iterates) within 2 % of the reference's."""
    A = P.q1_poisson(1025).astype(np.float32)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1).astype(np.float32))
    x_r, u_r, _ = ref.cg(A, b, eps=1e-5, max_iters=100000, tag="mc-sse")
    Ad = hb.SparseMatrixELL.from_reference(A)
    x = torch.zeros(A.rows, dtype=torch.float32, device="cuda")
    u_g = hb.CGSolver.value(Ad, None, dev(b), x, 100000, 1e-5)
    A64, b64 = A.astype(np.float64), b.astype(np.float64)
    rg = relres(oracle, A64, b64, host(x).astype(np.float64))
    rr = relres(oracle, A64, b64, x_r.astype(np.float64))
    print(f"CG FP32 1025^2: GPU {u_g} iterations, relres {rg:.6e}; reference {u_r}, {rr:.6e}")
    assert abs(u_g - u_r) <= 1, (u_g, u_r)
    assert abs(rg - rr) <= 0.02 * rr, (rg, rr)


@pytest.fixture(scope="module")
def h2049():
    return P.mg_hierarchy(2049)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["f64", "f32"])
def test_mg_2049_matches_reference(hb, oracle, ref, h2049, dt):
    """V(2,2) MG, damped Jacobi 0.7, PROLMAT transfers, 9^2 coarse CG capped at 100 iterations
    (max_iters_coarse of honei/math/mg_TEST.cc:421).  FP64 to 1e-8; FP32 to 1e-6 (FP32 V-cycles
    stagnate near 1e-7)."""
    H = h2049 if dt == np.float64 else h2049.astype(np.float32)
    A64 = h2049.A[-1]
    eps = 1e-8 if dt == np.float64 else 1e-6
    b64 = oracle.spmv(A64, P.uniform_vector(A64.rows, 5))
    b = b64.astype(dt)
    x_r, u_r, _ = ref.mg(H, b, eps=eps, max_iters=100, max_iters_coarse=100, tag="mc-sse")
    data = hb.MGData.from_hierarchy(H, dt, eps=eps, max_iters=100, max_iters_coarse=100)
    x = torch.zeros(A64.rows, dtype=torch.float64 if dt == np.float64 else torch.float32, device="cuda")
    u_g, r0, r1 = hb.MGSolver.value(data, dev(b), x)
    x_g = host(x)
    data.close()
    # residuals of both solutions in FP64 against the FP64 system
    rg = relres(oracle, A64, b64, x_g.astype(np.float64))
    rr = relres(oracle, A64, b64, x_r.astype(np.float64))
    print(f"MG 2049^2 {np.dtype(dt).name}: GPU {u_g} cycles, relres {rg:.6e}; reference {u_r}, {rr:.6e}")
    assert abs(u_g - u_r) <= 1, (u_g, u_r)
    if dt == np.float64:
        tol = 1e-10 if u_g == u_r else 2 * (1 - contraction(u_r, rr)) * rr + 1e-10
    else:
        # FP32: the V-cycle's own rounding (~1e-7 relative) bounds the agreement
        tol = 1e-7 if u_g == u_r else 2 * (1 - contraction(u_r, rr)) * rr + 1e-7
    assert abs(rg - rr) <= tol, (rg, rr, u_g, u_r)


def test_ir_2049_contrast_1e4_matches_reference(hb, oracle, ref):
    """IRSolver (honei/math/ir.hh:30-78, warm-started inner MG as the reference runs it): FP64
    defect / norm / update around FP32 V(2,2) cycles to 1e-3, outer target 1e-10, on the 2049^2
    grid with a cellwise coefficient 10^U(-2,2) and Galerkin coarse levels."""
    M = 2049
    coef = P.log_uniform_coef(M, 1e-2, 1e2, 3)
    H = P.mg_hierarchy(M, coef=coef)
    H32 = H.astype(np.float32)
    A = H.A[-1]
    b = oracle.spmv(A, P.uniform_vector(A.rows, 4))
    x_r, u_r, _ = ref.ir_mg(H, H32, b, eps=1e-10, inner_eps=1e-3, max_iters=100, inner_max_iters=100,
                            max_iters_coarse=100, tag="mc-sse")
    A64 = hb.SparseMatrixELL.from_reference(A)
    mg32 = hb.MGData.from_hierarchy(H, dtype=np.float32, eps=1e-3, max_iters=100, max_iters_coarse=100)
    x = torch.zeros(A.rows, dtype=torch.float64, device="cuda")
    u_g, r0, r1 = hb.IRSolver.value(A64, dev(b), x, mg32, eps=1e-10, max_iters=100, warm_start=True)
    x_g = host(x)
    mg32.close()
    rg, rr = relres(oracle, A, b, x_g), relres(oracle, A, b, x_r)
    print(f"IR 2049^2: GPU {u_g} outer steps, relres {rg:.6e}; reference {u_r}, {rr:.6e}; "
          f"|x_g - x_r| / |x_r| = {np.linalg.norm(x_g - x_r) / np.linalg.norm(x_r):.3e}")
    assert abs(u_g - u_r) <= 1, (u_g, u_r)
    assert rg < 1e-10 and rr < 1e-10, (rg, rr)
    assert abs(rg - rr) <= 1e-10
    # the two solutions agree to the accuracy the 1e-10 residual target gives
    assert np.linalg.norm(x_g - x_r) <= 1e-6 * np.linalg.norm(x_r), np.linalg.norm(x_g - x_r) / np.linalg.norm(x_r)


BATCH_SEED = 2024


def _batch_sides(n=512, seed=BATCH_SEED):
    return np.random.default_rng(seed).integers(17, 258, size=n)


@pytest.mark.parametrize("shape", [(2, 512, 4), (4, 256, 1), (8, 256, 1)], ids=lambda t: "c%d_t%d_r%d" % t)
def test_batch_512_cg64_within_the_references_own_spread(hb, oracle, shape):
    """The 512-system batch of the benchmark, FP64 CG, solved in one launch at the shapes the
    tuner picks (clusters of 4 or 8 CTAs of 256 threads, one row per thread) and at the
    four-row layout, against the reference's CGSolver<tags::CPU> on every system
    (tests/golden/batch512.npz, written by the compiled reference).

    On these systems (contrast 10^2, up to 872 iterations) the iteration count at which the
    1e-8 test fires depends on the summation order of the dot products.  The reference's own
    tags show it: tags::CPU::SSE and tags::CPU::MultiCore::SSE on 4 and on 16 threads differ from
    tags::CPU only in that order, and land on tags::CPU's count for 176 to 239 of the 512
    systems; the more partial sums a tag splits a dot product into, the wider the spread (mean
    |difference| 0.78, 0.99, 1.07 iterations, largest 6, 7, 8; the same fixture).  The GPU sums
    each dot product over 1024 threads of the cluster, further from the sequential order than
    any reference tag.  The bar is the reference's own spread with that allowance: the largest
    |iterations - tags::CPU's| over the batch within 2 of the reference tags' largest, the mean
    within 1.25 times theirs, every final true residual below the target, and its distance from
    tags::CPU's within the largest such distance between the reference's tags."""
    from conftest import load_golden
    from honei_b200 import batch as B
    g = load_golden("batch512")
    sides = _batch_sides()
    assert np.array_equal(sides, g["sides"])
    systems = B.q1_batch(sides, coef_range=(1e-1, 1e1), seed=BATCH_SEED, mode="cg64", eps=1e-8)
    res = B.BatchSolver(systems).solve(B.HbBatchConfig(shape[0], shape[1], 0, shape[2]))
    tags = [t for t in ("sse", "mc4", "mc16") if f"{t}_used" in g]
    d_ref = {t: np.abs(g[f"{t}_used"] - g["cpu_used"]) for t in tags}
    r_ref = {t: np.abs(g[f"{t}_relres"] - g["cpu_relres"]) for t in tags}
    D = max(1, max(int(d.max()) for d in d_ref.values()))
    Dmean = max(float(d.mean()) for d in d_ref.values())
    Rr = max(float(r.max()) for r in r_ref.values())
    u_g = np.array([r["iterations"] for r in res])
    r_g = np.array([r["true_relres"] for r in res])
    st = np.array([r["status"] for r in res])
    du = np.abs(u_g - g["cpu_used"])
    dr = np.abs(r_g - g["cpu_relres"])
    ref_txt = "; ".join(f"{t}: {int(np.sum(d == 0))} equal, max {int(d.max())}, mean {d.mean():.2f}"
                        for t, d in d_ref.items())
    print(f"batch 512 cg64 {shape}: |GPU - tags::CPU| iterations: {int(np.sum(du == 0))} equal, {int(np.sum(du == 1))} "
          f"one apart, max {int(du.max())}, mean {du.mean():.2f}; reference tags: {ref_txt}; residual gap max "
          f"{dr.max():.3e} (reference tags {Rr:.3e})")
    assert np.all(st == 0)
    assert np.all(r_g < 1e-8 * (1 + 1e-6)), r_g.max()
    assert du.max() <= D + 2 and du.mean() <= 1.25 * Dmean, (int(du.max()), D, du.mean(), Dmean)
    assert dr.max() <= Rr, (dr.max(), Rr)
    # spot check: the device-reported true residual is the host's on a few systems
    for i in (0, 17, 255):
        A = systems[i].A64.to_host()
        b, x = host(systems[i].b), host(systems[i].x)
        assert abs(relres(oracle, A, b, x) - r_g[i]) <= 1e-6 * r_g[i]


def test_batch_512_ir32_every_system_matches_oracle(hb, oracle):
    """The same batch in mixed precision (FP64 refinement around FP32 CG to 1e-3 per step, to a
    1e-8 FP64 residual), one row per thread on 4-CTA clusters of 256 threads: every system's
    outer step count against the oracle's scaled refinement around FP32 CG on the same matrix
    and right-hand side."""
    from honei_b200 import batch as B
    sides = _batch_sides()
    systems = B.q1_batch(sides, coef_range=(1e-1, 1e1), seed=BATCH_SEED, mode="ir32", eps=1e-8, inner_eps=1e-3)
    res = B.BatchSolver(systems).solve(B.HbBatchConfig(4, 256, 0, 1))
    mats = [s.A64.to_host() for s in systems]
    bs = [host(s.b) for s in systems]
    xs = [host(s.x) for s in systems]

    def ref_solve(i):
        A, b = mats[i], bs[i]
        _, u_o, _, _ = oracle.ir_cg(A, A.astype(np.float32), b, eps=1e-8, inner_eps=1e-3)
        return u_o, relres(oracle, A, b, xs[i])

    with ThreadPoolExecutor(CORES) as pool:
        out = list(pool.map(ref_solve, range(len(systems))))
    bad = [(i, int(sides[i]), r["outer"], u_o, rg) for i, (r, (u_o, rg)) in enumerate(zip(res, out))
           if r["status"] != 0 or abs(r["outer"] - u_o) > 1 or rg >= 1e-8]
    d = [abs(r["outer"] - o[0]) for r, o in zip(res, out)]
    print(f"batch 512 ir32: {d.count(0)} systems with the oracle's outer step count, {d.count(1)} one apart")
    assert not bad, f"{len(bad)} of {len(systems)} systems outside the bar: {bad[:8]}"
