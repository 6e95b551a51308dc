"""Batched persistent solver (hb_batch_*): parity against the oracle, the mixed-precision
target, and the same result alone and in the mix (bit for bit).  The batch systems are the SPD
form of the Q1 matrix (Dirichlet couplings eliminated), as the batched configurations ask."""
import os

import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def B():
    from honei_b200 import batch
    assert torch.cuda.is_available()
    return batch


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


SIDES = [5, 9, 17, 33, 65, 129, 3, 21, 47]


@pytest.mark.parametrize("rows", [4, 1])
def test_batch_cg64_parity_with_oracle(B, oracle, reference, rows):
    """Each system of a mixed-size batch against the oracle's CG (tags::CPU's order).  These
    systems' iteration counts depend on the dot products' summation order: the reference's own
    tags::CPU::SSE and tags::CPU::MultiCore::SSE (4 and 16 threads) are run on the same systems,
    and the GPU may differ from tags::CPU by their largest difference plus 2 (the GPU's dot
    products have more partial sums than any of them; tests/test_gpu_config_sizes.py measures
    the trend on 512 systems).  Its final true residual must meet the same stopping test and lie
    within the reference tags' largest residual difference or 5 % of tags::CPU's residual: at
    the same iteration count the residual at the stop is the last CG step's rounding amplified
    by the system's conditioning, and the GPU's wider summation trees move it by up to 2-3 %
    (21^2: 9.59e-9 against 9.81e-9, both after 92 iterations)."""
    systems = B.q1_batch(SIDES, coef_range=(1e-1, 1e1), seed=3, mode="cg64", eps=1e-8)
    res = B.BatchSolver(systems).solve(B.HbBatchConfig(4, 256, 0, rows))
    rows_out = []
    for s, r, M in zip(systems, res, SIDES):
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, s_seed(systems, s)), symmetric=True)
        b = host(s.b)
        x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=100000)
        nb = np.linalg.norm(b)
        ro = np.linalg.norm(oracle.defect(A, b, x_o)) / nb
        spread_u, spread_r = 1, 1e-10
        for tag, threads in (("sse", 1), ("mc-sse", 4), ("mc-sse", 16)):
            reference.set_threads(threads)
            x_t, u_t, _ = reference.cg(A, b, eps=1e-8, max_iters=100000, tag=tag)
            spread_u = max(spread_u, abs(u_t - u_o))
            spread_r = max(spread_r, abs(np.linalg.norm(oracle.defect(A, b, x_t)) / nb - ro))
        reference.set_threads(os.cpu_count() or 1)
        x = host(s.x)
        rg = np.linalg.norm(oracle.defect(A, b, x)) / nb
        rows_out.append((M, r["iterations"], u_o, spread_u, rg, ro, spread_r))
        assert r["status"] == 0
        assert abs(r["iterations"] - u_o) <= spread_u + 2, rows_out[-1]
        assert rg < 1.01e-8 and abs(rg - ro) <= max(spread_r, 0.05 * ro), rows_out[-1]
        assert abs(r["true_relres"] - rg) <= 1e-12 + 1e-6 * rg
    print(rows_out)


def s_seed(systems, s):
    return 3 + systems.index(s)


def test_batch_ir32_reaches_fp64_target(B, oracle):
    systems = B.q1_batch(SIDES, coef_range=(1e-2, 1e2), seed=11, mode="ir32", eps=1e-8, inner_eps=1e-3)
    res = B.BatchSolver(systems).solve(B.HbBatchConfig(2, 512))
    for s, r, M in zip(systems, res, SIDES):
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-2, 1e2, 11 + systems.index(s)), symmetric=True)
        b = host(s.b)
        rel = np.linalg.norm(oracle.defect(A, b, host(s.x))) / np.linalg.norm(b)
        assert r["status"] == 0 and r["outer"] >= 1
        assert rel < 1e-8, (M, rel, r)
        assert abs(r["true_relres"] - rel) <= 1e-12 + 1e-6 * rel
        # the oracle's scaled IR with an FP32 CG inner solve takes the same number of outer steps
        x_o, u_o, inner_o, _ = oracle.ir_cg(A, A.astype(np.float32), b, eps=1e-8, inner_eps=1e-3)
        assert abs(r["outer"] - u_o) <= 1, (M, r["outer"], u_o)


@pytest.mark.parametrize("cluster,threads,rows", [(1, 256, 4), (2, 512, 4), (4, 256, 4), (8, 512, 4), (16, 256, 4),
                                                  (1, 512, 1), (2, 256, 1), (8, 256, 1)])
def test_batch_alone_equals_in_the_mix(B, cluster, threads, rows):
    cfg = B.HbBatchConfig(cluster, threads, 0, rows)
    mix = B.q1_batch(SIDES, coef_range=(1e-1, 1e1), seed=5, mode="ir32")
    mix[1].mode = B.HB_BATCH_CG64
    res_mix = B.BatchSolver(mix).solve(cfg)
    for i, M in enumerate(SIDES):
        alone = B.q1_batch([M], coef_range=(1e-1, 1e1), seed=5 + i, mode="ir32")
        if i == 1:
            alone[0].mode = B.HB_BATCH_CG64
        res_alone = B.BatchSolver(alone).solve(cfg)
        assert res_alone[0] == res_mix[i]
        assert torch.equal(alone[0].x, mix[i].x)


def test_batch_tuner_and_every_shape_solves(B, tmp_path, monkeypatch):
    monkeypatch.setenv("HONEI_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    systems = B.q1_batch([17, 33, 65, 9, 129, 33, 17, 65], coef_range=(1e-1, 1e1), seed=1, mode="ir32")
    solver = B.BatchSolver(systems)
    cfg = solver.tune()
    assert cfg.cluster in B.CLUSTERS and cfg.threads in B.THREADS and cfg.rows_per_thread in B.ROWS_PER_THREAD
    assert len(solver.tune_times) == 20
    assert (tmp_path / "tune.json").exists()
    assert all(v > 0 for v in solver.tune_times.values())
    res = solver.solve(cfg)
    assert all(r["true_relres"] < 1e-8 for r in res)
    cfg2 = B.BatchSolver(systems).tune()            # cache hit
    assert (cfg2.cluster, cfg2.threads, cfg2.rows_per_thread) == (cfg.cluster, cfg.threads, cfg.rows_per_thread)


def test_batch_empty_and_single_row(B):
    assert B.BatchSolver([]).solve() == []
    s = B.q1_batch([1], coef_range=None, seed=0, mode="cg64")
    r = B.BatchSolver(s).solve()
    assert r[0]["status"] == 0 and host(s[0].x)[0] == host(s[0].b)[0]
