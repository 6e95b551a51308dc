"""Batched persistent solver (hb_batch_*): parity against the oracle, the mixed-precision
target, and the same result alone and in the mix (bit for bit).  The batch systems are the SPD
form of the Q1 matrix (Dirichlet couplings eliminated), as the batched configurations ask."""
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
def test_batch_cg64_parity_with_oracle(B, oracle, rows):
    systems = B.q1_batch(SIDES, coef_range=(1e-1, 1e1), seed=3, mode="cg64", eps=1e-8)
    res = B.BatchSolver(systems).solve(B.HbBatchConfig(4, 256, 0, rows))
    for s, r, M in zip(systems, res, SIDES):
        A = P.q1_poisson(M, P.log_uniform_coef(M, 1e-1, 1e1, s_seed(systems, s)), symmetric=True)
        b = host(s.b)
        x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=100000)
        assert r["status"] == 0
        assert abs(r["iterations"] - u_o) <= 1, (M, r["iterations"], u_o)
        x = host(s.x)
        ro = np.linalg.norm(oracle.defect(A, b, x_o)) / np.linalg.norm(b)
        rg = np.linalg.norm(oracle.defect(A, b, x)) / np.linalg.norm(b)
        # both stop at the 1e-8 target; the final true residuals agree to 1e-10 absolute or 5 %
        # (the cluster's reduction tree differs from the sequential reference sum, and CG
        # amplifies the round-off difference over the iterations); one iteration apart: to one
        # CG contraction step
        tol = max(1e-10, 0.05 * ro) if r["iterations"] == u_o else 0.1 * ro
        assert abs(rg - ro) <= tol, (M, rg, ro, r["iterations"], u_o)
        assert abs(r["true_relres"] - rg) <= 1e-12 + 1e-6 * rg


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
