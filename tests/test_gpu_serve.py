"""The serving loop (hb_server_*): every request of a mixed-size stream reaches the FP64 target,
a request's solution is the same served alone as served in the mix (bitwise), the plain-FP64-CG
baseline does what CGSolver does, and admission keeps the resident bytes within the budget."""
import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def S():
    from honei_b200 import serve
    assert torch.cuda.is_available()
    return serve


def host_relres(oracle, req, x):
    A = P.q1_poisson(req.M, req.coef.reshape(req.M - 1, req.M - 1), symmetric=True)
    b = oracle.spmv(A, req.x_true)
    return np.linalg.norm(oracle.defect(A, b, x)) / np.linalg.norm(b)


@pytest.mark.parametrize("mid", [0, 200])
def test_mixed_stream_reaches_target(S, oracle, mid):
    trace = S.poisson_trace(24, rate=400.0, side_range=(17, 300), seed=5)
    with S.Server(mode="mixed", small_max_side=96, large_workers=2, mid_max_side=mid) as srv:
        rep = S.replay(srv, trace)
    assert rep["completed"] == rep["ok"] == 24
    assert set(rep["paths"]) == ({"batch", "mgpcg"} if mid == 0 else {"batch", "mgbatch", "mgpcg"})
    by_tag = {c.tag: c for c in rep["records"]}
    for req in trace.requests:
        c = by_tag[req.tag]
        rel = host_relres(oracle, req, c.x)
        assert c.true_relres < 1e-8 and rel < 1e-8, (req.M, c)
        assert abs(rel - c.true_relres) <= 1e-6 * rel + 1e-14
        assert np.linalg.norm(c.x - req.x_true) <= 1e-4 * np.linalg.norm(req.x_true)


@pytest.mark.parametrize("mid", [0, 150])
def test_alone_equals_in_the_mix(S, mid):
    trace = S.poisson_trace(16, rate=0.0, side_range=(17, 200), seed=9)
    with S.Server(mode="mixed", small_max_side=64, large_workers=3, mid_max_side=mid) as srv:
        mix = {c.tag: c for c in S.replay(srv, trace, realtime=False)["records"]}
    with S.Server(mode="mixed", small_max_side=64, large_workers=3, mid_max_side=mid) as srv:
        for req in trace.requests:
            srv.submit(req)
            (c,) = srv.drain()
            m = mix[req.tag]
            assert c.status == m.status == 0 and c.path == m.path
            assert (c.iterations, c.outer) == (m.iterations, m.outer)
            assert np.array_equal(c.x, m.x), (req.M, c.path)


def test_plain_cg64_matches_cgsolver(S):
    from honei_b200 import la
    trace = S.poisson_trace(4, rate=0.0, side_range=(33, 129), seed=2)
    with S.Server(mode="plain") as srv:
        rec = {c.tag: c for c in S.replay(srv, trace, realtime=False)["records"]}
    for req in trace.requests:
        c = rec[req.tag]
        assert c.path == "cg64" and c.status == 0 and c.true_relres < 1e-8
        A = la.SparseMatrixELL.q1_poisson(req.M, torch.from_numpy(req.coef).cuda(), symmetric=True)
        xt = torch.from_numpy(req.x_true).cuda()
        b = torch.empty_like(xt)
        la.Product.value(b, A, xt)
        x = torch.zeros_like(b)
        used = la.CGSolver.value(A, None, b, x, 1000000, 1e-8)
        assert used == c.iterations
        assert np.array_equal(x.cpu().numpy(), c.x)


def test_admission_budget(S):
    trace = S.poisson_trace(10, rate=0.0, side_range=(150, 260), seed=3)
    biggest = max((1 << 20) + 512 * r.M * r.M for r in trace.requests)   # the MG-PCG path's charge
    budget = biggest + biggest // 2          # at most one large request resident at a time
    with S.Server(mode="mixed", budget_bytes=budget, small_max_side=0, large_workers=4, mid_max_side=0) as srv:
        rep = S.replay(srv, trace, realtime=False)
        st = srv.stats()
        with pytest.raises(Exception):
            srv.submit(S.Request(M=2 * int(np.sqrt(budget / 512)) + 1, x_true=np.zeros(4)))
    assert rep["ok"] == 10 and st["bytes_in_use"] == 0 and st["bytes_peak"] <= budget
    # admission kept FIFO order
    recs = sorted(rep["records"], key=lambda c: c.tag)
    assert all(a.t_admit <= b.t_admit for a, b in zip(recs, recs[1:]))


def test_empty_and_single_node_requests(S):
    with S.Server(mode="mixed", small_max_side=64) as srv:
        for tag, M in enumerate((1, 2, 3)):
            srv.submit(S.Request(M=M, x_true=np.ones(M * M), tag=tag))
        out = {c.tag: c for c in srv.drain()}
    for tag, M in enumerate((1, 2, 3)):
        assert out[tag].status == 0, out[tag]
        assert np.allclose(out[tag].x, 1.0, rtol=1e-8)


def test_plain_batched_baseline_solves_every_request(S):
    """The plain FP64 CG baseline with the mixed server's concurrency: grids up to mid_max_side in
    batched cluster launches, larger ones on concurrent whole-GPU CG workers; every request
    reaches the target, and a batched request's solution equals the same system solved in a
    batch of its own."""
    trace = S.poisson_trace(20, rate=0.0, side_range=(17, 400), seed=6)
    with S.Server(mode="plain_batched", mid_max_side=200, large_workers=2) as srv:
        rep = S.replay(srv, trace, realtime=False)
    assert rep["completed"] == rep["ok"] == 20
    assert set(rep["paths"]) == {"batch_cg64", "cg64"}
    assert rep["max_true_relres"] < 1e-8
    by_tag = {c.tag: c for c in rep["records"]}
    with S.Server(mode="plain_batched", mid_max_side=200, large_workers=2) as srv:
        for req in trace.requests[:6]:
            srv.submit(req)
            (c,) = srv.drain()
            m = by_tag[req.tag]
            assert c.path == m.path and c.iterations == m.iterations
            assert np.array_equal(c.x, m.x), (req.M, c.path)


def test_stream_replay_closed_and_open_loop(S):
    """The on-demand stream: a prefix of a long stream is the short stream, and both replays
    (closed loop with a window, open loop at arrival times) serve every request once."""
    long = S.stream_trace(200, rate=300.0, side_range=(17, 200), seed=4)
    short = S.poisson_trace(30, rate=300.0, side_range=(17, 200), seed=4)
    for i, r in enumerate(short.requests):
        q = long.request(i)
        assert q.M == r.M and np.array_equal(q.coef, r.coef) and np.array_equal(q.x_true, r.x_true)
    with S.Server(mode="mixed", small_max_side=64, large_workers=2, mid_max_side=128) as srv:
        rep = S.replay_stream(srv, long.prefix(60), realtime=False, window=8, producers=2)
        assert rep["completed"] == rep["ok"] == 60 and rep["max_true_relres"] < 1e-8
        rep = S.replay_stream(srv, long.prefix(40), realtime=True, producers=2)
        assert rep["completed"] == rep["ok"] == 40
        assert sorted(c.tag for c in rep["records"]) == list(range(40))


def test_admission_charge_covers_the_pool(S):
    """What the stream-ordered pool really held never exceeds what admission charged: the
    high-water mark of the pool's used bytes stays under the peak of the admitted charges."""
    trace = S.poisson_trace(40, rate=0.0, side_range=(17, 700), seed=8)
    for mode in ("mixed", "plain_batched", "plain"):
        with S.Server(mode=mode, mid_max_side=200) as srv:
            rep = S.replay(srv, trace, realtime=False)
            st = srv.stats()
        assert rep["ok"] == 40
        assert "pool_used_high" in st, st
        assert 0 < st["pool_used_high"] <= st["bytes_peak"], (mode, st["pool_used_high"], st["bytes_peak"])
