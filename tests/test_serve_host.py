"""Host-side logic of the serving loop: the trace generator and, without a GPU, that requests
whose workers cannot start complete with an error instead of hanging the drain."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_poisson_trace_is_seeded_and_shaped():
    from honei_b200 import serve
    a = serve.poisson_trace(400, rate=200.0, seed=4)
    b = serve.poisson_trace(400, rate=200.0, seed=4)
    assert [r.M for r in a.requests] == [r.M for r in b.requests]
    assert all(np.array_equal(x.coef, y.coef) for x, y in zip(a.requests, b.requests))
    sides = np.array([r.M for r in a.requests])
    assert sides.min() >= 33 and sides.max() <= 1025
    # log-uniform: the median side is near the geometric mean of the range
    assert 0.7 < np.median(sides) / np.sqrt(33 * 1025) < 1.4
    arr = np.array([r.arrival for r in a.requests])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert 0.8 < (len(arr) - 1) / arr[-1] / 200.0 < 1.25
    c = a.requests[3].coef
    assert c.size == (a.requests[3].M - 1) ** 2 and 1e-2 <= c.min() and c.max() <= 1e2


@pytest.mark.skipif(torch.cuda.is_available(), reason="exercises the no-device failure path")
def test_requests_fail_cleanly_without_a_device():
    from honei_b200 import serve
    from honei_b200._lib import HBError
    trace = serve.poisson_trace(6, rate=0.0, side_range=(17, 300), seed=1)
    with serve.Server(mode="mixed", budget_bytes=1 << 30, small_max_side=64, pinned=False) as srv:
        rep = serve.replay(srv, trace, realtime=False)
        assert rep["completed"] == 6 and rep["ok"] == 0
        assert all(c.status != 0 for c in rep["records"])
        st = srv.stats()
        assert st["submitted"] == st["completed"] == 6 and st["bytes_in_use"] == 0
        with pytest.raises(HBError):
            srv.submit(serve.Request(M=4000, x_true=np.zeros(16)))
    with serve.Server(mode="plain", pinned=False) as srv:
        rep = serve.replay(srv, trace, realtime=False)
        assert {c.path for c in rep["records"]} == {"cg64"}
