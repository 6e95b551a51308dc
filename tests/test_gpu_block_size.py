"""hb_set_block_size: the per-context threads-per-block knob that HONEI's honeirc block-size keys
(cuda::product_smell_dv_*, cuda::product_bmdv_q1_*, cuda::scaled_sum_two_* ...) set.  Every
allowed size gives bit-identical results; sizes outside the kernel's range are refused."""
import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def la():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_every_block_size_gives_the_same_bits(la, oracle, dt):
    td = torch.float64 if dt == np.float64 else torch.float32
    A = P.q1_poisson(65).astype(dt)
    Ad = la.SparseMatrixELL.from_reference(A)
    Ab = la.BandedMatrixQ1.from_ell(Ad)
    xh = P.uniform_vector(A.rows, 1).astype(dt)
    x = torch.from_numpy(xh).cuda()
    b = torch.from_numpy(P.uniform_vector(A.rows, 2).astype(dt)).cuda()
    want_y = oracle.spmv(A, xh)
    ref = {}
    try:
        for bs in (0, 32, 64, 96, 128, 160, 256):
            la.set_block_size("ell", bs)
            la.set_block_size("q1band", bs)
            la.set_block_size("vector", bs)
            y, r, q, s = (torch.empty_like(x) for _ in range(4))
            la.Product.value(y, Ad, x)
            la.Defect.value(r, b, Ad, x)
            la.Product.value(q, Ab, x)
            s.copy_(x)
            la.ScaledSum.value(s, b, 0.25)
            assert np.array_equal(y.cpu().numpy(), want_y), bs
            got = {"r": r.cpu().numpy(), "q": q.cpu().numpy(), "s": s.cpu().numpy()}
            if not ref:
                ref = got
            for k in got:
                assert np.array_equal(got[k], ref[k]), (bs, k)
        for bs in (512, 1024):
            la.set_block_size("vector", bs)
            s = x.clone()
            la.ScaledSum.value(s, b, 0.25)
            assert np.array_equal(s.cpu().numpy(), ref["s"]), bs
    finally:
        for f in ("ell", "q1band", "vector"):
            la.set_block_size(f, 0)


def test_block_size_limits(la):
    from honei_b200._lib import lib
    ctx = la.default_context().handle
    for fam, bad in ((0, 512), (1, 1024), (2, 2048), (0, 31), (0, 100), (3, 64), (-1, 64)):
        assert lib().hb_set_block_size(ctx, fam, bad) == -1, (fam, bad)
    assert la.set_block_size("ell", 64) == 0
    assert la.set_block_size("ell", 0) == 64
    with pytest.raises(ValueError):
        la.set_block_size("vector", 33)
