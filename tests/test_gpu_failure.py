"""Failure handling on the device without a GPU fault: a bounded wait that runs out reports
HB_ERR_TIMEOUT to the host and leaves the context usable; errors from bad inputs are refused
before any launch."""
import time

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


def test_bounded_wait_times_out_and_the_context_stays_usable(hb, oracle):
    from honei_b200._lib import lib
    ctx = hb.default_context()
    t0 = time.perf_counter()
    st = lib().hb_selftest_wait_timeout(ctx.handle)
    dt = time.perf_counter() - t0
    assert st == 5, st                    # HB_ERR_TIMEOUT: both waits (barrier, counter) gave up
    assert 3.5 < dt < 40.0
    # the same context solves normally afterwards (the barrier words were reset), in the
    # resident and in the streaming CG kernel
    A = P.q1_poisson(65)
    b = oracle.spmv(A, P.uniform_vector(A.rows, 1))
    Ad = hb.SparseMatrixELL.from_reference(A)
    x_o, u_o = oracle.cg(A, b, eps=1e-8, max_iters=5000)
    for resident in (True, False):
        prev = hb.CGSolver.set_resident(resident)
        try:
            x = torch.zeros(A.rows, dtype=torch.float64, device="cuda")
            used = hb.CGSolver.value(Ad, None, torch.from_numpy(b).cuda(), x, 5000, 1e-8)
        finally:
            hb.CGSolver.set_resident(prev)
        assert abs(used - u_o) <= 1


def test_invalid_inputs_are_refused_before_launch(hb):
    from honei_b200._lib import HBError, lib
    ctx = hb.default_context()
    A = hb.SparseMatrixELL.from_reference(P.q1_poisson(9))
    torch.cuda.synchronize()
    launches = ctx.launches()
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Product.value(torch.empty(80, dtype=torch.float64, device="cuda"), A,
                         torch.empty(81, dtype=torch.float64, device="cuda"))
    # a misaligned matrix array is refused by the C ABI itself
    import ctypes as C
    from honei_b200._lib import HbEll
    bad = HbEll(81, 81, A.K, A.ld, A.Aj.data_ptr() + 4, A.Ax.data_ptr(), 0, 0)
    x = torch.zeros(81, dtype=torch.float64, device="cuda")
    assert lib().hb_spmv_f64(ctx.handle, C.byref(bad), x.data_ptr(), x.data_ptr()) == 1
    assert ctx.launches() == launches


def test_ell_validate_counts_bad_columns(hb):
    """The debug check of a hand-built matrix: 0 for imported and assembled matrices; every slot
    whose column is neither the padding mark nor inside [0, cols) is counted (no product runs on
    the corrupted copy)."""
    A = hb.SparseMatrixELL.from_reference(P.q1_poisson(33))
    assert A.validate() == 0
    assert hb.SparseMatrixELL.q1_poisson(65).validate() == 0
    Aj = A.Aj.clone()
    Aj[5] = A.columns()            # one past the end
    Aj[17] = -2                    # below the padding mark
    Aj[100] = 2 ** 31 - 1
    Aj[200] = -1                   # padding: fine
    bad = hb.SparseMatrixELL(A.rows(), A.columns(), A.K, A.ld, Aj, A.Ax)
    assert bad.validate() == 3
