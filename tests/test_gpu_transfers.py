"""Matrix-free geometric transfers on the device (hb_prolongate_*, hb_restrict_*) bit for bit
against the oracle's literal restatement of Prolongation / Restriction<methods::NONE> (pinned to
the reference in test_oracle_pin)."""
import numpy as np
import pytest

from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MASKS = [[2] * 8, [0] * 8, [2, 0, 2, 0, 2, 2, 0, 0], [0, 2, 0, 2, 0, 0, 2, 2], [2, 2, 2, 2, 0, 0, 0, 0]]


@pytest.fixture(scope="module")
def hb():
    from honei_b200 import la
    assert torch.cuda.is_available()
    return la


@pytest.mark.parametrize("side", [1, 3, 5, 9, 17, 33, 129, 1025])
@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_transfers_match_oracle(hb, oracle, side, dt):
    tdt = torch.float64 if dt == np.float64 else torch.float32
    rng = np.random.default_rng(side)
    nf, nc = side * side, ((side - 1) // 2 + 1) ** 2
    for mask in (MASKS if side <= 129 else MASKS[:1]):
        c = rng.uniform(-1, 1, nc).astype(dt)
        f = rng.uniform(-1, 1, nf).astype(dt)
        fine = torch.empty(nf, dtype=tdt, device="cuda")
        hb.Prolongation.value(fine, torch.from_numpy(c).cuda(), mask)
        assert np.array_equal(fine.cpu().numpy(), oracle.prolongate(c, mask, nf)), (side, mask)
        coarse = torch.empty(nc, dtype=tdt, device="cuda")
        hb.Restriction.value(coarse, torch.from_numpy(f).cuda(), mask)
        assert np.array_equal(coarse.cpu().numpy(), oracle.restrict(f, mask)), (side, mask)


def test_transfer_errors(hb):
    from honei_b200._lib import HBError
    with pytest.raises(hb.VectorSizeDoesNotMatch):
        hb.Prolongation.value(torch.empty(81, dtype=torch.float64, device="cuda"),
                              torch.empty(24, dtype=torch.float64, device="cuda"), [2] * 8)
    with pytest.raises(HBError) as e:
        hb.Restriction.value(torch.empty(16, dtype=torch.float64, device="cuda"),
                             torch.empty(64, dtype=torch.float64, device="cuda"), [2] * 8)   # even side
    assert e.value.status == 6
