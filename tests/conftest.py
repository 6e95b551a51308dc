"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs the oracle pins, host logic and ABI checks on any machine; `-m gpu` runs
the parity tests that call libhonei_b200.so on a B200.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libhonei_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.bindings import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference's own CPU path, where it was built (not on machines without it)."""
    from oracle.bindings import REF_SO, Reference
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libhonei_ref.so not built here")
    return Reference()


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def golden_csr(d, key, dtype=np.float64):
    """problems.CsrMatrix stored in a golden npz under key_{Ar,Aj,Ax,info}."""
    from honei_b200 import problems as P
    rows, cols, bs, used = (int(v) for v in d[key + "_info"])
    return P.CsrMatrix(rows, cols, bs, d[key + "_Ar"], d[key + "_Aj"], d[key + "_Ax"].astype(dtype), used)


def golden_matrix(d, name, dtype=np.float64):
    """EllMatrix (reference layout, T = 1) from a CSR stored in a golden npz."""
    from honei_b200 import problems as P
    rows, cols = (int(v) for v in d[f"{name}_shape"])
    return P.ell_from_csr(rows, cols, d[f"{name}_indptr"], d[f"{name}_indices"], d[f"{name}_data"], 1, dtype)


@pytest.fixture(scope="session")
def featflow():
    """The MGSolverTest fixture (poisson_advanced4, levels 1..4) as a hierarchy + vectors."""
    from honei_b200 import problems as P
    d = load_golden("featflow_pa4")
    A = [golden_matrix(d, f"A_{l}") for l in range(1, 5)]
    prol = [golden_matrix(d, f"prol_{l}") for l in range(2, 5)]
    res = [P.ell_from_csr(p.cols, p.rows, *P.transpose_csr(p.rows, p.cols, *p.to_csr())) for p in prol]
    return P.MGHierarchy(A, prol, res, [0] * 4), d


def q1band_test_data(size, dtype):
    """The vectors of the reference's banded product test (honei/la/product_TEST.cc:196-219):
    bands (dv3, dv2, dv4, dv2, dv3, dv4, dv4, dv3, dv2) and x = dv1, v[i] = (i + k) % 311."""
    i = np.arange(size)
    dv1, dv2, dv3, dv4 = [((i + k) % 311).astype(dtype) for k in (2, 1, 25, 7)]
    return [dv3, dv2, dv4, dv2, dv3, dv4, dv4, dv3, dv2], dv1


def q1band_used_mask(n):
    """(9, n) mask of the band entries the banded product reads (column inside [0, n))."""
    root = int(np.sqrt(n))
    offs = [-root - 1, -root, -root + 1, -1, 0, 1, root - 1, root, root + 1]
    r = np.arange(n)
    return np.stack([(r + o >= 0) & (r + o < n) for o in offs])
