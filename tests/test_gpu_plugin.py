"""HONEI's own operators and solver templates on tags::GPU::CUDA through the B200 plugin
(honei_b200/plugin): the C++ programs in tests/plugin link HONEI's CPU library and the plugin,
and compare every GPU-tag result with tags::CPU on the same inputs.  The MG case loads its
hierarchy with HONEI's MGUtil::load_data from files written in HONEI's formats."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from honei_b200 import problems as P

pytestmark = pytest.mark.gpu
BUILD = os.path.join(ROOT, "tests", "plugin", "_build")


def _run(name, *args):
    exe = os.path.join(BUILD, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -C tests/plugin needs the HONEI headers)")
    p = subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)
    print(p.stdout)
    print(p.stderr[-2000:])
    fails = [l for l in p.stdout.splitlines() if l.startswith("FAIL")]
    assert p.returncode == 0 and not fails, fails or p.stderr[-2000:]
    return p.stdout


def test_plugin_operators_and_generic_solvers(tmp_path):
    L = _write_hierarchy(tmp_path, 65)
    out = _run("plugin_ops_test", str(tmp_path), str(L))
    assert "PASS MGSolver<GPU::CUDA>" in out
    assert "FAIL" not in out
    assert out.count("PASS") >= 54
    assert out.count("BandedMatrixQx") == 14
    assert out.count("SparseMatrixCSR") == 14
    assert out.count("PASS SPAI2<GPU::CUDA>") == 4


def test_plugin_cg_specialisation():
    out = _run("plugin_cg_test")
    assert out.count("PASS") == 8 and "FAIL" not in out
    assert out.count("PASS CGSolver<GPU::CUDA, VAR>") == 4


def _write_hierarchy(tmp_path, M, seed=4):
    H = P.mg_hierarchy(M)
    L = len(H.A)
    for l, A in enumerate(H.A, 1):
        P.write_ell(str(tmp_path / f"A_{l}.ell"), A)
    for l, Pm in enumerate(H.prol, 2):
        P.write_ell(str(tmp_path / f"prol_{l}.ell"), Pm)
    A = H.A[-1]
    xt = P.uniform_vector(A.rows, seed)
    ip, ix, dv = A.to_csr()
    P.write_exp(str(tmp_path / f"rhs_{L}"), np.add.reduceat(dv * xt[ix], ip[:-1]))
    P.write_exp(str(tmp_path / f"init_{L}"), np.zeros(A.rows))
    return L


def test_plugin_mg_fast_path(tmp_path):
    """HONEI's MGSolver / MGCycleCreation / RISmoother / IRSolver on tags::GPU::CUDA with the
    plugin's specialisations (honei_b200/plugin/mg_b200.hh), on a hierarchy loaded by
    MGUtil::load_data: smoother sweeps and one coarse-free cycle bit-exact to tags::CPU, the
    solve within +-1 cycle and 1e-10 of tags::CPU's residual, IRSolver within +-1 outer step."""
    import re
    L = _write_hierarchy(tmp_path, 257)
    out = _run("plugin_mg_test", str(tmp_path), str(L))
    assert out.count("PASS") == 5 and "FAIL" not in out
    # the same solve through HONEI's generic templates on the GPU tag (one operator call per
    # step of the cycle, tests/plugin/plugin_ops_test.cc): same cycles, slower
    gen = _run("plugin_ops_test", str(tmp_path), str(L))
    fast_ms = float(re.search(r"fast path vs tags::CPU.*ms cpu \S+ gpu (\S+)", out).group(1))
    gen_ms = float(re.search(r"MGSolver<GPU::CUDA> \(MGUtil.*ms cpu \S+ gpu (\S+)", gen).group(1))
    print(f"MGSolver<GPU::CUDA> 257^2: fast path {fast_ms:.1f} ms, generic operator path {gen_ms:.1f} ms")
    assert fast_ms < gen_ms
