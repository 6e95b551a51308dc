"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(hb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "hb_spmv_f64" in names and "hb_cg_f64" in names and len(names) > 30


def test_library_exports_every_declared_symbol():
    from honei_b200 import _lib
    lib = _lib.lib()  # loads libhonei_b200.so (no CUDA call is made)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    from honei_b200 import _lib
    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_status_strings():
    from honei_b200 import _lib
    assert _lib.status_string(0) == "ok"
    assert "sizes" in _lib.status_string(2)


def test_entry_points_refuse_invalid_arguments_before_any_device_call():
    """A null context or matrix is HB_ERR_INVALID, returned before any CUDA call (so this runs
    without a GPU)."""
    from honei_b200 import _lib
    lib = _lib.lib()
    invalid = 1
    for name, args in (("hb_spai2_f64", [None] * 3), ("hb_spai2_f32", [None] * 3), ("hb_csr_spmv_f64", [None] * 4),
                       ("hb_csr_defect_f32", [None] * 5), ("hb_spmv_f64", [None] * 4), ("hb_defect_f64", [None] * 5),
                       ("hb_cg_f64", [None] * 4 + [10, 1e-8, None, None])):
        st = getattr(lib, name)(*args)
        assert st == invalid, (name, st)
    e = _lib.HbEll(9, 9, 1, 64, 0, 0, 0, 0)
    assert lib.hb_spai2_f64(None, ctypes.byref(e), ctypes.byref(e)) == invalid
