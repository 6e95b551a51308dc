"""ctypes binding of libhonei_b200.so (the C ABI in include/honei_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback anywhere in this
package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhonei_b200.so")

_lib = None


class HBError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {status_string(status)} (status {status})"
        if detail:
            msg += f" [{detail}]"
        super().__init__(msg)


class HbEll(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("K", C.c_int64), ("ld", C.c_int64),
                ("Aj", C.c_void_p), ("Ax", C.c_void_p), ("dtype", C.c_int32), ("pad_", C.c_int32)]


class HbQ1Band(C.Structure):
    _fields_ = [("n", C.c_int64), ("root", C.c_int64), ("band", C.c_void_p * 9), ("dtype", C.c_int32),
                ("pad_", C.c_int32)]


class HbCsr(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("blocksize", C.c_int64), ("nblocks", C.c_int64),
                ("Ar", C.c_void_p), ("Aj", C.c_void_p), ("Ax", C.c_void_p), ("dtype", C.c_int32),
                ("pad_", C.c_int32)]


class HbMGParams(C.Structure):
    _fields_ = [("max_iters", C.c_int64), ("max_iters_coarse", C.c_int64), ("n_pre", C.c_int64),
                ("n_post", C.c_int64), ("damping", C.c_double), ("eps", C.c_double)]


i64, vp, f64, f32, i32 = C.c_int64, C.c_void_p, C.c_double, C.c_float, C.c_int
P_i64 = C.POINTER(C.c_int64)
P_ell = C.POINTER(HbEll)
P_band = C.POINTER(HbQ1Band)
P_csr = C.POINTER(HbCsr)

# name -> (restype, argtypes)
SIGNATURES = {
    "hb_create": (i32, [C.POINTER(vp), i32]),
    "hb_destroy": (i32, [vp]),
    "hb_set_stream": (i32, [vp, vp]),
    "hb_synchronize": (i32, [vp]),
    "hb_status_string": (C.c_char_p, [i32]),
    "hb_last_error": (C.c_char_p, [vp]),
    "hb_launch_count": (C.c_uint64, [vp]),
    "hb_reserve": (i32, [vp, i64]),
    "hb_cg_set_resident": (i32, [vp, i32]),
    "hb_cg_set_layout": (i32, [vp, i32]),
    "hb_set_block_size": (i32, [vp, i32, i32]),
    "hb_ell_validate": (i32, [vp, P_ell, P_i64]),
    "hb_ell_layout": (i32, [i64, i64, i64, P_i64, P_i64]),
    "hb_ell_import_f64": (i32, [vp, i64, i64, i64, i64, i64, vp, vp, vp, P_ell]),
    "hb_ell_import_f32": (i32, [vp, i64, i64, i64, i64, i64, vp, vp, vp, P_ell]),
    "hb_ell_cast_f64_f32": (i32, [vp, P_ell, P_ell]),
    "hb_ell_cm_order": (i32, [vp, P_ell, vp, vp, P_i64]),
    "hb_ell_bandwidth": (i32, [vp, P_ell, vp, P_i64]),
    "hb_ell_permute": (i32, [vp, P_ell, vp, vp, P_ell]),
    "hb_ell_permute_sorted": (i32, [vp, P_ell, vp, vp, P_ell, vp]),
    "hb_spmv_ranked_f64": (i32, [vp, P_ell, vp, vp, vp, vp]),
    "hb_spmv_ranked_f32": (i32, [vp, P_ell, vp, vp, vp, vp]),
    "hb_spmv_rows_f64": (i32, [vp, P_ell, vp, vp, vp]),
    "hb_spmv_rows_f32": (i32, [vp, P_ell, vp, vp, vp]),
    "hb_ell_pack_offsets": (i32, [vp, P_ell, vp]),
    "hb_spmv_packed_f64": (i32, [vp, P_ell, vp, vp, vp, vp]),
    "hb_spmv_packed_f32": (i32, [vp, P_ell, vp, vp, vp, vp]),
    "hb_gather_f64": (i32, [vp, i64, vp, vp, vp]),
    "hb_gather_f32": (i32, [vp, i64, vp, vp, vp]),
    "hb_spai2_f64": (i32, [vp, P_ell, P_ell]),
    "hb_spai2_f32": (i32, [vp, P_ell, P_ell]),
    "hb_q1_assemble_f64": (i32, [vp, i64, vp, i32, P_ell]),
    "hb_spmv_f64": (i32, [vp, P_ell, vp, vp]),
    "hb_spmv_f32": (i32, [vp, P_ell, vp, vp]),
    "hb_defect_f64": (i32, [vp, P_ell, vp, vp, vp]),
    "hb_defect_f32": (i32, [vp, P_ell, vp, vp, vp]),
    "hb_jacobi_sweeps_f64": (i32, [vp, P_ell, vp, vp, vp, vp, i64]),
    "hb_jacobi_sweeps_f32": (i32, [vp, P_ell, vp, vp, vp, vp, i64]),
    "hb_dot_f64": (i32, [vp, i64, vp, vp, C.POINTER(f64)]),
    "hb_dot_f32": (i32, [vp, i64, vp, vp, C.POINTER(f32)]),
    "hb_norm_l2_f64": (i32, [vp, i64, vp, i32, C.POINTER(f64)]),
    "hb_norm_l2_f32": (i32, [vp, i64, vp, i32, C.POINTER(f32)]),
    "hb_scaled_sum_f64": (i32, [vp, i64, vp, vp, f64]),
    "hb_scaled_sum_f32": (i32, [vp, i64, vp, vp, f32]),
    "hb_scaled_sum3_f64": (i32, [vp, i64, vp, vp, vp, f64]),
    "hb_scaled_sum3_f32": (i32, [vp, i64, vp, vp, vp, f32]),
    "hb_scale_f64": (i32, [vp, i64, vp, f64]),
    "hb_scale_f32": (i32, [vp, i64, vp, f32]),
    "hb_sum_f64": (i32, [vp, i64, vp, vp]),
    "hb_sum_f32": (i32, [vp, i64, vp, vp]),
    "hb_difference_f64": (i32, [vp, i64, vp, vp, vp]),
    "hb_difference_f32": (i32, [vp, i64, vp, vp, vp]),
    "hb_element_product_f64": (i32, [vp, i64, vp, vp, vp]),
    "hb_element_product_f32": (i32, [vp, i64, vp, vp, vp]),
    "hb_copy": (i32, [vp, vp, vp, i64]),
    "hb_fill_f64": (i32, [vp, i64, vp, f64]),
    "hb_fill_f32": (i32, [vp, i64, vp, f32]),
    "hb_convert_f64_f32": (i32, [vp, i64, vp, vp]),
    "hb_convert_f32_f64": (i32, [vp, i64, vp, vp]),
    "hb_cg_f64": (i32, [vp, P_ell, vp, vp, i64, f64, P_i64, C.POINTER(f64)]),
    "hb_cg_f32": (i32, [vp, P_ell, vp, vp, i64, f32, P_i64, C.POINTER(f32)]),
    "hb_selftest_wait_timeout": (i32, [vp]),
    "hb_cg_var_diag_f64": (i32, [vp, P_ell, vp, vp, vp, i64, f64, P_i64, C.POINTER(f64)]),
    "hb_cg_var_diag_f32": (i32, [vp, P_ell, vp, vp, vp, i64, f32, P_i64, C.POINTER(f32)]),
    "hb_cg_var_ell_f64": (i32, [vp, P_ell, P_ell, vp, vp, i64, f64, P_i64, C.POINTER(f64)]),
    "hb_cg_var_ell_f32": (i32, [vp, P_ell, P_ell, vp, vp, i64, f32, P_i64, C.POINTER(f32)]),
    "hb_cg_f64_noalloc": (i32, [P_ell, vp, vp, i64, f64, P_i64, C.POINTER(f64), vp]),
    "hb_mg_create": (i32, [vp, i32, P_ell, P_ell, P_ell, C.POINTER(HbMGParams), C.POINTER(vp)]),
    "hb_mg_create_banded": (i32, [vp, i32, P_ell, P_band, C.POINTER(HbMGParams), C.POINTER(vp)]),
    "hb_mg_destroy": (i32, [vp]),
    "hb_mg_set_params": (i32, [vp, C.POINTER(HbMGParams)]),
    "hb_mg_solve_f64": (i32, [vp, vp, vp, P_i64, C.POINTER(f64)]),
    "hb_mg_solve_f32": (i32, [vp, vp, vp, P_i64, C.POINTER(f32)]),
    "hb_mg_cycle_f64": (i32, [vp, vp, vp]),
    "hb_mg_cycle_f32": (i32, [vp, vp, vp]),
    "hb_mg_set_smoother": (i32, [vp, i32, vp]),
    "hb_ir_mg_solve": (i32, [vp, P_ell, vp, vp, vp, f64, i64, i32, P_i64, C.POINTER(f64)]),
    "hb_ir_cg_solve": (i32, [vp, P_ell, P_ell, vp, vp, f64, f32, i64, i64, P_i64, P_i64, C.POINTER(f64)]),
    # batched solves (struct pointers passed as void*; honei_b200.batch declares the structs)
    "hb_batch_workspace_bytes": (i32, [vp, i64, C.POINTER(C.c_size_t)]),
    "hb_batch_solve": (i32, [vp, vp, i64, vp, vp, vp]),
    "hb_batch_prepare": (i32, [vp, vp, i64, vp]),
    "hb_batch_run": (i32, [vp, i64, vp, vp]),
    "hb_batch_results": (i32, [vp, i64, vp, vp]),
    "hb_batch_tune": (i32, [vp, vp, i64, vp, vp, vp]),
    # served Q1 systems (device-built multigrid)
    "hb_q1_coarse_side": (i32, [i64]),
    "hb_q1_transfers": (i32, [vp, i64, P_ell, P_ell]),
    "hb_q1_galerkin": (i32, [vp, i64, P_ell, P_ell]),
    "hb_q1_create": (i32, [vp, i64, vp, C.POINTER(vp)]),
    "hb_q1_destroy": (i32, [vp]),
    "hb_q1_levels": (i32, [vp, C.POINTER(i32), P_i64]),
    "hb_q1_level": (i32, [vp, i32, P_ell, P_ell, P_ell, P_ell]),
    "hb_q1_solve": (i32, [vp, vp, vp, f64, f64, i64, i64, vp]),
    "hb_q1_set_fused_tail": (i32, [vp, i64]),
    "hb_q1_batch_solve": (i32, [vp, vp, vp, vp, i64, f64, f64, i64, i64, vp, vp]),
    # geometric transfers
    "hb_prolongate_f64": (i32, [vp, i64, vp, vp, vp]),
    "hb_prolongate_f32": (i32, [vp, i64, vp, vp, vp]),
    "hb_restrict_f64": (i32, [vp, i64, vp, vp, vp]),
    "hb_restrict_f32": (i32, [vp, i64, vp, vp, vp]),
    # ELL files
    "hb_ell_file_info": (i32, [C.c_char_p, P_i64]),
    "hb_ell_read_file_f64": (i32, [vp, C.c_char_p, P_ell]),
    "hb_ell_read_file_f32": (i32, [vp, C.c_char_p, P_ell]),
    "hb_ell_write_file": (i32, [vp, P_ell, C.c_char_p]),
    # banded Q1 matrices
    "hb_q1band_root": (i64, [i64]),
    "hb_csr_import_f64": (i32, [vp, vp, vp, vp, P_csr]),
    "hb_csr_import_f32": (i32, [vp, vp, vp, vp, P_csr]),
    "hb_csr_spmv_f64": (i32, [vp, P_csr, vp, vp]),
    "hb_csr_spmv_f32": (i32, [vp, P_csr, vp, vp]),
    "hb_csr_defect_f64": (i32, [vp, P_csr, vp, vp, vp]),
    "hb_csr_defect_f32": (i32, [vp, P_csr, vp, vp, vp]),
    "hb_q1band_spmv_f64": (i32, [vp, P_band, vp, vp]),
    "hb_q1band_spmv_f32": (i32, [vp, P_band, vp, vp]),
    "hb_q1band_defect_f64": (i32, [vp, P_band, vp, vp, vp]),
    "hb_q1band_defect_f32": (i32, [vp, P_band, vp, vp, vp]),
    "hb_q1band_fill_poisson": (i32, [vp, i64, P_band]),
    "hb_q1band_from_ell": (i32, [vp, P_ell, P_band]),
    # serving loop
    "hb_server_create": (i32, [vp, C.POINTER(vp)]),
    "hb_server_submit": (i32, [vp, vp]),
    "hb_server_poll": (i32, [vp, vp, i32, C.POINTER(i32), i32]),
    "hb_server_drain": (i32, [vp]),
    "hb_server_clock": (f64, [vp]),
    "hb_server_stats": (i32, [vp, P_i64, P_i64, P_i64, P_i64]),
    "hb_server_pool_stats": (i32, [vp, P_i64, P_i64]),
    "hb_server_destroy": (i32, [vp]),
}


def lib():
    """The loaded library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m honei_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(status: int) -> str:
    try:
        return lib().hb_status_string(status).decode()
    except Exception:  # pragma: no cover - only when the library cannot load
        return "unknown"


def check(status: int, where: str, ctx=None) -> None:
    if status != 0:
        detail = ""
        if ctx is not None:
            detail = lib().hb_last_error(ctx).decode()
        raise HBError(status, where, detail)
