"""ctypes binding of libpiro_b200.so (the C ABI declared in include/piro.h).

The library is the product path: there is no CPU fallback.  `lib()` raises if
the shared library is missing or does not export a declared symbol, and every
wrapper in piro_b200.ops raises PiroError on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libpiro_b200.so")
HEADERS = [os.path.join(ROOT, "include", "piro.h")]

i32, i64, f32, f64, vp, sz = C.c_int, C.c_int64, C.c_float, C.c_double, C.c_void_p, C.c_size_t
pi64 = C.POINTER(C.c_int64)
psz = C.POINTER(C.c_size_t)
pint = C.POINTER(C.c_int)


class Buf(C.Structure):
    _fields_ = [("id", C.c_int32), ("n", C.c_int64)]


class Op(C.Structure):
    _fields_ = [("kind", C.c_int32)]


class CaseInfo(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("n_cells", C.c_int64),
                ("timescheme", C.c_int32), ("spacescheme", C.c_int32), ("solverscheme", C.c_int32),
                ("datatype", C.c_int32), ("simindex", C.c_int32), ("timestep", C.c_float), ("totaltime", C.c_float),
                ("steps_done", C.c_int64), ("n_fields", C.c_int32), ("bc_cells", C.c_int64)]


class BeInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("outer_iterations", C.c_int), ("inner_iterations", C.c_int),
                ("fallbacks", C.c_int), ("rel_residual", C.c_double)]


# name -> (restype, argtypes).  Pointers to device memory are passed as
# integers (c_void_p).
SIGNATURES = {
    "piro_status_string": (C.c_char_p, [i32]),
    "piro_last_error": (C.c_char_p, []),
    "piro_version": (C.c_char_p, []),
    "piro_set_wait_limit": (i32, [C.c_longlong]),
    "piro_laplacian_nnz": (i32, [i32, i32, i32, pi64]),
    "piro_csr_laplacian": (i32, [i32, i32, i32, i32, f32, vp, vp, vp, vp]),
    "piro_coo_laplacian": (i32, [i32, i32, i32, i32, f32, vp, vp, vp, vp]),
    "piro_gradient_nnz": (i32, [i32, i32, i32, i32, pi64]),
    "piro_csr_gradient": (i32, [i32, i32, i32, i32, i32, f32, vp, vp, vp, vp]),
    "piro_gradient_nnz_rows": (i32, [i32, i32, i32, i32, i64, i64, pi64]),
    "piro_csr_gradient_rows": (i32, [i32, i32, i32, i32, i32, f32, i64, i64, i64, vp, vp, vp, vp]),
    "piro_csr_rowscale": (i32, [i64, vp, vp, vp, vp]),
    "piro_ht_table_size": (i32, [i64, i64, i32, f32, f32, f32, f32, pi64]),
    "piro_ht_build_workspace": (i32, [i64, psz]),
    "piro_ht_build": (i32, [i64, vp, vp, vp, i64, i64, vp, vp, vp, sz, vp]),
    "piro_csr_fe_step": (i32, [i32, i32, i32, vp, vp, vp, f32, vp, vp, vp]),
    "piro_csr_fe_step_bc": (i32, [i32, i32, i32, vp, vp, vp, f32, vp, vp, vp, vp]),
    "piro_csr_i1": (i32, [i32, i32, i32, vp, vp, vp, f32, vp, vp, vp]),
    "piro_coo_spmv": (i32, [i64, i64, vp, vp, vp, f32, vp, vp, vp]),
    "piro_coo_fe_step": (i32, [i64, i64, vp, vp, vp, f32, vp, vp, vp]),
    "piro_coo_row_index": (i32, [i64, i64, vp, vp, vp, sz, vp]),
    "piro_coo_step_indexed": (i32, [i64, vp, vp, vp, f32, i32, vp, vp, vp]),
    "piro_ht_spmv": (i32, [i32, i32, i32, vp, vp, i64, f32, i32, vp, vp, vp]),
    "piro_ht_row_order_workspace": (i32, [i64, i64, C.POINTER(sz)]),
    "piro_ht_row_order": (i32, [i64, i64, vp, vp, sz, vp]),
    "piro_ht_spmv_ordered": (i32, [i32, i32, i32, vp, vp, i64, f32, i32, vp, vp, vp, vp]),
    "piro_ht_stage_bytes": (i32, [i64, C.POINTER(sz)]),
    "piro_ht_spmv_staged": (i32, [i32, i32, i32, vp, vp, i64, f32, i32, vp, vp, sz, vp, vp, vp]),
    "piro_dense_laplacian": (i32, [i32, i32, i32, i32, f32, vp, sz, vp]),
    "piro_dense_fe_step": (i32, [i64, vp, f32, vp, vp, vp]),
    "piro_dense_check": (i32, [vp]),
    "piro_stencil_check": (i32, [vp]),
    "piro_ht_lu_reference": (i32, [i64, vp, vp, i64, vp]),
    "piro_ht_lu_band_bytes": (i32, [i64, i64, C.POINTER(sz)]),
    "piro_ht_lu_factor": (i32, [i64, i64, vp, vp, i64, f32, f32, vp, sz, vp]),
    "piro_ht_lu_solve": (i32, [i64, i64, vp, sz, vp, vp, vp]),
    "piro_ht_lu_pivots": (i32, [i64, i64, vp, sz, vp]),
    "piro_stencil_fe_step": (i32, [i32, i32, i32, f32, f32, f32, f32, vp, vp, vp, vp]),
    "piro_set_bc": (i32, [i64, vp, vp, vp, vp]),
    "piro_face_count": (i32, [i32, i32, i32, pi64, pi64]),
    "piro_face_lists": (i32, [i32, i32, i32, vp, vp]),
    "piro_vec_op": (i32, [i32, i64, vp, vp, vp, vp]),
    "piro_vec_op_scalar": (i32, [i32, i64, f32, vp, vp, vp]),
    "piro_vec_urf": (i32, [i64, vp, vp, f32, vp]),
    "piro_scan_workspace": (i32, [i64, psz]),
    "piro_csrgeam3": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz, vp]),
    "piro_csrgeam3_noalloc": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "piro_csrgeam2_count": (i32, [i64, vp, vp, vp, vp, vp, vp, sz, vp]),
    "piro_csrgeam2_fill": (i32, [i64, vp, vp, vp, f32, vp, vp, vp, vp, vp, vp, vp]),
    "piro_csr_identity": (i32, [i64, vp, vp, vp, vp]),
    "piro_reduce_workspace": (i32, [i64, psz]),
    "piro_dot_f64": (i32, [i64, vp, vp, vp, vp, sz, vp]),
    "piro_be_create": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "piro_be_create_stencil": (i32, [i32, i32, i32, vp, vp, vp, vp, f32, f32, vp, C.POINTER(vp)]),
    "piro_be_inner_operator": (i32, [vp, pint]),
    "piro_be_persistent_bytes": (i32, [vp, C.POINTER(C.c_double)]),
    "piro_be_solve": (i32, [vp, vp, vp, f64, i32, i32, C.POINTER(BeInfo)]),
    "piro_be_solution_f64": (i32, [vp, C.POINTER(vp)]),
    "piro_be_kernel_stats": (i32, [vp, i32, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                   C.POINTER(C.c_longlong)]),
    "piro_be_destroy": (i32, [vp]),
    "piro_be_jli": (i32, [i32, i32, i32, vp, vp, vp, f32, vp, vp, vp, f32, f32, i32, pint, vp]),
    "piro_pcnet_num_params": (i32, [pi64]),
    "piro_pcnet_create": (i32, [C.c_uint64, C.POINTER(vp)]),
    "piro_pcnet_get_params": (i32, [vp, vp, i64, i32]),
    "piro_pcnet_set_params": (i32, [vp, vp, i64]),
    "piro_pcnet_forward": (i32, [vp, i32, i32, i32, i32, vp, vp, vp, vp]),
    "piro_pcnet_loss_grad": (i32, [vp, i32, i32, i32, i32, vp, vp, vp, vp, C.POINTER(C.c_double), vp, vp]),
    "piro_pcnet_adam_step": (i32, [vp, f32, vp]),
    "piro_pcnet_stats": (i32, [vp, C.POINTER(C.c_longlong)]),
    "piro_pcnet_set_engine": (i32, [vp, i32]),
    "piro_pcnet_destroy": (i32, [vp]),
    "piro_be_set_preconditioner": (i32, [vp, i32, vp]),
    "piro_be_pc_stats": (i32, [vp, i32, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
    "piro_write_paraview": (i32, [vp, C.c_char_p, i32]),
    "piro_set_output": (i32, [vp, C.c_char_p]),
    "piro_interior_gather": (i32, [i32, i32, i32, i32, vp, vp, vp]),
    "piro_laplacian_nnz_rows": (i32, [i32, i32, i32, i64, i64, pi64]),
    "piro_csr_laplacian_rows": (i32, [i32, i32, i32, i32, f32, i64, i64, i64, vp, vp, vp, vp]),
    "piro_csr_fe_step_rows": (i32, [i32, i32, i32, i64, i64, vp, vp, vp, f32, vp, i64, vp, vp]),
    "piro_slab_workspace": (i32, [pi64]),
    "piro_slab_be_residual": (i32, [i32, i32, i32, i32, i32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "piro_slab_cg_spmv": (i32, [i32, i32, i32, i32, i32, f32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "piro_slab_cg_update": (i32, [i32, i32, i32, i32, i32, f32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "piro_slab_x_update": (i32, [i32, i32, i32, i32, i32, vp, vp, vp]),
    "piro_slab_cg_spmv_dev": (i32, [i32, i32, i32, i32, i32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "piro_slab_cg_update_dev": (i32, [i32, i32, i32, i32, i32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                      vp]),
    "piro_slab_cg_scalars": (i32, [vp, vp, vp, vp]),
    "piro_batch_create": (i32, [i32, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "piro_batch_layout": (i32, [vp, vp, pi64]),
    "piro_batch_set_fields": (i32, [vp, vp, i32]),
    "piro_batch_get_fields": (i32, [vp, vp, i32]),
    "piro_batch_field_ptr": (i32, [vp, C.POINTER(vp)]),
    "piro_batch_step": (i32, [vp, i32, f64, C.POINTER(C.c_double)]),
    "piro_batch_member_info": (i32, [vp, vp, vp, vp, vp]),
    "piro_batch_autotune": (i32, [vp, f64, pint, pint]),
    "piro_batch_schedule": (i32, [vp, pint]),
    "piro_batch_set_schedule": (i32, [vp, i32, i32]),
    "piro_batch_destroy": (i32, [vp]),
    "piro_open": (i32, [C.c_char_p, C.c_char_p, C.POINTER(vp)]),
    "piro_close": (None, [vp]),
    "piro_ctx_query": (i32, [vp, C.POINTER(CaseInfo)]),
    "piro_set_alpha_mode": (i32, [vp, i32]),
    "piro_set_lu_mode": (i32, [vp, i32]),
    "piro_ddt_r": (i32, [vp, C.c_char_p, C.POINTER(Buf)]),
    "piro_vector": (i32, [vp, C.c_char_p, C.POINTER(Buf)]),
    "piro_field": (i32, [vp, C.c_char_p, C.POINTER(Buf)]),
    "piro_field_upload": (i32, [vp, Buf, vp, i64]),
    "piro_field_download": (i32, [vp, Buf, vp, i64]),
    "piro_field_device_ptr": (i32, [vp, Buf, C.POINTER(vp)]),
    "piro_laplacian": (i32, [vp, C.c_char_p, C.c_char_p, C.POINTER(Op)]),
    "piro_gradient": (i32, [vp, C.c_char_p, C.POINTER(Op)]),
    "piro_dot": (i32, [vp, Buf, Op, C.POINTER(Op)]),
    "piro_div": (i32, [vp, C.c_char_p, C.c_char_p, C.POINTER(Op)]),
    "piro_assign": (i32, [vp, Buf, Op, C.POINTER(Buf)]),
    "piro_step_solve": (i32, [vp, Buf, f32]),
    "piro_solve": (i32, [vp, C.POINTER(C.c_int64)]),
    "piro_op_export_csr": (i32, [vp, Op, vp, vp, vp, i64, C.POINTER(C.c_int64)]),
}


def declared_symbols() -> list[str]:
    """Every function name declared in include/*.h."""
    names = []
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(piro_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


_lib = None


def lib() -> C.CDLL:
    """Load libpiro_b200.so; raise if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m piro_b200.build` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class PiroError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.piro_last_error().decode(errors="replace")
        name = L.piro_status_string(status).decode()
        super().__init__(f"{where}: {name} ({status}): {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != 0:
        raise PiroError(status, where)
