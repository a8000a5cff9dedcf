"""ctypes binding of the C ABI declared in ``include/rvvla.h``.

The shared library is built in-tree (``rvvlasparse_b200/lib/librvvla_b200.so``)
by ``rvvlasparse_b200.build``.  Loading fails loudly when it is missing: there
is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "librvvla_b200.so")

RVVLA_OK = 0
RVVLA_ERR_INVALID_ARG = 1
RVVLA_ERR_CUDA = 2
RVVLA_ERR_FORMAT = 3
RVVLA_ERR_UNSUPPORTED = 4
RVVLA_ERR_TOO_LARGE = 5
RVVLA_ERR_TIMEOUT = 6
RVVLA_ERR_NO_DEVICE = 7
RVVLA_ERR_IO = 8

RVVLA_F64 = 0
RVVLA_F32 = 1
RVVLA_BF16 = 2

i64 = C.c_int64
i32 = C.c_int32
u64 = C.c_uint64
vp = C.c_void_p
dbl = C.c_double
flt = C.c_float
cint = C.c_int


class RvvlaError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


class rvvla_host_crs(C.Structure):
    _fields_ = [("m", i64), ("n", i64), ("nz", i64), ("Rst", vp), ("Col", vp), ("Val", vp)]


class rvvla_crs(C.Structure):
    _fields_ = [("m", i64), ("n", i64), ("nz", i64), ("Rst", vp), ("Col", vp), ("Val", vp), ("plan", vp),
                ("plan_tiles", i64), ("plan_kind", i32)]


class rvvla_sell(C.Structure):
    _fields_ = [("m", i64), ("n", i64), ("cnt_b", i64), ("nz", i64), ("C", i32), ("Sigma", i32), ("vCl", vp),
                ("vCs", vp), ("vBs", vp), ("vSBs", vp), ("vCol", vp), ("vPerm", vp), ("vVal", vp), ("len", i64)]


class rvvla_sell_owned(C.Structure):
    _fields_ = [("h", rvvla_sell), ("vCl", vp), ("vCs", vp), ("vBs", vp), ("vSBs", vp), ("vCol", vp),
                ("vPerm", vp), ("vVal", vp)]


VNEC_ARRAYS = ("ptr", "indices", "val", "thread_coord_start", "thread_coord_end", "ecr_indices", "NEC_NUM",
               "use_x_ptr", "use_x_indices", "v_row_ptr", "col_start", "val_align", "tasks", "task_start",
               "task_end", "spvv_len", "row_begin", "row_end", "reorder_col", "reorder_nnz", "plan")


class rvvla_transpose(C.Structure):
    _fields_ = [("AT", rvvla_crs), ("perm", vp), ("val_bytes", i32)]


class rvvla_transpose_owned(C.Structure):
    _fields_ = [("h", rvvla_transpose), ("Rst", vp), ("Col", vp), ("perm", vp), ("plan", vp), ("Val", vp)]


class rvvla_batch(C.Structure):
    _fields_ = [("count", i64), ("k", i64), ("x_len", i64), ("y_len", i64), ("ntiles", i64), ("val_bytes", i32),
                ("grid", i32), ("block", i32), ("mats", vp), ("tiles", vp)]


class rvvla_batch_owned(C.Structure):
    _fields_ = [("h", rvvla_batch), ("mats", vp), ("tiles", vp), ("x_off", C.POINTER(i64)),
                ("y_off", C.POINTER(i64)), ("sell", vp), ("nmats", i64)]


class rvvla_lav(C.Structure):
    _fields_ = [("SIMD_Lanes", i64), ("m", i64), ("n", i64), ("nz", i64), ("segment_count", i64),
                ("chunk_count", i64), ("segment_len", i64), ("n_steps", i64), ("T", dbl), ("chunk_offsets", vp),
                ("chunk_offsets_full_mask", vp), ("segment_ptr", vp), ("out_order", vp), ("mask", vp), ("val", vp),
                ("col_id", vp), ("sparse_part", rvvla_crs), ("row_order", vp), ("lane_of_slot", vp),
                ("long_chunks", i64)]


class rvvla_lav_owned(C.Structure):
    _fields_ = [("h", rvvla_lav), ("chunk_offsets", vp), ("chunk_offsets_full_mask", vp), ("segment_ptr", vp),
                ("out_order", vp), ("mask", vp), ("val", vp), ("col_id", vp), ("sp_Rst", vp), ("sp_Col", vp),
                ("sp_Val", vp), ("row_order", vp), ("lane_of_slot", vp), ("sp_plan", vp)]


class rvvla_vnec(C.Structure):
    _fields_ = [("m", i64), ("n", i64), ("nz", i64), ("NUM_THREADS_VNEC", i32), ("nLanes", i32), ("vnec_t", i32),
                ("max_nec", i32), ("IRD_mat", flt), ("ptr", vp), ("indices", vp), ("val", vp),
                ("thread_coord_start", vp), ("thread_coord_end", vp), ("ecr_indices", vp), ("NEC_NUM", vp),
                ("use_x_ptr", vp), ("use_x_indices", vp), ("v_row_ptr", vp), ("col_start", vp),
                ("val_align", vp), ("ngroups", i64), ("tasks", vp), ("task_start", vp), ("task_end", vp),
                ("spvv_len", vp), ("row_begin", vp), ("row_end", vp), ("reorder_col", vp), ("reorder_nnz", vp),
                ("ntasks", i64), ("nreorder", i64), ("plan", vp), ("plan_tiles", i64), ("plan_kind", i32)]


class rvvla_vnec_owned(C.Structure):
    _fields_ = [("h", rvvla_vnec)] + [(k, vp) for k in VNEC_ARRAYS]


class rvvla_vhcc(C.Structure):
    _fields_ = [("num_rows", i64), ("num_cols", i64), ("num_entries", i64), ("num_vectors", i64),
                ("pad_entries", i64), ("pad_rows", i64), ("num_threads", i32), ("num_panels", i32),
                ("tile_row", i32), ("tile_col", i32), ("vec_size", i32), ("n_masks", i32), ("thr_info", vp),
                ("veceor_ptr", vp), ("n_eor", i64), ("scan_mask", vp), ("scan_mask_bytes", i64), ("row_arr", vp),
                ("n_rowarr", i64), ("col_arr", vp), ("vals_arr", vp)]


class rvvla_vhcc_owned(C.Structure):
    _fields_ = [("h", rvvla_vhcc), ("thr_info", vp), ("veceor_ptr", vp), ("scan_mask", vp), ("row_arr", vp),
                ("col_arr", vp), ("vals_arr", vp)]


class rvvla_cvr(C.Structure):
    _fields_ = [("nItems", i64), ("numRows", i64), ("numCols", i64), ("SIMD_LEN", i32), ("Nthreads", i32),
                ("Nthreads_avail", i32), ("no_empty_rows", i32), ("vPack_vec_vals", vp), ("vPack_vec_cols", vp),
                ("vPack_vec_record", vp), ("n_record", i64), ("writeback_pos_record", vp), ("n_writeback", i64)]


class rvvla_cvr_owned(C.Structure):
    _fields_ = [("h", rvvla_cvr), ("vPack_vec_vals", vp), ("vPack_vec_cols", vp), ("vPack_vec_record", vp),
                ("writeback_pos_record", vp)]


class rvvla_csr5(C.Structure):
    _fields_ = [("m", i64), ("n", i64), ("nnz", i64), ("bit_y_offset", i32), ("bit_seg_offset", i32),
                ("tile_desc_len", i32), ("tail_tile_start", i32), ("p", i32), ("omega", i32), ("sigma", i32),
                ("num_offsets", i32), ("csr_row_pointer", vp), ("csr_column_index", vp), ("csr_value", vp),
                ("tile_pointer", vp), ("tile_descriptor", vp), ("tile_empty_offset_pointer", vp),
                ("tile_empty_offset", vp), ("no_empty_rows", i32)]


class rvvla_csr5_owned(C.Structure):
    _fields_ = [("h", rvvla_csr5), ("csr_row_pointer", vp), ("csr_column_index", vp), ("csr_value", vp),
                ("tile_pointer", vp), ("tile_descriptor", vp), ("tile_empty_offset_pointer", vp),
                ("tile_empty_offset", vp)]


class rvvla_hcsr(C.Structure):
    _fields_ = [("R", i64), ("C", i64), ("m", i64), ("n", i64), ("nz", i64), ("b_m", i64), ("b_n", i64),
                ("block_ptr", vp), ("row_offset", vp), ("row_ptr", vp), ("col_idx", vp), ("values", vp),
                ("row_ptr_len", i64)]


class rvvla_hcsr_owned(C.Structure):
    _fields_ = [("h", rvvla_hcsr), ("block_ptr", vp), ("row_offset", vp), ("row_ptr", vp), ("col_idx", vp),
                ("values", vp)]


RVVLA_FMT_HCSR, RVVLA_FMT_SELL, RVVLA_FMT_CSR5, RVVLA_FMT_LAV, RVVLA_FMT_VHCC, RVVLA_FMT_CVR = 1, 2, 3, 4, 5, 6


class rvvla_tune_params(C.Structure):
    _fields_ = [("R", i64), ("C", i64), ("p", C.c_double), ("sigma", i64), ("threads", i64), ("simd_lanes", i64),
                ("segment_len", i64), ("T", C.c_double)]


_lib = None


def _proto(lib, name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)


def load():
    """Load the library (once) and declare every prototype of rvvla.h."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA extension first "
            "(python -m rvvlasparse_b200.build); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    _proto(lib, "rvvla_version", C.c_char_p)
    _proto(lib, "rvvla_status_string", C.c_char_p, cint)
    _proto(lib, "rvvla_last_error", C.c_char_p)
    _proto(lib, "rvvla_device_info", cint, P(cint), P(cint), P(cint))
    _proto(lib, "rvvla_kernel_launch_count", u64)
    _proto(lib, "rvvla_memcpy", cint, vp, vp, C.c_size_t, vp)
    _proto(lib, "rvvla_copy_h2d", cint, vp, vp, C.c_size_t, vp)
    _proto(lib, "rvvla_autotune", cint, cint, P(rvvla_crs), cint, cint, cint, P(rvvla_tune_params),
           P(C.c_double), P(rvvla_tune_params), P(C.c_double), cint, P(cint), vp)
    _proto(lib, "rvvla_copy_d2h", cint, vp, vp, C.c_size_t, vp)
    _proto(lib, "rvvla_malloc", cint, P(vp), C.c_size_t)
    _proto(lib, "rvvla_free", cint, vp)
    _proto(lib, "rvvla_device_status", cint, P(cint), vp)
    # CRS
    _proto(lib, "rvvla_crs_plan_len", i64, i64, i64, cint)
    _proto(lib, "rvvla_crs_analyze", cint, P(rvvla_crs), cint, vp, P(i64), P(i32), vp)
    _proto(lib, "rvvla_crs_spmv_f64", cint, P(rvvla_crs), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_crs_spmv_f32", cint, P(rvvla_crs), flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_crs_spmv_mixed", cint, P(rvvla_crs), cint, flt, vp, flt, vp, vp)
    # HCSR
    _proto(lib, "rvvla_hcsr_build", cint, P(rvvla_crs), cint, i64, i64, dbl, P(rvvla_hcsr_owned), vp)
    _proto(lib, "rvvla_hcsr_free", None, P(rvvla_hcsr_owned))
    _proto(lib, "rvvla_hcsr_spmv_f64", cint, P(rvvla_hcsr), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_hcsr_spmv_f32", cint, P(rvvla_hcsr), flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_hcsr_spmv_mixed", cint, P(rvvla_hcsr), cint, flt, vp, flt, vp, vp)
    # SELL-C-sigma
    _proto(lib, "rvvla_sell_build", cint, P(rvvla_crs), cint, i64, i64, P(rvvla_sell_owned), vp)
    _proto(lib, "rvvla_sell_free", None, P(rvvla_sell_owned))
    _proto(lib, "rvvla_sell_spmv_f64", cint, P(rvvla_sell), cint, dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_sell_spmv_f32", cint, P(rvvla_sell), cint, flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_sell_spmv_mixed", cint, P(rvvla_sell), cint, flt, vp, flt, vp, vp)
    # LAV
    _proto(lib, "rvvla_lav_build", cint, P(rvvla_crs), cint, i64, dbl, i64, P(rvvla_lav_owned), vp)
    _proto(lib, "rvvla_lav_free", None, P(rvvla_lav_owned))
    _proto(lib, "rvvla_lav_spmv_f64", cint, P(rvvla_lav), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_lav_spmv_f32", cint, P(rvvla_lav), flt, vp, flt, vp, vp)
    # VNEC
    _proto(lib, "rvvla_vnec_build", cint, P(rvvla_crs), cint, i64, cint, P(rvvla_vnec_owned), vp)
    _proto(lib, "rvvla_vnec_free", None, P(rvvla_vnec_owned))
    _proto(lib, "rvvla_vnec_spmv_f64", cint, P(rvvla_vnec), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_vnec_spmv_f32", cint, P(rvvla_vnec), flt, vp, flt, vp, vp)
    # VHCC
    _proto(lib, "rvvla_vhcc_build", cint, P(rvvla_crs), cint, i64, P(rvvla_vhcc_owned), vp)
    _proto(lib, "rvvla_vhcc_free", None, P(rvvla_vhcc_owned))
    _proto(lib, "rvvla_vhcc_spmv_f64", cint, P(rvvla_vhcc), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_vhcc_spmv_f32", cint, P(rvvla_vhcc), flt, vp, flt, vp, vp)
    # CVR
    _proto(lib, "rvvla_cvr_build", cint, P(rvvla_crs), cint, i64, P(rvvla_cvr_owned), vp)
    _proto(lib, "rvvla_cvr_free", None, P(rvvla_cvr_owned))
    _proto(lib, "rvvla_cvr_spmv_f64", cint, P(rvvla_cvr), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_cvr_spmv_f32", cint, P(rvvla_cvr), flt, vp, flt, vp, vp)
    # CSR5
    _proto(lib, "rvvla_csr5_build", cint, P(rvvla_crs), cint, cint, cint, P(rvvla_csr5_owned), vp)
    _proto(lib, "rvvla_csr5_free", None, P(rvvla_csr5_owned))
    _proto(lib, "rvvla_csr5_spmv_f64", cint, P(rvvla_csr5), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_csr5_spmv_f32", cint, P(rvvla_csr5), flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_csr5_spmv_mixed", cint, P(rvvla_csr5), cint, flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_csr5_spmv_f64_noalloc", cint, P(rvvla_csr5), dbl, vp, dbl, vp, vp)
    # adjoint
    _proto(lib, "rvvla_csr_transpose", cint, P(rvvla_crs), cint, P(rvvla_transpose_owned), vp)
    _proto(lib, "rvvla_csr_transpose_free", None, P(rvvla_transpose_owned))
    _proto(lib, "rvvla_csr_transpose_values", cint, P(rvvla_transpose), vp, vp, vp)
    _proto(lib, "rvvla_spmv_adjoint_x_f64", cint, P(rvvla_transpose), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_spmv_adjoint_x_f32", cint, P(rvvla_transpose), flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_spmv_adjoint_x_values_f64", cint, P(rvvla_transpose), vp, dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_spmv_adjoint_x_values_f32", cint, P(rvvla_transpose), vp, flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_sddmm_values_f64", cint, P(rvvla_crs), vp, vp, vp, vp)
    _proto(lib, "rvvla_sddmm_values_f32", cint, P(rvvla_crs), vp, vp, vp, vp)
    # batched
    _proto(lib, "rvvla_batched_plan", cint, P(rvvla_crs), i64, cint, cint, vp, vp, P(rvvla_batch_owned), vp)
    _proto(lib, "rvvla_batched_free", None, P(rvvla_batch_owned))
    _proto(lib, "rvvla_batched_spmv_f64", cint, P(rvvla_batch), dbl, vp, dbl, vp, vp)
    _proto(lib, "rvvla_batched_spmv_f32", cint, P(rvvla_batch), flt, vp, flt, vp, vp)
    _proto(lib, "rvvla_batched_graph", cint, P(rvvla_batch), dbl, vp, dbl, vp, vp, P(vp))
    _proto(lib, "rvvla_batched_graph_launch", cint, vp, vp)
    _proto(lib, "rvvla_batched_graph_free", None, vp)
    _proto(lib, "rvvla_batched_autotune", cint, P(rvvla_crs), i64, cint, cint, vp, vp, P(dbl), vp)
    # workloads
    _proto(lib, "rvvla_gen_laplace2d", i64, i64, vp, vp, vp)
    _proto(lib, "rvvla_gen_stencil27", i64, i64, u64, vp, vp, vp)
    _proto(lib, "rvvla_gen_powerlaw", i64, i64, dbl, dbl, i64, i64, dbl, u64, vp, vp, vp)
    _proto(lib, "rvvla_gen_random_rows", i64, i64, i64, cint, dbl, cint, u64, vp, vp, vp)
    _proto(lib, "rvvla_gen_vector", None, i64, u64, cint, dbl, dbl, vp)
    _proto(lib, "rvvla_cg_f64", cint, P(rvvla_crs), vp, vp, i64, dbl, i64, P(i64), P(dbl), vp)
    _proto(lib, "rvvla_cg_f32", cint, P(rvvla_crs), vp, vp, i64, dbl, i64, P(i64), P(dbl), vp)
    _proto(lib, "rvvla_bicgstab_f64", cint, P(rvvla_crs), vp, vp, i64, dbl, i64, P(i64), P(dbl), P(cint), vp)
    _proto(lib, "rvvla_bicgstab_f32", cint, P(rvvla_crs), vp, vp, i64, dbl, i64, P(i64), P(dbl), P(cint), vp)
    _proto(lib, "rvvla_crs_spmv_dot_f64", cint, P(rvvla_crs), vp, vp, vp, vp)
    _proto(lib, "rvvla_crs_spmv_dot_f32", cint, P(rvvla_crs), vp, vp, vp, vp)
    cp = C.c_char_p
    _proto(lib, "rvvla_host_crs_free", None, P(rvvla_host_crs))
    _proto(lib, "rvvla_mm_read", cint, cp, P(rvvla_host_crs))
    _proto(lib, "rvvla_mm_write", cint, cp, i64, i64, vp, vp, vp)
    _proto(lib, "rvvla_crs_save", cint, cp, i64, i64, i64, vp, vp, vp, cint)
    _proto(lib, "rvvla_crs_load_info", cint, cp, P(i64), P(i64), P(i64), P(cint))
    _proto(lib, "rvvla_crs_load", cint, cp, vp, vp, vp)
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != RVVLA_OK:
        lib = load()
        raise RvvlaError(status, where, lib.rvvla_last_error().decode())


def declared_symbols() -> list[str]:
    """Function names declared in include/rvvla.h (parsed from the header)."""
    import re

    hdr = os.path.join(os.path.dirname(_HERE), "include", "rvvla.h")
    text = open(hdr).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rvvla_[a-z0-9_]+)\s*\(", text)))
