"""ctypes binding of libswiftb200.so (the C ABI declared in include/swift_b200.h).

The library is loaded from this directory.  There is no fallback: if the shared object is
missing or no sm_100 device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswiftb200.so")

# enums (include/swift_b200.h)
OK, ERR_INVALID_ARG, ERR_BAD_CSR, ERR_BAD_PERM, ERR_UNSUPPORTED, ERR_CUDA, ERR_ALLOC, \
    ERR_OVERFLOW, ERR_TIMEOUT, ERR_NO_DEVICE, ERR_VERIFY = range(11)
F32, F64, BF16, F16 = 0, 1, 2, 3
ROW_MAJOR, COL_MAJOR = 0, 1
HOST, DEVICE = 0, 1
ENGINE_AUTO, ENGINE_TILED, ENGINE_ROWWISE = 0, 1, 2


class SwiftError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})" + (f" -- {detail}" if detail else ""))


class swift_csr(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int),
                ("rowptr", C.c_void_p), ("colidx", C.c_void_p), ("val", C.c_void_p),
                ("val_type", C.c_int), ("mem", C.c_int)]


class swift_plan_opts(C.Structure):
    _fields_ = [("col_perm", C.c_void_p), ("col_perm_mem", C.c_int), ("long_row_split", C.c_int),
                ("build_transpose", C.c_int)]


class swift_plan_stats(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int), ("nsteps", C.c_int),
                ("tilenum", C.c_int), ("regular_nnz", C.c_int), ("reside_col", C.c_int),
                ("reside_nnz", C.c_int), ("numblk", C.c_int), ("fmt_count", C.c_int * 3),
                ("empty_cols", C.c_int), ("max_col_nnz", C.c_int), ("max_row_nnz", C.c_int),
                ("long_rows", C.c_int), ("long_pieces", C.c_int), ("long_row_split", C.c_int),
                ("build_ms", C.c_double), ("device_bytes", C.c_size_t)]


def _slide(vt):
    P, I = C.POINTER(vt), C.POINTER(C.c_int)
    names = ["sortval", "sortrowidx", "tile_ptr", "tile_len", "tile_colidx", "tile_tall",
             "tile_format", "countrow", "segmentoffset", "segptr", "seginfo", "seglength",
             "sortrowindex", "val_position", "val_offset"]
    f = [(n, P if n == "sortval" else I) for n in names]
    f += [("tilenum", C.c_int), ("segsum", C.c_int), ("regular_nnz", C.c_int),
          ("reside_col", C.c_int), ("reside_nnz", C.c_int), ("reside_cscptr", I),
          ("reside_cscrowidx", I), ("reside_val", P), ("numblk", C.c_int),
          ("colorblk", C.POINTER(C.c_uint)), ("blkstart", I), ("blkstop", I), ("blkptr", I)]
    return type("swift_slide_matrix", (C.Structure,), {"_fields_": f})


swift_slide_matrix_f32 = _slide(C.c_float)
swift_slide_matrix_f64 = _slide(C.c_double)

_lib = None

# (name, restype, argtypes)
_P = C.c_void_p
_I64 = C.c_int64
_SIGS = [
    ("swift_status_string", C.c_char_p, [C.c_int]),
    ("swift_version", C.c_char_p, []),
    ("swift_last_error", C.c_char_p, []),
    ("swift_device_check", C.c_int, [C.POINTER(C.c_int)] * 3),
    ("swift_plan_create", C.c_int, [C.POINTER(swift_csr), C.POINTER(swift_plan_opts), _P, C.POINTER(_P)]),
    ("swift_plan_destroy", C.c_int, [_P]),
    ("swift_plan_get_stats", C.c_int, [_P, C.POINTER(swift_plan_stats)]),
    ("swift_plan_export_f32", C.c_int, [_P, C.POINTER(swift_slide_matrix_f32), C.c_int, C.POINTER(C.c_float)]),
    ("swift_plan_export_f64", C.c_int, [_P, C.POINTER(swift_slide_matrix_f64), C.c_int, C.POINTER(C.c_float)]),
    ("swift_slide_free_f32", None, [C.POINTER(swift_slide_matrix_f32)]),
    ("swift_slide_free_f64", None, [C.POINTER(swift_slide_matrix_f64)]),
    ("swift_plan_export_sorted", C.c_int, [_P, _P, _P, _P, _P]),
    ("swift_spmm", C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P, _I64, C.c_int, C.c_int, _P, _I64, C.c_int, _P]),
    ("swift_spmm_transposed", C.c_int, [_P, C.c_int, C.c_int, _P, _I64, _P, _I64, _P]),
    ("swift_sddmm", C.c_int, [_P, C.c_int, C.c_int, _P, _I64, _P, _I64, _P, _P]),
    ("swift_fused_forward_backward", C.c_int, [_P, C.c_int, C.c_int, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _P]),
    ("swift_spmm_f64_reference", C.c_int, [_P, C.c_int, _P, _I64, _P, _I64, _P]),
    ("swift_plan_autotune", C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("swift_spmm_noalloc", C.c_int, [_P, C.c_int, C.c_int, _P, _I64, _P, _I64, _P]),
    ("swift_plan_set_rowwise_params", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("swift_plan_get_rowwise_params", C.c_int, [_P, C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 4),
    ("swift_batch_create", C.c_int, [C.POINTER(_P), C.c_int, _P, C.POINTER(_P)]),
    ("swift_batch_destroy", C.c_int, [_P]),
    ("swift_batch_set_operands", C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    ("swift_batch_run", C.c_int, [_P, _P]),
    ("swift_batch_run_graph", C.c_int, [_P, _P]),
]


def lib():
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python __graft_entry__.py` "
                          "(nvcc, sm_100a); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    for name, res, args in _SIGS:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def status_string(s: int) -> str:
    try:
        return lib().swift_status_string(s).decode()
    except ImportError:
        return str(s)


def check(status: int, what: str):
    if status != OK:
        raise SwiftError(status, what, lib().swift_last_error().decode())
    return status
