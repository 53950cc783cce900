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
    ERR_OVERFLOW, ERR_TIMEOUT, ERR_NO_DEVICE, ERR_VERIFY, ERR_IO, ERR_FORMAT = range(13)
F32, F64, BF16, F16 = 0, 1, 2, 3
ROW_MAJOR, COL_MAJOR = 0, 1
HOST, DEVICE = 0, 1
ENGINE_AUTO, ENGINE_TILED, ENGINE_ROWWISE, ENGINE_TILED_GROUPED, ENGINE_BAND = 0, 1, 2, 3, 4
BAND_PROFILE_MAX = 128


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

# array name -> (length as a function of the struct, numpy dtype; None = the value type)
_SLIDE_LEN = {
    "tile_ptr": (lambda s: s.tilenum + 1, "i4"), "tile_len": (lambda s: s.tilenum, "i4"),
    "tile_colidx": (lambda s: s.tilenum, "i4"), "tile_tall": (lambda s: s.tilenum, "i4"),
    "tile_format": (lambda s: s.tilenum, "i4"), "sortrowidx": (lambda s: s.regular_nnz, "i4"),
    "sortval": (lambda s: s.regular_nnz, None), "countrow": (lambda s: s.tilenum + 1, "i4"),
    "segmentoffset": (lambda s: s.segsum + 1, "i4"), "sortrowindex": (lambda s: s.regular_nnz, "i4"),
    "val_position": (lambda s: s.regular_nnz, "i4"), "val_offset": (lambda s: s.regular_nnz, "i4"),
    "reside_cscptr": (lambda s: s.reside_col + 1, "i4"), "reside_cscrowidx": (lambda s: s.reside_nnz, "i4"),
    "reside_val": (lambda s: s.reside_nnz, None), "colorblk": (lambda s: s.numblk, "u4"),
    "blkstart": (lambda s: s.numblk, "i4"), "blkstop": (lambda s: s.numblk, "i4"),
    "blkptr": (lambda s: s.numblk, "i4"),
}
_SLIDE_INTS = ("tilenum", "regular_nnz", "reside_col", "reside_nnz", "numblk", "segsum")


def slide_arrays(s, vdt, with_row_sort=True) -> dict:
    """numpy copies of the arrays a slide_matrix struct holds (NULL pointers are skipped)."""
    import numpy as np
    out = {k: int(getattr(s, k)) for k in _SLIDE_INTS}
    for name, (n_of, dt) in _SLIDE_LEN.items():
        if not with_row_sort and name in ("val_position", "val_offset"):
            continue
        ptr, n = getattr(s, name), n_of(s)
        if not ptr:
            continue
        out[name] = (np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt or vdt, copy=True)
                     if n > 0 else np.zeros(0, dt or vdt))
    return out


def slide_from_arrays(d: dict, vdt):
    """A slide_matrix struct pointing at numpy arrays of `d`; returns (struct, keep-alive list)."""
    import numpy as np
    S = swift_slide_matrix_f64 if np.dtype(vdt) == np.float64 else swift_slide_matrix_f32
    s, keep = S(), []
    for k in _SLIDE_INTS:
        setattr(s, k, int(d.get(k, 0)))
    for name, (_, dt) in _SLIDE_LEN.items():
        if name not in d:
            continue
        a = np.ascontiguousarray(d[name], dtype=dt or vdt)
        if a.size == 0:
            a = np.zeros(1, dt or vdt)
        keep.append(a)
        setattr(s, name, a.ctypes.data_as(type(getattr(s, name))))
    return s, keep

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
    ("swift_plan_set_values", C.c_int, [_P, _P, C.c_int, _P]),
    ("swift_plan_is_symmetric", C.c_int, [_P, C.POINTER(C.c_int), _P]),
    ("swift_plan_band_profile", C.c_int, [_P, _P, C.POINTER(C.c_int), _P]),
    ("swift_band_timeout_flag", C.c_int, [C.POINTER(C.c_int), C.c_int]),
    ("swift_plan_block_histogram", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P]),
    ("swift_gather_bound", C.c_int, [_P, C.c_int, _P, _I64, C.c_int, _P, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("swift_plan_set_symmetry", C.c_int, [_P, C.c_int]),
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
    ("swift_spmm_scaled", C.c_int, [_P, C.c_int, C.c_int, _P, _I64, _P, _P, _I64, _P, _P]),
    ("swift_plan_set_rowwise_params", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("swift_plan_get_rowwise_params", C.c_int, [_P, C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 4),
    ("swift_batch_create", C.c_int, [C.POINTER(_P), C.c_int, _P, C.POINTER(_P)]),
    ("swift_batch_destroy", C.c_int, [_P]),
    ("swift_batch_set_operands", C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    ("swift_batch_run", C.c_int, [_P, _P]),
    ("swift_batch_run_graph", C.c_int, [_P, _P]),
    ("swift_batch_autotune", C.c_int, [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("swift_batch_get_task_sizes", C.c_int, [_P, _P]),
    ("swift_batch_set_n_split", C.c_int, [_P, _P, _P]),
    ("swift_batch_get_n_split", C.c_int, [_P, _P]),
    ("swift_mtx_read", C.c_int, [C.c_char_p, C.c_int] + [C.POINTER(C.c_int)] * 4
     + [C.POINTER(C.POINTER(C.c_int))] * 2 + [C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
    ("swift_host_free", None, [_P]),
]
# reference-convention functions (host buffers), one per value type
_FP = C.POINTER(C.c_float)
for _sfx, _S in (("f32", swift_slide_matrix_f32), ("f64", swift_slide_matrix_f64)):
    _SP = C.POINTER(_S)
    _SIGS += [
        (f"swift_ref_csr_to_csc_{_sfx}", C.c_int, [_FP, C.c_int, C.c_int, C.c_int] + [_P] * 7),
        (f"swift_ref_col_sort_{_sfx}", C.c_int, [_FP, C.c_int, C.c_int, C.c_int] + [_P] * 9),
        (f"swift_ref_formattransation_{_sfx}", C.c_int,
         [_FP, _SP, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)]),
        (f"swift_ref_formatTransform_{_sfx}", C.c_int,
         [_FP, _SP, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
        (f"swift_ref_block_catgory_{_sfx}", C.c_int, [_SP, C.POINTER(C.c_double)]),
        (f"swift_ref_balance_{_sfx}", C.c_int, [_SP, C.c_int, C.c_int, C.c_int, _P, _P]),
        (f"swift_ref_row_idx_sort_{_sfx}", C.c_int, [_SP, C.c_int, C.c_int, C.c_int, _FP]),
        (f"swift_ref_spmm_{_sfx}", C.c_int, [C.c_int, _SP, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _FP]),
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
