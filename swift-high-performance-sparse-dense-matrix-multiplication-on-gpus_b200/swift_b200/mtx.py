"""MatrixMarket input (swift_mtx_read in include/swift_b200.h), the reference's on-disk format.

``read_mtx(path)`` returns the host CSR that the reference's reader builds from the file
(mmio_allinone, src/auxiliary.h:167-332): entries in file order inside each row, duplicates
kept, symmetric and hermitian files expanded to both triangles.  ``Plan.from_mtx`` builds a
plan from it directly.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _capi as capi


@dataclass
class MtxMatrix:
    rows: int
    cols: int
    rowptr: np.ndarray  # int32, rows + 1
    colidx: np.ndarray  # int32, nnz
    val: np.ndarray     # float32 or float64, nnz
    symmetric: bool     # the file said symmetric or hermitian (and was expanded)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    @property
    def shape(self):
        return (self.rows, self.cols)


def _take(addr, n, dt):
    """A numpy copy of n elements at the malloc'd address, which is then freed."""
    if not addr:
        return np.zeros(max(n, 0), dt)
    ct = np.ctypeslib.as_ctypes_type(np.dtype(dt))
    out = (np.ctypeslib.as_array(C.cast(C.c_void_p(addr), C.POINTER(ct)), shape=(n,)).copy()
           if n > 0 else np.zeros(0, dt))
    capi.lib().swift_host_free(C.c_void_p(addr))
    return out


def read_mtx(path, dtype=np.float64) -> MtxMatrix:
    """The CSR of a MatrixMarket coordinate file; raises capi.SwiftError (status ERR_IO,
    ERR_FORMAT or ERR_UNSUPPORTED) with the reason when the file cannot be read."""
    dt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    m, n, nnz, sym, ref_code = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
    rp, ci, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.c_void_p()
    st = capi.lib().swift_mtx_read(os.fsencode(path), capi.F64 if dt == np.float64 else capi.F32,
                                   C.byref(m), C.byref(n), C.byref(nnz), C.byref(sym), C.byref(rp),
                                   C.byref(ci), C.byref(vv), C.byref(ref_code))
    capi.check(st, f"swift_mtx_read({path})")
    rowptr = _take(C.cast(rp, C.c_void_p).value, m.value + 1, np.int32)
    colidx = _take(C.cast(ci, C.c_void_p).value, nnz.value, np.int32)
    val = _take(vv.value, nnz.value, dt)
    return MtxMatrix(m.value, n.value, rowptr, colidx, val, bool(sym.value))


def reference_code(path) -> int:
    """What the reference's reader returns for this file: 0, -1 (cannot open), -2 (banner),
    -4 (size line), -5 (an entry it would read undefined values from)."""
    m, n, nnz, sym, code = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
    rp, ci, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.c_void_p()
    st = capi.lib().swift_mtx_read(os.fsencode(path), capi.F64, C.byref(m), C.byref(n), C.byref(nnz),
                                   C.byref(sym), C.byref(rp), C.byref(ci), C.byref(vv), C.byref(code))
    if st == capi.OK:
        for p in (C.cast(rp, C.c_void_p), C.cast(ci, C.c_void_p), vv):
            capi.lib().swift_host_free(p)
    return code.value
