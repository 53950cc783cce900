"""Test helper: the reference's preprocessing and SpMM functions under their own names (host
numpy buffers), so that the compatibility tests read like the reference's driver.

Each function calls the matching ``swift_ref_*`` entry point of libswiftb200.so, which runs the
stage on the GPU.  Names, argument meanings and the order of calls follow the reference driver
(src/main.cu:200-450):

    csc_val, csc_row, csc_ptr, nnzpercol, ms = csr_to_csc(m, n, nnz, val, rowptr, colidx)
    srow, sval, snnz, sdense, ms = col_sort(colA, width, nnzpercol, csc_ptr, csc_row, csc_val, B)
    mat, reside_ratio = formattransation(srow, sval, snnz, nnz, rowA, colA)
    shuffle_ratio = block_catgory(mat)
    C, ms = Swift_gpu1(mat, rowA, colA, width, nnz, sdense_colmajor)
    balance(mat, rowA, mat.reside_col, mat.reside_nnz, reside_ptr, reside_row)
    ...
    blockratio = row_idx_sort(mat, rowA, colA, width)
    C, ms = Swift_GPU_4(mat, rowA, colA, width, nnz, sdense_colmajor)

The driver's input comes from ``mmio_allinone(filename)`` (src/auxiliary.h:167-332), which
returns the reference's code with the CSR: ``rc, m, n, nnz, isSymmetric, rowptr, colidx, val``.

SpMM wrappers take the column-sorted dense operand and return C in the wrapper's own layout:
column-major (numpy Fortran order, M x N) for Swift_GPU / Swift_gpu1 / Swift_GPU_3 / Swift_GPU_4
and row-major for Swift_gpu2, as the reference wrappers do (src/main.cu:338-340).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from swift_b200 import _capi as capi

_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]
_libc.free.restype = None


def _sfx(vdt) -> str:
    vdt = np.dtype(vdt)
    if vdt == np.float32:
        return "f32"
    if vdt == np.float64:
        return "f64"
    raise TypeError(f"value type {vdt} (float32 or float64)")


def _fn(name, vdt):
    return getattr(capi.lib(), f"swift_ref_{name}_{_sfx(vdt)}")


def _ptr(a):
    return None if a is None else a.ctypes.data


class SlideMatrix:
    """A reference ``slide_matrix`` (src/format.h:6-39).  Arrays malloc'd by the library are
    freed on close(); arrays supplied from numpy (``from_arrays``) stay owned by numpy."""

    def __init__(self, vdt):
        self.vdt = np.dtype(vdt)
        S = capi.swift_slide_matrix_f64 if self.vdt == np.float64 else capi.swift_slide_matrix_f32
        self.s = S()
        self._keep = []

    @classmethod
    def from_arrays(cls, d: dict, vdt):
        m = cls(vdt)
        m.s, m._keep = capi.slide_from_arrays(d, vdt)
        return m

    def __getattr__(self, k):
        if k in capi._SLIDE_INTS:
            return int(getattr(self.s, k))
        raise AttributeError(k)

    def arrays(self) -> dict:
        return capi.slide_arrays(self.s, self.vdt, with_row_sort=True)

    def ref(self):
        return C.byref(self.s)

    def close(self):
        owned = {a.ctypes.data for a in self._keep}
        for name in capi._SLIDE_LEN:
            p = getattr(self.s, name)
            addr = C.cast(p, C.c_void_p).value
            if addr and addr not in owned:
                _libc.free(addr)
            setattr(self.s, name, type(p)())
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def csr_to_csc(m, n, nnz, csr_val, csr_row_ptr, csr_col_ind):
    """src/gpu_csr2csc.h:51 -> (csc_val, csc_row_ind, csc_col_ptr, nnzpercol, ms)."""
    vdt = np.asarray(csr_val).dtype
    rp = np.ascontiguousarray(csr_row_ptr, np.int32)
    ci = np.ascontiguousarray(csr_col_ind, np.int32)
    v = np.ascontiguousarray(csr_val, vdt)
    cv = np.zeros(max(nnz, 1), vdt)
    cr = np.zeros(max(nnz, 1), np.int32)
    cp = np.zeros(n + 1, np.int32)
    cnt = np.zeros(max(n, 1), np.int32)
    ms = C.c_float(0)
    capi.check(_fn("csr_to_csc", vdt)(C.byref(ms), m, n, nnz, _ptr(v), _ptr(rp), _ptr(ci), _ptr(cv),
                                      _ptr(cr), _ptr(cp), _ptr(cnt)), "csr_to_csc")
    return cv[:nnz], cr[:nnz], cp, cnt[:n], ms.value


def col_sort(colA, width, nnzpercol, csccolptr, cscrowidx, cscval, dense_mtx=None):
    """src/coo2csc.h:82 / src/ColSort_cuda.h:48 -> (sortrowidx, sortval, sortnnz, sort_dense, ms).
    dense_mtx is row-major colA x width; sort_dense[i] = dense_mtx[perm[i]]."""
    vdt = np.asarray(cscval).dtype
    cp = np.ascontiguousarray(csccolptr, np.int32)
    nnz = int(cp[colA]) if colA > 0 else 0
    cnt = np.ascontiguousarray(nnzpercol, np.int32)
    cr = np.ascontiguousarray(cscrowidx, np.int32)
    cv = np.ascontiguousarray(cscval, vdt)
    sr = np.zeros(max(nnz, 1), np.int32)
    sv = np.zeros(max(nnz, 1), vdt)
    sn = np.zeros(max(colA, 1), np.int32)
    B = sB = None
    if dense_mtx is not None:
        B = np.ascontiguousarray(dense_mtx, vdt)
        sB = np.zeros_like(B)
    ms = C.c_float(0)
    capi.check(_fn("col_sort", vdt)(C.byref(ms), colA, nnz, width, _ptr(cnt), _ptr(cp), _ptr(cr), _ptr(cv),
                                    _ptr(sr), _ptr(sv), _ptr(sn), _ptr(B), _ptr(sB)), "col_sort")
    return sr[:nnz], sv[:nnz], sn[:colA], sB, ms.value


def formattransation(sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA):
    """src/coo2csc.h:137 -> (SlideMatrix with tiles + reside part, reside_ratio)."""
    vdt = np.asarray(sortval_tmp).dtype
    sr = np.ascontiguousarray(sortrowidx_tmp, np.int32)
    sv = np.ascontiguousarray(sortval_tmp, vdt)
    sn = np.ascontiguousarray(sortnnz_tmp, np.int32)
    m = SlideMatrix(vdt)
    rr = C.c_double(0)
    capi.check(_fn("formattransation", vdt)(None, m.ref(), _ptr(sr), _ptr(sv), _ptr(sn), nnz, rowA, colA,
                                            C.byref(rr)), "formattransation")
    return m, rr.value


def formatTransform(sortrowidx_tmp, sortval_tmp, sortnnz_tmp, nnz, rowA, colA):
    """src/formatTransform_cuda.h:198 (regular tiles only) -> (SlideMatrix, h_count, ms)."""
    vdt = np.asarray(sortval_tmp).dtype
    sr = np.ascontiguousarray(sortrowidx_tmp, np.int32)
    sv = np.ascontiguousarray(sortval_tmp, vdt)
    sn = np.ascontiguousarray(sortnnz_tmp, np.int32)
    m = SlideMatrix(vdt)
    hc = C.c_int(0)
    ms = C.c_float(0)
    capi.check(_fn("formatTransform", vdt)(C.byref(ms), m.ref(), _ptr(sr), _ptr(sv), _ptr(sn), nnz, rowA,
                                           colA, C.byref(hc)), "formatTransform")
    return m, hc.value, ms.value


def block_catgory(m: SlideMatrix) -> float:
    """src/block_catgory.h:1 -> shuffle_ratio (share of single-row tiles)."""
    r = C.c_double(0)
    capi.check(_fn("block_catgory", m.vdt)(m.ref(), C.byref(r)), "block_catgory")
    return r.value


def balance(m: SlideMatrix, rows, n, nnz, cscptr, cscrowidx=None):
    """src/balance.h:1 over the reside part (n columns, pointer cscptr)."""
    cp = np.ascontiguousarray(cscptr, np.int32)
    cr = None if cscrowidx is None else np.ascontiguousarray(cscrowidx, np.int32)
    capi.check(_fn("balance", m.vdt)(m.ref(), rows, n, nnz, _ptr(cp), _ptr(cr)), "balance")


def row_idx_sort(m: SlideMatrix, rowA, colA, width) -> float:
    """src/back_process.h:23 -> blockratio; sortrowidx is overwritten with the sorted keys."""
    br = C.c_float(0)
    capi.check(_fn("row_idx_sort", m.vdt)(m.ref(), rowA, colA, width, C.byref(br)), "row_idx_sort")
    return br.value


def _spmm(variant, m: SlideMatrix, rowA, colA, width, nnz, sort_dense):
    vdt = m.vdt
    if variant == 2:
        B = np.ascontiguousarray(sort_dense, vdt)
        Cm = np.zeros((rowA, width), vdt)
    else:
        B = np.asfortranarray(sort_dense, vdt)
        Cm = np.zeros((rowA, width), vdt, order="F")
    ms = C.c_float(0)
    capi.check(_fn("spmm", vdt)(variant, m.ref(), rowA, colA, width, nnz, B.ctypes.data, Cm.ctypes.data,
                                C.byref(ms)), "swift_ref_spmm")
    return Cm, ms.value


def Swift_GPU(m, rowA, colA, width, nnz, sort_dense):
    """src/Swift.h:184 (column-major operands) -> (C, ms)."""
    return _spmm(0, m, rowA, colA, width, nnz, sort_dense)


def Swift_gpu1(m, rowA, colA, width, nnz, sort_dense):
    """src/Swift_gpu_col_major.h:171 (column-major, reside part without balance) -> (C, ms)."""
    return _spmm(1, m, rowA, colA, width, nnz, sort_dense)


def Swift_gpu2(m, rowA, colA, width, nnz, sort_dense):
    """src/Swift_gpu_row_major.h:136 (row-major operands) -> (C, ms)."""
    return _spmm(2, m, rowA, colA, width, nnz, sort_dense)


def Swift_GPU_3(m, rowA, colA, width, nnz, sort_dense):
    """src/Swift_3.h:216 (column-major operands) -> (C, ms)."""
    return _spmm(3, m, rowA, colA, width, nnz, sort_dense)


def Swift_GPU_4(m, rowA, colA, width, nnz, sort_dense):
    """src/Swift_4.h:305 (column-major; after row_idx_sort, slot rows via val_position) -> (C, ms)."""
    return _spmm(4, m, rowA, colA, width, nnz, sort_dense)


def mmio_allinone(filename, dtype=np.float64):
    """src/auxiliary.h:167-332 -> (rc, m, n, nnz, isSymmetric, csrrowptr, csrcolidx, csrval).

    rc is the reference's return code (0, -1 cannot open, -2 banner, -4 size line) or -5 where
    the reference would go on with undefined values; the arrays are None unless rc == 0."""
    from swift_b200.mtx import read_mtx, reference_code
    try:
        mm = read_mtx(filename, dtype)
    except capi.SwiftError:
        return reference_code(filename) or -5, 0, 0, 0, 0, None, None, None
    return 0, mm.rows, mm.cols, mm.nnz, int(mm.symmetric), mm.rowptr, mm.colidx, mm.val
