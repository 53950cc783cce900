"""ctypes view of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, and only as the checker.  The library itself never loads it.

Two implementations sit behind the same Python functions:

* ``impl="oracle"`` -- this project's C restatement (``oracle/liboracle.so``), which every
  function cites against the reference line by line;
* ``impl="ref"``    -- the reference's own host code compiled in place from its checkout
  (``oracle/_ref/libswiftref_{f32,f64}.so``, built by ``oracle/Makefile``), used to pin the
  restatement and as the reference CPU baseline.

``ref_gpu_spmm`` runs the reference's own GPU SpMM wrappers (``oracle/_ref/libswiftrefgpu_*.so``,
compiled in place for sm_100a) -- a context measurement and a cross-check, never the product.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}

_I = C.POINTER(C.c_int)
_U = C.POINTER(C.c_uint)


def _slide_struct(vt):
    P = C.POINTER(vt)
    fields = [
        ("tilenum", C.c_int), ("regular_nnz", C.c_int), ("nsteps", C.c_int),
        ("tile_ptr", _I), ("tile_len", _I), ("tile_colidx", _I), ("tile_tall", _I),
        ("sortrowidx", _I), ("sortval", P),
        ("reside_col", C.c_int), ("reside_nnz", C.c_int),
        ("reside_cscptr", _I), ("reside_cscrowidx", _I), ("reside_val", P),
        ("segsum", C.c_int),
        ("tile_format", _I), ("countrow", _I), ("segmentoffset", _I), ("sortrowindex", _I),
        ("numblk", C.c_int), ("colorblk", _U), ("blkstart", _I), ("blkstop", _I), ("blkptr", _I),
        ("val_position", _I), ("val_offset", _I),
    ]
    return type("or_slide", (C.Structure,), {"_fields_": fields})


_SLIDE = {np.float32: _slide_struct(C.c_float), np.float64: _slide_struct(C.c_double)}
_CT = {np.float32: C.c_float, np.float64: C.c_double}
_SFX = {np.float32: "_f32", np.float64: "_f64"}


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f"libswiftref{s}.so")) for s in ("_f32", "_f64"))


def _lib(impl: str, dt):
    key = (impl, dt if impl == "ref" else None)
    if key in _LIBS:
        return _LIBS[key]
    if impl == "oracle":
        path = os.path.join(HERE, "liboracle.so")
    elif impl == "ref":
        path = os.path.join(HERE, "_ref", f"libswiftref{_SFX[dt]}.so")
    else:
        raise ValueError(impl)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    _LIBS[key] = lib
    return lib


def _p(a, ct=C.c_int):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def _dt(x):
    return np.float64 if np.dtype(x) == np.float64 else np.float32


@dataclass
class Slide:
    """Host copy of every Swift format array (the reference's slide_matrix, src/format.h:6-39)."""
    dtype: type
    tilenum: int = 0
    regular_nnz: int = 0
    nsteps: int = 0
    reside_col: int = 0
    reside_nnz: int = 0
    segsum: int = 0
    numblk: int = 0
    arrays: dict = field(default_factory=dict)

    def __getitem__(self, k):
        return self.arrays[k]


def _arr(ptr, n, dt):
    if n <= 0 or not ptr:
        return np.zeros(0, dt)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)


def _read_slide(s, dt) -> Slide:
    out = Slide(dt, s.tilenum, s.regular_nnz, s.nsteps, s.reside_col, s.reside_nnz, s.segsum, s.numblk)
    T, R, RC, RN, NB = s.tilenum, s.regular_nnz, s.reside_col, s.reside_nnz, s.numblk
    a = out.arrays
    a["tile_ptr"] = _arr(s.tile_ptr, T + 1, np.int32)
    a["tile_len"] = _arr(s.tile_len, T, np.int32)
    a["tile_colidx"] = _arr(s.tile_colidx, T, np.int32)
    a["tile_tall"] = _arr(s.tile_tall, T, np.int32)
    a["sortrowidx"] = _arr(s.sortrowidx, R, np.int32)
    a["sortval"] = _arr(s.sortval, R, dt)
    a["reside_cscptr"] = _arr(s.reside_cscptr, RC + 1, np.int32)
    a["reside_cscrowidx"] = _arr(s.reside_cscrowidx, RN, np.int32)
    a["reside_val"] = _arr(s.reside_val, RN, dt)
    a["tile_format"] = _arr(s.tile_format, T, np.int32)
    if s.countrow:
        a["countrow"] = _arr(s.countrow, T + 1, np.int32)
    a["segmentoffset"] = _arr(s.segmentoffset, s.segsum + 1, np.int32)
    a["sortrowindex"] = _arr(s.sortrowindex, R, np.int32)
    a["colorblk"] = _arr(s.colorblk, NB, np.uint32)
    a["blkstart"] = _arr(s.blkstart, NB, np.int32)
    a["blkstop"] = _arr(s.blkstop, NB, np.int32)
    a["blkptr"] = _arr(s.blkptr, NB, np.int32)
    if s.val_position:
        a["val_position"] = _arr(s.val_position, R, np.int32)
        a["val_offset"] = _arr(s.val_offset, R, np.int32)
    return out


def csr2csc(M, K, rowptr, colidx, val, impl="oracle"):
    dt = _dt(val.dtype)
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    val = np.ascontiguousarray(val, dt)
    nnz = int(rowptr[-1])
    r = np.zeros(max(nnz, 1), np.int32)
    p = np.zeros(K + 1, np.int32)
    cnt = np.zeros(max(K, 1), np.int32)
    v = np.zeros(max(nnz, 1), dt)
    if impl == "ref":
        fn = getattr(_lib("ref", dt), "ref_csr2csc" + _SFX[dt])
    else:
        fn = getattr(_lib("oracle", dt), "or_csr2csc" + _SFX[dt])
    rc = fn(M, K, nnz, _p(rowptr), _p(colidx), _p(val, _CT[dt]), _p(r), _p(p), _p(cnt), _p(v, _CT[dt]))
    if impl == "oracle" and rc != 0:
        raise ValueError("malformed CSR")
    return r[:nnz], p, cnt[:K], v[:nnz]


def perm_stable(nnzpercol):
    cnt = np.ascontiguousarray(nnzpercol, np.int32)
    perm = np.zeros(max(cnt.size, 1), np.int32)
    _lib("oracle", None).or_col_perm_stable(cnt.size, _p(cnt), _p(perm))
    return perm[:cnt.size]


def perm_std_sort(nnzpercol, dt=np.float32):
    """The reference host col_sort's own (std::sort, unstable) column order."""
    cnt = np.ascontiguousarray(nnzpercol, np.int32)
    perm = np.zeros(max(cnt.size, 1), np.int32)
    getattr(_lib("ref", dt), "ref_std_sort_perm" + _SFX[dt])(cnt.size, _p(cnt), _p(perm))
    return perm[:cnt.size]


def col_sort(K, N, nnzpercol, perm, csccolptr, cscrowidx, cscval, B=None, impl="oracle", native=False):
    dt = _dt(cscval.dtype)
    nnz = int(csccolptr[-1])
    cnt = np.ascontiguousarray(nnzpercol, np.int32)
    perm = np.ascontiguousarray(perm, np.int32) if perm is not None else None
    cp = np.ascontiguousarray(csccolptr, np.int32)
    cr = np.ascontiguousarray(cscrowidx, np.int32)
    cv = np.ascontiguousarray(cscval, dt)
    sr = np.zeros(max(nnz, 1), np.int32)
    sv = np.zeros(max(nnz, 1), dt)
    sn = np.zeros(max(K, 1) + 1, np.int32)
    Bc = np.ascontiguousarray(B, dt) if B is not None else None
    sB = np.zeros_like(Bc) if Bc is not None else None
    if impl == "ref" and native:
        Bc2 = Bc if Bc is not None else np.zeros((K, max(N, 1)), dt)
        sB2 = sB if sB is not None else np.zeros_like(Bc2)
        getattr(_lib("ref", dt), "ref_col_sort_native" + _SFX[dt])(
            K, N, _p(cnt), _p(cp), _p(cr), _p(cv, _CT[dt]), _p(sr), _p(sv, _CT[dt]), _p(sn),
            _p(Bc2, _CT[dt]), _p(sB2, _CT[dt]))
        if sB is not None:
            sB = sB2
    else:
        name = ("ref_col_sort" if impl == "ref" else "or_col_sort") + _SFX[dt]
        getattr(_lib(impl, dt), name)(
            K, N, _p(cnt), _p(perm), _p(cp), _p(cr), _p(cv, _CT[dt]), _p(sr), _p(sv, _CT[dt]),
            _p(sn), _p(Bc, _CT[dt]), _p(sB, _CT[dt]))
    return sr[:nnz], sv[:nnz], sn[:K], sB


def build(sortrowidx_tmp, sortval_tmp, sortnnz_tmp, M, K, impl="oracle", row_sort=True, N=32):
    """formattransation + block_catgory + balance (+ row_idx_sort) -> Slide."""
    dt = _dt(sortval_tmp.dtype)
    S = _SLIDE[dt]
    s = S()
    sr = np.ascontiguousarray(sortrowidx_tmp, np.int32)
    sv = np.ascontiguousarray(sortval_tmp, dt)
    sn = np.ascontiguousarray(np.append(np.asarray(sortnnz_tmp, np.int32), 0), np.int32)
    nnz = int(sr.size)
    sr1 = sr if nnz else np.zeros(1, np.int32)
    sv1 = sv if nnz else np.zeros(1, dt)
    br = C.c_float(0)
    if impl == "ref":
        lib = _lib("ref", dt)
        getattr(lib, "ref_build" + _SFX[dt])(C.byref(s), _p(sr1), _p(sv1, _CT[dt]), _p(sn), nnz, M, K)
        out0 = _read_slide(s, dt)  # before the in-place row sort mutates sortrowidx
        if row_sort:
            getattr(lib, "ref_row_idx_sort" + _SFX[dt])(C.byref(s), M, K, N, C.byref(br))
    else:
        lib = _lib("oracle", dt)
        rc = getattr(lib, "or_formattransation" + _SFX[dt])(C.byref(s), _p(sr1), _p(sv1, _CT[dt]), _p(sn), nnz, M, K)
        if rc != 0:
            raise ValueError(f"formattransation failed ({rc})")
        getattr(lib, "or_block_catgory" + _SFX[dt])(C.byref(s))
        getattr(lib, "or_balance" + _SFX[dt])(C.byref(s))
        out0 = _read_slide(s, dt)
        if row_sort:
            getattr(lib, "or_row_idx_sort" + _SFX[dt])(C.byref(s), C.byref(br))
    if row_sort:
        after = _read_slide(s, dt)
        out0.arrays["rowsorted_rowidx"] = after.arrays["sortrowidx"]
        out0.arrays["val_position"] = after.arrays["val_position"]
        out0.arrays["val_offset"] = after.arrays["val_offset"]
        out0.arrays["blockratio"] = np.float32(br.value)
    # both implementations allocate with malloc; the oracle's free releases either
    getattr(_lib("oracle", None), "or_slide_free" + _SFX[dt])(C.byref(s))
    return out0


def swift_cpu(slide: Slide, M, K, N, sortB, impl="oracle"):
    """C = A*B over the format in the reference's exact accumulation order (Swift_cpu)."""
    dt = slide.dtype
    S = _SLIDE[dt]
    s = S()
    keep = []

    def put(name, arr, ct=C.c_int):
        a = np.ascontiguousarray(arr)
        if a.size == 0:
            a = np.zeros(1, a.dtype)
        keep.append(a)
        setattr(s, name, a.ctypes.data_as(C.POINTER(ct)))

    s.tilenum, s.regular_nnz = slide.tilenum, slide.regular_nnz
    s.reside_col, s.reside_nnz = slide.reside_col, slide.reside_nnz
    put("tile_ptr", slide["tile_ptr"])
    put("tile_len", slide["tile_len"])
    put("tile_colidx", slide["tile_colidx"])
    put("sortrowidx", slide["sortrowidx"])
    put("sortval", slide["sortval"].astype(dt), _CT[dt])
    put("reside_cscptr", slide["reside_cscptr"])
    put("reside_cscrowidx", slide["reside_cscrowidx"])
    put("reside_val", slide["reside_val"].astype(dt), _CT[dt])
    sB = np.ascontiguousarray(sortB, dt)
    Cm = np.zeros((M, N), dt)
    if impl == "ref":
        ms = getattr(_lib("ref", dt), "ref_swift_cpu" + _SFX[dt])
        ms.restype = C.c_double
        ms(C.byref(s), M, K, N, _p(sB, _CT[dt]), _p(Cm, _CT[dt]))
    else:
        getattr(_lib("oracle", None), "or_swift_cpu" + _SFX[dt])(C.byref(s), M, K, N, _p(sB, _CT[dt]), _p(Cm, _CT[dt]))
    return Cm


def pipeline(M, K, rowptr, colidx, val, B, impl="oracle", perm="stable", row_sort=True):
    """Full reference host pipeline on one CSR: csr2csc -> col_sort -> format -> Swift_cpu.

    Returns a dict with the CSC, the permutation, sorted arrays, the Slide and C."""
    dt = _dt(val.dtype)
    N = 0 if B is None else B.shape[1]
    r, p, cnt, v = csr2csc(M, K, rowptr, colidx, val, impl=impl)
    if isinstance(perm, str) and perm == "stable":
        pm = perm_stable(cnt)
    elif isinstance(perm, str) and perm == "std":
        pm = perm_std_sort(cnt, dt)
    else:
        pm = np.asarray(perm, np.int32)
    sr, sv, sn, sB = col_sort(K, max(N, 1), cnt, pm, p, r, v, B=B, impl=impl)
    sl = build(sr, sv, sn, M, K, impl=impl, row_sort=row_sort, N=max(N, 1))
    out = dict(cscrowidx=r, csccolptr=p, nnzpercol=cnt, cscval=v, perm=pm,
               sortrowidx_tmp=sr, sortval_tmp=sv, sortnnz_tmp=sn, sortB=sB, slide=sl)
    if B is not None:
        out["C"] = swift_cpu(sl, M, K, N, sB, impl=impl)
    return out


def csr_spmm_f64(M, K, rowptr, colidx, val, B):
    N = B.shape[1]
    Bc = np.ascontiguousarray(B, np.float64)
    out = np.zeros((M, N), np.float64)
    vv = np.ascontiguousarray(val, np.float64)
    _lib("oracle", None).or_csr_spmm_f64(M, K, N, _p(np.ascontiguousarray(rowptr, np.int32)),
                                         _p(np.ascontiguousarray(colidx, np.int32)),
                                         _p(vv, C.c_double), _p(Bc, C.c_double), _p(out, C.c_double))
    return out


def csr_spmm_t_f64(M, K, rowptr, colidx, val, dY):
    N = dY.shape[1]
    d = np.ascontiguousarray(dY, np.float64)
    out = np.zeros((K, N), np.float64)
    vv = np.ascontiguousarray(val, np.float64)
    _lib("oracle", None).or_csr_spmm_t_f64(M, K, N, _p(np.ascontiguousarray(rowptr, np.int32)),
                                           _p(np.ascontiguousarray(colidx, np.int32)),
                                           _p(vv, C.c_double), _p(d, C.c_double), _p(out, C.c_double))
    return out


def sddmm_f64(M, K, rowptr, colidx, U, V):
    N = U.shape[1]
    nnz = int(rowptr[-1])
    out = np.zeros(max(nnz, 1), np.float64)
    Uc = np.ascontiguousarray(U, np.float64)
    Vc = np.ascontiguousarray(V, np.float64)
    _lib("oracle", None).or_sddmm_f64(M, K, N, _p(np.ascontiguousarray(rowptr, np.int32)),
                                      _p(np.ascontiguousarray(colidx, np.int32)),
                                      _p(Uc, C.c_double), _p(Vc, C.c_double), _p(out, C.c_double))
    return out[:nnz]


class CpuSwift:
    """Swift_cpu held ready for repeated timed samples over tile ranges (CPU baseline).

    ``impl="ref"`` runs the reference's own Swift_cpu (compiled from its checkout) on a view
    of the format; ``impl="oracle"`` the restatement.  Both are single-threaded by
    construction, as the reference is."""

    def __init__(self, slide: Slide, M, K, N, sortB, impl="ref"):
        self.dt = slide.dtype
        self.impl = impl if (impl != "ref" or ref_available()) else "oracle"
        self.M, self.K, self.N = M, K, N
        self.tilenum = slide.tilenum
        S = _SLIDE[self.dt]
        self.s = S()
        self._keep = []

        def put(name, arr, ct=C.c_int):
            a = np.ascontiguousarray(arr)
            if a.size == 0:
                a = np.zeros(1, a.dtype)
            self._keep.append(a)
            setattr(self.s, name, a.ctypes.data_as(C.POINTER(ct)))

        self.s.tilenum, self.s.regular_nnz = slide.tilenum, slide.regular_nnz
        self.s.reside_col, self.s.reside_nnz = slide.reside_col, slide.reside_nnz
        put("tile_ptr", slide["tile_ptr"])
        put("tile_len", slide["tile_len"])
        put("tile_colidx", slide["tile_colidx"])
        put("sortrowidx", slide["sortrowidx"])
        put("sortval", slide["sortval"].astype(self.dt), _CT[self.dt])
        put("reside_cscptr", slide["reside_cscptr"])
        put("reside_cscrowidx", slide["reside_cscrowidx"])
        put("reside_val", slide["reside_val"].astype(self.dt), _CT[self.dt])
        self.sortB = np.ascontiguousarray(sortB, self.dt)
        self.C = np.zeros((M, N), self.dt)
        if self.impl == "ref":
            self.fn = getattr(_lib("ref", self.dt), "ref_swift_cpu_tiles" + _SFX[self.dt])
            self.fn.restype = C.c_double
        else:
            self.fn = getattr(_lib("oracle", None), "or_swift_cpu_tiles" + _SFX[self.dt])
            self.fn.restype = None

    def run(self, t0, t1, with_reside=False):
        """Adds the product of tiles [t0, t1) (and the reside part) into self.C; returns
        (seconds, nonzeros processed)."""
        import time
        a = time.perf_counter()
        self.fn(C.byref(self.s), int(t0), int(t1), int(with_reside), self.M, self.K, self.N,
                _p(self.sortB, _CT[self.dt]), _p(self.C, _CT[self.dt]))
        sec = time.perf_counter() - a
        nnz = (t1 - t0) * 32 + (int(self.s.reside_nnz) if with_reside else 0)
        return sec, nnz


# ---------------------------------------------------------------- reference GPU wrappers
REF_GPU_VARIANTS = {0: "Swift_GPU", 1: "Swift_gpu1", 2: "Swift_gpu2", 3: "Swift_GPU_3", 4: "Swift_GPU_4"}
REF_GPU_OK, REF_GPU_CHECK_FAILED, REF_GPU_REFUSED, REF_GPU_CUDA_ERROR = 0, 1, 2, 3


def ref_gpu_available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f"libswiftrefgpu{s}.so")) for s in ("_f32", "_f64"))


def ref_gpu_accepts(variant, arrays, N, dt) -> bool:
    """The inputs the reference-GPU entry point accepts (oracle/ref_gpu.cu states why)."""
    T, RN = int(arrays["tilenum"]), int(arrays["reside_nnz"])
    if N <= 0 or N % 32 or T <= 0 or RN <= 0:
        return False
    if variant == 4 and (np.dtype(dt) == np.float64 or T % 8 or "val_position" not in arrays):
        return False
    if variant != 1 and int(arrays.get("numblk", 0)) <= 0:
        return False
    return True


def ref_gpu_spmm(variant, arrays, M, K, N, nnz, B, golden):
    """One call of the reference's GPU wrapper ``REF_GPU_VARIANTS[variant]`` on the format
    ``arrays`` (a swift_b200 Plan.export() dict; variant 4 needs the row-sorted export).

    B: sorted dense operand K x N (any order; passed column-major except to Swift_gpu2, which
    takes it row-major); golden: row-major M x N.  Returns (status, ms, C as M x N), ms being
    the wrapper's own CUDA-event time of its kernels."""
    dt = _dt(B.dtype)
    key = ("refgpu", dt)
    if key not in _LIBS:
        _LIBS[key] = C.CDLL(os.path.join(HERE, "_ref", f"libswiftrefgpu{_SFX[dt]}.so"), mode=C.RTLD_LOCAL)
    lib = _LIBS[key]
    S = _SLIDE[dt]
    s = S()
    keep = []

    def put(name, arr, ct=C.c_int):
        a = np.ascontiguousarray(arr)
        if a.size == 0:
            a = np.zeros(1, a.dtype)
        keep.append(a)
        setattr(s, name, a.ctypes.data_as(C.POINTER(ct)))

    for k in ("tilenum", "regular_nnz", "reside_col", "reside_nnz", "segsum", "numblk"):
        setattr(s, k, int(arrays.get(k, 0)))
    for k in ("tile_ptr", "tile_len", "tile_colidx", "tile_tall", "sortrowidx", "reside_cscptr",
              "reside_cscrowidx", "tile_format", "countrow", "segmentoffset", "sortrowindex", "blkstart",
              "blkstop", "blkptr", "val_position", "val_offset"):
        if k in arrays:
            put(k, arrays[k].astype(np.int32))
    put("sortval", arrays["sortval"].astype(dt), _CT[dt])
    put("reside_val", arrays["reside_val"].astype(dt), _CT[dt])
    if "colorblk" in arrays:
        put("colorblk", arrays["colorblk"].astype(np.uint32), C.c_uint)
    Bm = np.ascontiguousarray(B, dt) if variant == 2 else np.asfortranarray(B, dt)
    Cm = np.zeros((M, N), dt, order="C" if variant == 2 else "F")
    gold = np.ascontiguousarray(golden, dt)
    ms = C.c_float(0)
    fn = getattr(lib, "refgpu_spmm" + _SFX[dt])
    st = fn(int(variant), C.byref(s), M, K, N, int(nnz), _p(Bm, _CT[dt]), _p(Cm, _CT[dt]), _p(gold, _CT[dt]),
            C.byref(ms))
    return int(st), float(ms.value), Cm


# ---------------------------------------------------------------- reference MatrixMarket reader
def ref_mmio(path):
    """The reference's own mmio_allinone (src/auxiliary.h:167-332, FP64 build) on a file.
    Returns (return code, rows, cols, is_symmetric, rowptr, colidx, val); the arrays are None
    unless the code is 0.  Only for well-formed files, a missing file or a bad banner (its
    size-line loop does not end on other malformed input)."""
    lib = _lib("ref", np.float64)
    m, n, nnz, sym = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
    rp, ci, vv = _I(), _I(), C.POINTER(C.c_double)()
    fn = lib.ref_mmio_allinone_f64
    fn.restype = C.c_int
    rc = fn(os.fsencode(path), C.byref(m), C.byref(n), C.byref(nnz), C.byref(sym), C.byref(rp), C.byref(ci),
            C.byref(vv))
    if rc != 0:
        return rc, 0, 0, 0, None, None, None
    out = (rc, m.value, n.value, sym.value, _arr(rp, m.value + 1, np.int32), _arr(ci, nnz.value, np.int32),
           _arr(vv, nnz.value, np.float64))
    for p in (rp, ci, vv):
        lib.ref_host_free(C.cast(p, C.c_void_p))
    return out
