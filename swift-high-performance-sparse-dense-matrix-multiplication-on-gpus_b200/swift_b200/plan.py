"""Python view of a Swift plan (thin layer over the C ABI; device memory comes from torch).

    plan = Plan.from_csr(rowptr, colidx, val, (M, K))   # numpy (host) or CUDA tensors
    C = plan.spmm(B)                                     # C = A @ B on the current stream
    X = plan.spmm_t(Y)                                   # A^T @ Y
    dA = plan.sddmm(dY, X)                               # dY[row_e] . X[col_e] per nonzero
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as capi

_DT = {}


def _torch():
    import torch
    return torch


def _dtype_code(t):
    torch = _torch()
    m = {torch.float32: capi.F32, torch.float64: capi.F64, torch.bfloat16: capi.BF16, torch.float16: capi.F16}
    if t not in m:
        raise TypeError(f"unsupported dtype {t}")
    return m[t]


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dense(t, rows, cols, name, dtype=None):
    """Checks an operand before its pointer reaches a kernel: a 2-D CUDA tensor of rows x cols
    (and dtype); a wrong shape or a host tensor would otherwise be read or written out of bounds."""
    torch = _torch()
    if not isinstance(t, torch.Tensor) or t.dim() != 2:
        raise ValueError(f"{name} must be a 2-D tensor")
    if tuple(t.shape) != (rows, cols):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected ({rows}, {cols})")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    return t


def _vec(t, n, name, dtype):
    """As _dense for a contiguous 1-D CUDA tensor of n elements of dtype."""
    torch = _torch()
    if not isinstance(t, torch.Tensor) or t.numel() != n or not t.is_contiguous() or t.dtype != dtype:
        raise ValueError(f"{name} must be a contiguous {dtype} tensor of {n} elements")
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    return t


def _ld(t, layout):
    if t.dim() != 2:
        raise ValueError("dense operands are 2-D")
    if layout == capi.ROW_MAJOR:
        if t.stride(1) != 1:
            raise ValueError("row-major operand needs unit column stride")
        return t.stride(0)
    if t.stride(0) != 1:
        raise ValueError("column-major operand needs unit row stride")
    return t.stride(1)


class Plan:
    """A Swift format resident on the current CUDA device."""

    def __init__(self, handle, M, K, nnz, val_dtype, keep):
        self._h = handle
        self.M, self.K, self.nnz = M, K, nnz
        self.val_dtype = val_dtype  # numpy dtype of A's values
        self._keep = keep

    # ------------------------------------------------------------------ construction
    @classmethod
    def from_mtx(cls, path, dtype=np.float32, **kw):
        """A plan over the matrix of a MatrixMarket coordinate file (swift_b200.mtx.read_mtx,
        the reference reader's CSR); keyword arguments as for from_csr."""
        from .mtx import read_mtx
        m = read_mtx(path, dtype)
        return cls.from_csr(m.rowptr, m.colidx, m.val, m.shape, **kw)

    @classmethod
    def from_csr(cls, rowptr, colidx, val, shape, col_perm=None, long_row_split=0,
                 build_transpose=False, stream=None):
        torch = _torch()
        M, K = int(shape[0]), int(shape[1])
        keep = []
        on_dev = isinstance(rowptr, torch.Tensor) and rowptr.is_cuda
        if on_dev:
            rp = rowptr.to(torch.int32).contiguous()
            ci = colidx.to(torch.int32).contiguous()
            vv = val.contiguous()
            if vv.dtype not in (torch.float32, torch.float64):
                raise TypeError("A values must be float32 or float64")
            keep += [rp, ci, vv]
            ptrs = (rp.data_ptr(), ci.data_ptr(), vv.data_ptr())
            vt = capi.F64 if vv.dtype == torch.float64 else capi.F32
            nnz = int(ci.numel())
            mem = capi.DEVICE
            vdt = np.float64 if vt == capi.F64 else np.float32
        else:
            rp = np.ascontiguousarray(rowptr, np.int32)
            ci = np.ascontiguousarray(colidx, np.int32)
            vdt = np.float64 if np.asarray(val).dtype == np.float64 else np.float32
            vv = np.ascontiguousarray(val, vdt)
            keep += [rp, ci, vv]
            ptrs = (rp.ctypes.data, ci.ctypes.data if ci.size else rp.ctypes.data,
                    vv.ctypes.data if vv.size else rp.ctypes.data)
            vt = capi.F64 if vdt == np.float64 else capi.F32
            nnz = int(ci.size)
            mem = capi.HOST
        a = capi.swift_csr(M, K, nnz, ptrs[0], ptrs[1], ptrs[2], vt, mem)
        o = capi.swift_plan_opts()
        o.long_row_split = int(long_row_split)
        o.build_transpose = int(bool(build_transpose))
        if col_perm is not None:
            if isinstance(col_perm, torch.Tensor) and col_perm.is_cuda:
                cp = col_perm.to(torch.int32).contiguous()
                o.col_perm, o.col_perm_mem = cp.data_ptr(), capi.DEVICE
            else:
                cp = np.ascontiguousarray(col_perm, np.int32)
                o.col_perm, o.col_perm_mem = cp.ctypes.data, capi.HOST
            keep.append(cp)
        h = C.c_void_p()
        capi.check(capi.lib().swift_plan_create(C.byref(a), C.byref(o), _stream_ptr(stream), C.byref(h)),
                   "swift_plan_create")
        return cls(h, M, K, nnz, vdt, [] if not on_dev else keep)

    def close(self):
        if self._h is not None and self._h.value:
            capi.lib().swift_plan_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------------ introspection
    def stats(self) -> dict:
        s = capi.swift_plan_stats()
        capi.check(capi.lib().swift_plan_get_stats(self._h, C.byref(s)), "swift_plan_get_stats")
        d = {k: getattr(s, k) for k, _ in s._fields_}
        d["fmt_count"] = list(s.fmt_count)
        return d

    def is_symmetric(self, stream=None) -> bool:
        """A == A^T with equal values (checked once on the GPU, then cached)."""
        s = C.c_int(0)
        capi.check(capi.lib().swift_plan_is_symmetric(self._h, C.byref(s), _stream_ptr(stream)),
                   "swift_plan_is_symmetric")
        return s.value == 1

    def set_symmetry(self, use: bool):
        """Whether fused_forward_backward may compute dX = A dY in its first pass when A is
        symmetric (default True)."""
        capi.check(capi.lib().swift_plan_set_symmetry(self._h, int(bool(use))), "swift_plan_set_symmetry")

    def set_values(self, val, stream=None):
        """New values for the fixed pattern (CSR order; numpy or a CUDA tensor of the plan's
        value type)."""
        torch = _torch()
        if isinstance(val, torch.Tensor) and val.is_cuda:
            want = torch.float64 if self.val_dtype == np.float64 else torch.float32
            v = val.detach()
            if v.dtype != want or not v.is_contiguous():
                v = v.to(want).contiguous()
            if v.numel() != self.nnz:
                raise ValueError(f"{v.numel()} values for {self.nnz} nonzeros")
            capi.check(capi.lib().swift_plan_set_values(self._h, v.data_ptr(), capi.DEVICE, _stream_ptr(stream)),
                       "swift_plan_set_values")
            self._vals_in_flight = v  # the copy is stream-ordered: keep the source alive
        else:
            v = np.ascontiguousarray(val, self.val_dtype)
            if v.size != self.nnz:
                raise ValueError(f"{v.size} values for {self.nnz} nonzeros")
            capi.check(capi.lib().swift_plan_set_values(self._h, v.ctypes.data if v.size else None, capi.HOST,
                                                        _stream_ptr(stream)), "swift_plan_set_values")

    def export(self, with_row_sort=False) -> dict:
        """Every reference slide_matrix array as numpy (host copies made on the GPU)."""
        f64 = self.val_dtype == np.float64
        S = capi.swift_slide_matrix_f64 if f64 else capi.swift_slide_matrix_f32
        s = S()
        br = C.c_float(0)
        fn = capi.lib().swift_plan_export_f64 if f64 else capi.lib().swift_plan_export_f32
        capi.check(fn(self._h, C.byref(s), int(with_row_sort), C.byref(br)), "swift_plan_export")
        out = capi.slide_arrays(s, np.float64 if f64 else np.float32, with_row_sort)
        if with_row_sort:
            out["blockratio"] = np.float32(br.value)
        (capi.lib().swift_slide_free_f64 if f64 else capi.lib().swift_slide_free_f32)(C.byref(s))
        return out

    def export_sorted(self):
        """(perm, sortnnz, sorted CSC row indices, sorted CSC values) as numpy."""
        perm = np.zeros(max(self.K, 1), np.int32)
        sn = np.zeros(max(self.K, 1), np.int32)
        sr = np.zeros(max(self.nnz, 1), np.int32)
        sv = np.zeros(max(self.nnz, 1), self.val_dtype)
        capi.check(capi.lib().swift_plan_export_sorted(self._h, perm.ctypes.data, sn.ctypes.data,
                                                        sr.ctypes.data, sv.ctypes.data),
                   "swift_plan_export_sorted")
        return perm[:self.K], sn[:self.K], sr[:self.nnz], sv[:self.nnz]

    # ------------------------------------------------------------------ products
    def spmm(self, B, C_out=None, engine="auto", b_presorted=False, layout="row", stream=None):
        """C = A @ B.  layout 'row' (row-major B/C) or 'col' (column-major, Fortran order);
        engine 'auto', 'rowwise', 'tiled', 'tiled_grouped' (row-major, FP32/FP64) or 'band'
        (dense diagonal tiles + row walk; FP32 plans, row-major, N >= 128)."""
        torch = _torch()
        lay = capi.ROW_MAJOR if layout == "row" else capi.COL_MAJOR
        N = int(B.shape[1])
        _dense(B, self.K, N, "B")
        if C_out is None:
            C_out = torch.empty((self.M, N), dtype=B.dtype, device=B.device)
            if lay == capi.COL_MAJOR:
                C_out = torch.empty((N, self.M), dtype=B.dtype, device=B.device).t()
        _dense(C_out, self.M, N, "C_out", B.dtype)
        eng = {"auto": capi.ENGINE_AUTO, "tiled": capi.ENGINE_TILED, "rowwise": capi.ENGINE_ROWWISE,
               "tiled_grouped": capi.ENGINE_TILED_GROUPED, "band": capi.ENGINE_BAND}[engine]
        capi.check(capi.lib().swift_spmm(self._h, eng, N, _dtype_code(B.dtype), B.data_ptr(), _ld(B, lay), lay,
                                         int(b_presorted), C_out.data_ptr(), _ld(C_out, lay), lay,
                                         _stream_ptr(stream)), "swift_spmm")
        return C_out

    def spmm_scaled(self, B, b_scale=None, C_out=None, c_scale=None, stream=None):
        """C, c_scale with A @ (b_scale[:, None] * B) == c_scale[:, None] * C: 16-bit (bf16 or
        f16) row-major B and C scaled per row (swift_spmm_scaled).  b_scale: K floats or None
        (all 1); c_scale is written with one power of two per row of C."""
        torch = _torch()
        N = int(B.shape[1])
        _dense(B, self.K, N, "B")
        if C_out is None:
            C_out = torch.empty((self.M, N), dtype=B.dtype, device=B.device)
        _dense(C_out, self.M, N, "C_out", B.dtype)
        if c_scale is None:
            c_scale = torch.empty(self.M, dtype=torch.float32, device=B.device)
        if b_scale is not None:
            _vec(b_scale, self.K, "b_scale", torch.float32)
        _vec(c_scale, self.M, "c_scale", torch.float32)
        capi.check(capi.lib().swift_spmm_scaled(self._h, N, _dtype_code(B.dtype), B.data_ptr(), _ld(B, 0),
                                                b_scale.data_ptr() if b_scale is not None else None,
                                                C_out.data_ptr(), _ld(C_out, 0), c_scale.data_ptr(),
                                                _stream_ptr(stream)), "swift_spmm_scaled")
        return C_out, c_scale

    def spmm_t(self, Y, X_out=None, stream=None):
        """X = A^T @ Y (row-major)."""
        torch = _torch()
        N = int(Y.shape[1])
        _dense(Y, self.M, N, "Y")
        if X_out is None:
            X_out = torch.empty((self.K, N), dtype=Y.dtype, device=Y.device)
        _dense(X_out, self.K, N, "X_out", Y.dtype)
        capi.check(capi.lib().swift_spmm_transposed(self._h, N, _dtype_code(Y.dtype), Y.data_ptr(),
                                                    _ld(Y, 0), X_out.data_ptr(), _ld(X_out, 0),
                                                    _stream_ptr(stream)), "swift_spmm_transposed")
        return X_out

    def sddmm(self, U, V, out=None, stream=None):
        """out[e] = U[row_e] . V[col_e] for every nonzero e in CSR order."""
        torch = _torch()
        N = int(U.shape[1])
        _dense(U, self.M, N, "U")
        _dense(V, self.K, N, "V", U.dtype)
        vt = torch.float64 if self.val_dtype == np.float64 else torch.float32
        if out is None:
            out = torch.empty(self.nnz, dtype=vt, device=U.device)
        _vec(out, self.nnz, "out", vt)
        capi.check(capi.lib().swift_sddmm(self._h, N, _dtype_code(U.dtype), U.data_ptr(), _ld(U, 0),
                                          V.data_ptr(), _ld(V, 0), out.data_ptr(), _stream_ptr(stream)),
                   "swift_sddmm")
        return out

    def fused_forward_backward(self, X, dY, Y=None, dX=None, dA=None, want=("Y", "dX", "dA"), stream=None):
        torch = _torch()
        N = int(X.shape[1])
        if "Y" in want and Y is None:
            Y = torch.empty((self.M, N), dtype=X.dtype, device=X.device)
        if "dX" in want and dX is None:
            dX = torch.empty((self.K, N), dtype=X.dtype, device=X.device)
        if "dA" in want and dA is None:
            dA = torch.empty(self.nnz, dtype=X.dtype, device=X.device)
        _dense(X, self.K, N, "X")
        _dense(dY, self.M, N, "dY", X.dtype)
        if Y is not None:
            _dense(Y, self.M, N, "Y", X.dtype)
        if dX is not None:
            _dense(dX, self.K, N, "dX", X.dtype)
        if dA is not None:
            _vec(dA, self.nnz, "dA", X.dtype)

        def p(t):
            return t.data_ptr() if t is not None else None

        def ld(t):
            return _ld(t, 0) if t is not None else 0
        capi.check(capi.lib().swift_fused_forward_backward(
            self._h, N, _dtype_code(X.dtype), X.data_ptr(), ld(X), dY.data_ptr(), ld(dY), p(Y), ld(Y),
            p(dX), ld(dX), p(dA), _stream_ptr(stream)), "swift_fused_forward_backward")
        return Y, dX, dA

    def spmm_f64_reference(self, B64, stream=None):
        torch = _torch()
        N = int(B64.shape[1])
        _dense(B64, self.K, N, "B64", torch.float64)
        out = torch.empty((self.M, N), dtype=torch.float64, device=B64.device)
        capi.check(capi.lib().swift_spmm_f64_reference(self._h, N, B64.data_ptr(), _ld(B64, 0),
                                                       out.data_ptr(), _ld(out, 0), _stream_ptr(stream)),
                   "swift_spmm_f64_reference")
        return out

    def set_rowwise_params(self, task_size=0, loads_in_flight=0, vector_bytes=0, kernel=0):
        """Overrides the row engine's task size, loads in flight per lane, vector width and
        kernel variant (0 choose, 1 lean, 2 flagged indices, 3 general); task_size=0 returns to
        the tuned / default parameters."""
        capi.check(capi.lib().swift_plan_set_rowwise_params(self._h, int(task_size), int(loads_in_flight),
                                                            int(vector_bytes), int(kernel)),
                   "swift_plan_set_rowwise_params")

    def rowwise_params(self, N, dtype):
        v = [C.c_int(0) for _ in range(4)]
        capi.check(capi.lib().swift_plan_get_rowwise_params(self._h, int(N), _dtype_code(dtype),
                                                            *[C.byref(x) for x in v]),
                   "swift_plan_get_rowwise_params")
        return dict(zip(("task_size", "loads_in_flight", "vector_bytes", "kernel"), (x.value for x in v)))

    def autotune(self, B, C_out, stream=None):
        ms = C.c_double(0)
        eng = C.c_int(0)
        N = int(B.shape[1])
        _dense(B, self.K, N, "B")
        _dense(C_out, self.M, N, "C_out", B.dtype)
        capi.check(capi.lib().swift_plan_autotune(self._h, N, _dtype_code(B.dtype), B.data_ptr(),
                                                  C_out.data_ptr(), _stream_ptr(stream), C.byref(ms),
                                                  C.byref(eng)), "swift_plan_autotune")
        return {capi.ENGINE_TILED: "tiled", capi.ENGINE_ROWWISE: "rowwise",
                capi.ENGINE_TILED_GROUPED: "tiled_grouped", capi.ENGINE_BAND: "band"}[eng.value], ms.value

    def gather_bound(self, B, reps=10, stream=None):
        """(ms_stream, ms_l1, checksum): the time per launch of a kernel that only gathers B rows
        along A's column stream, the same with every row L1-resident, and the sum of the gathered
        elements (swift_gather_bound; FP32 row-major B, N in 32/64/128)."""
        N = int(B.shape[1])
        _dense(B, self.K, N, "B")
        a, b, c = C.c_double(0), C.c_double(0), C.c_double(0)
        capi.check(capi.lib().swift_gather_bound(self._h, N, B.data_ptr(), _ld(B, 0), reps, _stream_ptr(stream),
                                                 C.byref(a), C.byref(b), C.byref(c)), "swift_gather_bound")
        return a.value, b.value, c.value

    def block_histogram(self, bh, bw, sorted_columns=False, nbins=8, stream=None):
        """(blocks, nnz): occupied bh x bw blocks of A binned by fill f, bin k = (2^-(k+1), 2^-k]
        (the last bin: sparser), and their nonzeros (swift_plan_block_histogram)."""
        blocks = np.zeros(nbins, np.int64)
        nnz = np.zeros(nbins, np.int64)
        capi.check(capi.lib().swift_plan_block_histogram(self._h, bh, bw, int(bool(sorted_columns)), nbins,
                                                         blocks.ctypes.data, nnz.ctypes.data, _stream_ptr(stream)),
                   "swift_plan_block_histogram")
        return blocks, nnz

    def band_profile(self, stream=None):
        """(hist, half_width): nonzeros per |col - row| for 0..128 (measured on the GPU) and the
        band engine's half-width (-1 when no width pays)."""
        h = np.zeros(capi.BAND_PROFILE_MAX + 1, np.int64)
        w = C.c_int(0)
        capi.check(capi.lib().swift_plan_band_profile(self._h, h.ctypes.data, C.byref(w), _stream_ptr(stream)),
                   "swift_plan_band_profile")
        return h, w.value


class Batch:
    """Independent products C_i = A_i @ B_i (FP32, row-major) in one persistent launch.

        batch = Batch(plans)
        batch.set_operands(Bs, Cs)     # CUDA tensors, one pair per plan
        batch.run()                    # or batch.run_graph() (captured once, then replayed)
    The plans must stay alive while the batch exists."""

    def __init__(self, plans, stream=None):
        self.plans = list(plans)
        arr = (C.c_void_p * max(len(self.plans), 1))(*[p._h.value for p in self.plans])
        h = C.c_void_p()
        capi.check(capi.lib().swift_batch_create(arr, len(self.plans), _stream_ptr(stream), C.byref(h)),
                   "swift_batch_create")
        self._h = h
        self._keep = None

    def set_operands(self, Bs, Cs, stream=None):
        n = len(self.plans)
        if len(Bs) != n or len(Cs) != n:
            raise ValueError("one B and one C per plan")
        torch = _torch()
        for i, (p, b, c) in enumerate(zip(self.plans, Bs, Cs)):
            _dense(b, p.K, int(b.shape[1]) if b.dim() == 2 else -1, f"Bs[{i}]", torch.float32)
            _dense(c, p.M, int(b.shape[1]), f"Cs[{i}]", torch.float32)
        Ns = (C.c_int * max(n, 1))(*[int(b.shape[1]) for b in Bs])
        Bp = (C.c_void_p * max(n, 1))(*[b.data_ptr() for b in Bs])
        Cp = (C.c_void_p * max(n, 1))(*[c.data_ptr() for c in Cs])
        ldb = (C.c_int64 * max(n, 1))(*[_ld(b, capi.ROW_MAJOR) for b in Bs])
        ldc = (C.c_int64 * max(n, 1))(*[_ld(c, capi.ROW_MAJOR) for c in Cs])
        capi.check(capi.lib().swift_batch_set_operands(self._h, Ns, Bp, ldb, Cp, ldc, _stream_ptr(stream)),
                   "swift_batch_set_operands")
        self._keep = (list(Bs), list(Cs))

    def run(self, stream=None):
        capi.check(capi.lib().swift_batch_run(self._h, _stream_ptr(stream)), "swift_batch_run")

    def run_graph(self, stream=None):
        capi.check(capi.lib().swift_batch_run_graph(self._h, _stream_ptr(stream)), "swift_batch_run_graph")

    def autotune(self, stream=None):
        """Chooses the task size and the N-split per member class (N <= 32, N <= 64, wider);
        returns (the widest class's task size, ms per run)."""
        ms, U = C.c_double(0), C.c_int(0)
        capi.check(capi.lib().swift_batch_autotune(self._h, _stream_ptr(stream), C.byref(ms), C.byref(U)),
                   "swift_batch_autotune")
        return U.value, ms.value

    def task_sizes(self):
        """The task sizes in use for the member classes N <= 32, N <= 64 and wider."""
        out = (C.c_int * 3)()
        capi.check(capi.lib().swift_batch_get_task_sizes(self._h, out), "swift_batch_get_task_sizes")
        return list(out)

    def n_split(self):
        """The N-split (1 or 2 column halves) in use for the member classes N <= 32, N <= 64 and
        wider."""
        out = (C.c_int * 3)()
        capi.check(capi.lib().swift_batch_get_n_split(self._h, out), "swift_batch_get_n_split")
        return list(out)

    def set_n_split(self, splits, stream=None):
        """Walk the members of each class in 1 or 2 column halves (members whose N is a multiple
        of 8); rebuilds the launch table when operands are set."""
        arr = (C.c_int * 3)(*[int(x) for x in splits])
        capi.check(capi.lib().swift_batch_set_n_split(self._h, arr, _stream_ptr(stream)), "swift_batch_set_n_split")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.lib().swift_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
