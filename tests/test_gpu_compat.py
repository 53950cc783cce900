"""GPU parity of the reference-convention entry points (swift_ref_* in include/swift_b200.h,
called through swift_b200.compat, which keeps the reference's function names).

The reference driver's chain (src/main.cu:200-450) runs stage by stage on host buffers:
csr_to_csc -> col_sort -> formattransation -> block_catgory -> Swift_gpu1 -> balance ->
Swift_gpu2 -> Swift_GPU -> Swift_GPU_3 -> row_idx_sort -> Swift_GPU_4.  Every array is
compared bit-for-bit with the reference's own outputs (committed fixtures) or the oracle; every
C with the reference's Swift_cpu result (1e-5 FP32, 1e-12 FP64, normwise).
"""
import numpy as np
import pytest

import golden_io
import oracle
import ref_names as compat
from swift_b200 import capi

pytestmark = pytest.mark.gpu

TOL = {np.float32: 1e-5, np.float64: 1e-12}
TILE_KEYS = ["tile_ptr", "tile_len", "tile_colidx", "tile_tall", "sortrowidx", "sortval",
             "reside_cscptr", "reside_cscrowidx", "reside_val"]


def relerr(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    if ref.size == 0:
        return 0.0
    return float(np.abs(x - ref).max() / max(np.abs(ref).max(), 1e-300))


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b).astype(np.asarray(a).dtype))


def check_row_sort(ex, g):
    assert same(ex["val_offset"], g["val_offset"])
    assert same(ex["sortrowidx"], g["rowsorted_rowidx"])
    nr = ex["regular_nnz"]
    for g0 in range(0, nr, 256):  # val_position: ties of equal rows are unspecified
        g1 = min(g0 + 256, nr)
        p = ex["val_position"][g0:g1]
        assert np.array_equal(np.sort(p), np.arange(g1 - g0))
        assert np.array_equal(g["rowsorted_rowidx"][g0:g1][p], g["sortrowidx"][g0:g1])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", golden_io.ALL)
def test_reference_driver_chain(name, dt):
    g = golden_io.load(name, dt)
    M, K = g["M"], g["K"]
    nnz = int(g["rowptr"][-1])
    B = g["B"].astype(dt)
    N = B.shape[1]
    val = g["val"].astype(dt)

    cv, cr, cp, cnt, _ = compat.csr_to_csc(M, K, nnz, val, g["rowptr"], g["colidx"])
    assert same(cp, g["csccolptr"]) and same(cr, g["cscrowidx"]) and same(cnt, g["nnzpercol"])
    o_r, o_p, o_cnt, o_v = oracle.csr2csc(M, K, g["rowptr"], g["colidx"], val)
    assert same(cv, o_v)

    sr, sv, sn, sB, _ = compat.col_sort(K, N, cnt, cp, cr, cv, B)
    assert same(sn, g["sortnnz"])
    e_r, e_v, e_n, e_B = oracle.col_sort(K, N, cnt, oracle.perm_stable(cnt), cp, cr, cv, B)
    assert same(sr, e_r) and same(sv, e_v) and same(sn, e_n) and same(sB, e_B)
    assert same(sB, B[g["perm"]])

    mat, reside_ratio = compat.formattransation(sr, sv, sn, nnz, M, K)
    ex = mat.arrays()
    for k in ("tilenum", "regular_nnz", "reside_col", "reside_nnz"):
        assert ex[k] == g[k], k
    for k in TILE_KEYS:
        assert same(ex[k], g[k]), k
    assert reside_ratio == (g["reside_nnz"] / nnz if nnz else 0.0)

    shuffle = compat.block_catgory(mat)
    ex = mat.arrays()
    for k in ("tile_format", "segmentoffset", "sortrowindex"):
        assert same(ex[k], g[k]), k
    assert ex["segsum"] == g["segsum"]
    if g["tilenum"]:
        assert shuffle == np.count_nonzero(g["tile_format"] == 0) / g["tilenum"]

    Bf = np.asfortranarray(sB)
    C1, ms = compat.Swift_gpu1(mat, M, K, N, nnz, Bf)
    assert ms >= 0 and relerr(C1, g["C"]) <= TOL[dt]

    compat.balance(mat, M, ex["reside_col"], ex["reside_nnz"], ex["reside_cscptr"], ex["reside_cscrowidx"])
    ex = mat.arrays()
    assert ex["numblk"] == g["numblk"]
    for k in ("colorblk", "blkstart", "blkstop", "blkptr"):
        assert same(ex[k], g[k]), k

    C2, _ = compat.Swift_gpu2(mat, M, K, N, nnz, sB)
    assert C2.flags.c_contiguous and relerr(C2, g["C"]) <= TOL[dt]
    for fn in (compat.Swift_GPU, compat.Swift_GPU_3):
        Cx, _ = fn(mat, M, K, N, nnz, Bf)
        assert Cx.flags.f_contiguous and relerr(Cx, g["C"]) <= TOL[dt], fn.__name__

    blockratio = compat.row_idx_sort(mat, M, K, N)
    ex = mat.arrays()
    check_row_sort(ex, g)
    assert np.array_equal(np.float32(blockratio), np.float32(g["blockratio"]), equal_nan=True)
    C4, _ = compat.Swift_GPU_4(mat, M, K, N, nnz, Bf)
    assert relerr(C4, g["C"]) <= TOL[dt]
    mat.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["poisson4096", "long_col", "k_mod_31", "tiny_k", "empty"])
def test_format_transform_regular_part(name, dt):
    g = golden_io.load(name, dt)
    M, K = g["M"], g["K"]
    nnz = int(g["rowptr"][-1])
    cnt = g["nnzpercol"]
    cv = oracle.csr2csc(M, K, g["rowptr"], g["colidx"], g["val"].astype(dt))[3]
    sr, sv, sn, _ = oracle.col_sort(K, 1, cnt, g["perm"], g["csccolptr"], g["cscrowidx"], cv)
    mat, h_count, ms = compat.formatTransform(sr, sv, sn, nnz, M, K)
    ex = mat.arrays()
    assert h_count == g["nsteps"] and ms >= 0
    assert ex["tilenum"] == g["tilenum"] and ex["regular_nnz"] == g["regular_nnz"]
    for k in ("tile_ptr", "tile_len", "tile_colidx", "sortrowidx", "sortval"):
        assert same(ex[k], g[k]), k
    assert ex["reside_col"] == 0 and "reside_cscptr" not in ex
    mat.close()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["poisson4096", "long_col", "same_rows", "k32_exact"])
def test_wrappers_on_reference_format_arrays(name, dt):
    """The SpMM wrappers fed the reference's own format arrays (from the fixture, not built
    here), as a program that keeps the reference's preprocessing would call them."""
    g = golden_io.load(name, dt)
    M, K = g["M"], g["K"]
    nnz = int(g["rowptr"][-1])
    B = g["B"].astype(dt)[g["perm"]]
    N = B.shape[1]
    keys = TILE_KEYS + ["tile_format", "sortrowindex", "colorblk", "blkstart", "blkstop", "blkptr"]
    d = {k: g[k] for k in keys}
    d.update({k: g[k] for k in ("tilenum", "regular_nnz", "reside_col", "reside_nnz", "numblk")})
    mat = compat.SlideMatrix.from_arrays(d, dt)
    for v, fn in enumerate((compat.Swift_GPU, compat.Swift_gpu1, compat.Swift_gpu2, compat.Swift_GPU_3)):
        Cx, _ = fn(mat, M, K, N, nnz, B if v == 2 else np.asfortranarray(B))
        assert relerr(Cx, g["C"]) <= TOL[dt], fn.__name__
    d4 = dict(d, sortrowidx=g["rowsorted_rowidx"], val_position=g["val_position"], val_offset=g["val_offset"])
    mat4 = compat.SlideMatrix.from_arrays(d4, dt)
    C4, _ = compat.Swift_GPU_4(mat4, M, K, N, nnz, np.asfortranarray(B))
    assert relerr(C4, g["C"]) <= TOL[dt]
    mat.close()
    mat4.close()


def test_inconsistent_slide_matrix_rejected_on_host():
    g = golden_io.load("poisson4096", np.float32)
    M, K = g["M"], g["K"]
    nnz = int(g["rowptr"][-1])
    B = np.asfortranarray(g["B"][g["perm"]])
    base = {k: g[k] for k in TILE_KEYS + ["colorblk", "blkstart", "blkstop"]}
    base.update({k: g[k] for k in ("tilenum", "regular_nnz", "reside_col", "reside_nnz", "numblk")})
    bad_cases = [
        dict(tile_colidx=np.where(np.arange(g["tilenum"]) == 3, K - 31, g["tile_colidx"])),
        dict(sortrowidx=np.where(np.arange(g["regular_nnz"]) == 5, M, g["sortrowidx"])),
        dict(reside_cscptr=g["reside_cscptr"][::-1].copy()) if g["reside_col"] > 1 else dict(reside_col=33),
    ]
    for upd in bad_cases:
        mat = compat.SlideMatrix.from_arrays(dict(base, **upd), np.float32)
        with pytest.raises(capi.SwiftError) as e:
            compat.Swift_GPU(mat, M, K, B.shape[1], nnz, B)
        assert e.value.status == capi.ERR_INVALID_ARG
        mat.close()
