"""MatrixMarket input (swift_mtx_read, swift_b200.mtx, compat.mmio_allinone and the
mmio_allinone shim of include/swift_compat.h).

CPU: every well-formed file gives the same CSR, bit for bit, as the reference's own reader
(mmio_allinone, src/auxiliary.h:167-332, compiled from its sources under oracle/_ref): row
pointers, column order inside rows (file order, mirrored entries where they are met), values,
shape and the symmetric flag; FP32 values are the FP64 ones rounded.  The sums agree with
scipy.io.mmread as an independent reader.  Files the reference rejects give its return codes;
files where it would go on with undefined values are errors here.
GPU: a plan built from a file multiplies like the oracle's CSR product.
"""
import os

import numpy as np
import pytest

import oracle
from swift_b200 import capi
import ref_names as compat
from swift_b200.mtx import read_mtx, reference_code

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return str(p)


def mtx_text(M, N, entries, field="real", sym="general", banner=None, comments=("% made by a test",),
             eol="\n", fmt="{:.17g}"):
    lines = [banner or f"%%MatrixMarket matrix coordinate {field} {sym}"]
    lines += list(comments)
    lines.append(f"{M} {N} {len(entries)}")
    for e in entries:
        i, j = e[0], e[1]
        if field == "pattern":
            lines.append(f"{i} {j}")
        elif field == "integer":
            lines.append(f"{i} {j} {int(e[2])}")
        elif field == "complex":
            lines.append(f"{i} {j} {fmt.format(e[2])} {fmt.format(e[3])}")
        else:
            lines.append(f"{i} {j} {fmt.format(e[2])}")
    return eol.join(lines) + eol


def random_entries(M, N, n, seed, lower=False, field="real"):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        i, j = int(rng.integers(1, M + 1)), int(rng.integers(1, N + 1))
        if lower and j > i:
            i, j = j, i
        out.append((i, j, float(rng.uniform(-10, 10)), float(rng.uniform(-1, 1))) if field == "complex"
                   else (i, j, float(rng.integers(-50, 50)) if field == "integer" else float(rng.uniform(-10, 10))))
    return out


CASES = {
    "general_unsorted_dups": lambda: mtx_text(4, 5, [(3, 5, 1.5), (1, 2, -2.0), (3, 1, 0.25), (3, 5, 4.0),
                                                     (4, 4, 1e-300), (2, 3, -7.125)]),
    "symmetric_real": lambda: mtx_text(5, 5, [(1, 1, 2.0), (3, 1, -1.0), (5, 2, 0.5), (4, 4, 3.0), (5, 3, 9.0),
                                              (2, 1, 1.25)], sym="symmetric"),
    "pattern_general": lambda: mtx_text(6, 3, [(6, 3), (1, 1), (2, 3), (6, 1)], field="pattern"),
    "pattern_symmetric": lambda: mtx_text(4, 4, [(2, 1), (4, 3), (3, 3), (4, 1)], field="pattern", sym="symmetric"),
    "integer_symmetric": lambda: mtx_text(4, 4, [(1, 1, 5), (4, 2, -3), (3, 2, 7)], field="integer", sym="symmetric"),
    "complex_hermitian": lambda: mtx_text(3, 3, [(1, 1, 2.0, 0.0), (3, 1, 1.5, -0.5), (2, 2, -1.0, 0.0)],
                                          field="complex", sym="hermitian"),
    "complex_general": lambda: mtx_text(3, 4, [(1, 4, 0.5, 9.0), (3, 1, -2.0, 1.0)], field="complex"),
    "skew_symmetric": lambda: mtx_text(3, 3, [(2, 1, 1.0), (3, 2, -4.0)], sym="skew-symmetric"),
    "mixed_case_banner": lambda: mtx_text(2, 2, [(1, 2, 3.0)], banner="%%MatrixMarket MATRIX Coordinate Real GENERAL"),
    "crlf": lambda: mtx_text(3, 3, [(1, 1, 1.0), (3, 2, 2.0)], eol="\r\n"),
    "no_comments": lambda: mtx_text(3, 2, [(2, 2, 1.0)], comments=()),
    "number_formats": lambda: "%%MatrixMarket matrix coordinate real general\n3 3 4\n1 1 1e-3\n2 2 -2.5E+2\n"
                              "3 3 .5\n1 3 +7\n",
    "blank_line_before_size": lambda: "%%MatrixMarket matrix coordinate real general\n% c\n\n3 3 1\n2 1 4.5\n",
    "empty": lambda: mtx_text(3, 3, []),
    "random_general": lambda: mtx_text(300, 200, random_entries(300, 200, 2500, 1)),
    "random_symmetric": lambda: mtx_text(300, 300, random_entries(300, 300, 2500, 2, lower=True), sym="symmetric"),
    "random_integer": lambda: mtx_text(100, 120, random_entries(100, 120, 900, 3, field="integer"), field="integer"),
    "random_complex_hermitian": lambda: mtx_text(80, 80, random_entries(80, 80, 400, 4, lower=True, field="complex"),
                                                 field="complex", sym="hermitian"),
}


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_matches_reference_reader(name, tmp_path):
    path = write(tmp_path, name + ".mtx", CASES[name]())
    rc, m, n, sym, rp, ci, v = oracle.ref_mmio(path)
    assert rc == 0
    got = read_mtx(path, np.float64)
    assert (got.rows, got.cols, int(got.symmetric)) == (m, n, sym)
    assert np.array_equal(got.rowptr, rp)
    assert np.array_equal(got.colidx, ci)
    assert np.array_equal(got.val.view(np.uint64), v.view(np.uint64))
    g32 = read_mtx(path, np.float32)
    assert np.array_equal(g32.rowptr, rp) and np.array_equal(g32.colidx, ci)
    assert np.array_equal(g32.val, v.astype(np.float32))
    crc, cm, cn, cnnz, csym, crp, cci, cv = compat.mmio_allinone(path)
    assert (crc, cm, cn, cnnz, csym) == (0, m, n, int(rp[-1]), sym)
    assert np.array_equal(crp, rp) and np.array_equal(cci, ci) and np.array_equal(cv, v)
    assert reference_code(path) == 0


# skew-symmetric: scipy mirrors with negation, the reference not at all; number_formats: scipy's
# parser rejects an explicit '+' sign that strtod and "%lg" accept
@pytest.mark.filterwarnings("ignore::DeprecationWarning")
@pytest.mark.parametrize("name", sorted(set(CASES) - {"skew_symmetric", "number_formats"}))
def test_reader_sums_match_scipy(name, tmp_path):
    sio = pytest.importorskip("scipy.io")
    path = write(tmp_path, name + ".mtx", CASES[name]())
    got = read_mtx(path)
    A = np.zeros((got.rows, got.cols))
    rows = np.repeat(np.arange(got.rows), np.diff(got.rowptr))
    np.add.at(A, (rows, got.colidx), got.val)
    ref = sio.mmread(path)
    # complex files: the reference keeps the real part (scipy conjugates the mirrored hermitian
    # triangle, which leaves the real part as is)
    ref = np.real(ref.toarray() if hasattr(ref, "toarray") else ref)
    assert A.shape == ref.shape
    assert np.allclose(A, ref, rtol=1e-15, atol=0)


def test_skew_symmetric_is_read_as_stored(tmp_path):
    """The reference mirrors only symmetric and hermitian files (src/auxiliary.h:201-205)."""
    path = write(tmp_path, "skew.mtx", CASES["skew_symmetric"]())
    got = read_mtx(path)
    assert not got.symmetric and got.nnz == 2
    assert np.array_equal(got.rowptr, [0, 0, 1, 2]) and np.array_equal(got.colidx, [0, 1])


@needs_ref
def test_reference_return_codes(tmp_path):
    missing = str(tmp_path / "absent.mtx")
    bad_banner = write(tmp_path, "b.mtx", "%%NotMatrixMarket matrix coordinate real general\n1 1 0\n")
    short_banner = write(tmp_path, "s.mtx", "%%MatrixMarket matrix coordinate real\n1 1 0\n")
    bad_field = write(tmp_path, "f.mtx", "%%MatrixMarket matrix coordinate quaternion general\n1 1 0\n")
    no_size = write(tmp_path, "n.mtx", "%%MatrixMarket matrix coordinate real general\n% only comments\n")
    for path, code, status in ((missing, -1, capi.ERR_IO), (bad_banner, -2, capi.ERR_FORMAT),
                               (short_banner, -2, capi.ERR_FORMAT), (bad_field, -2, capi.ERR_FORMAT),
                               (no_size, -4, capi.ERR_FORMAT)):
        assert oracle.ref_mmio(path)[0] == code, path
        assert reference_code(path) == code
        assert compat.mmio_allinone(path)[0] == code
        with pytest.raises(capi.SwiftError) as e:
            read_mtx(path)
        assert e.value.status == status


def test_undefined_inputs_are_errors(tmp_path):
    """Files the reference reads with undefined results (it is never run on these)."""
    cases = {
        "row_out_of_range": ("%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n", capi.ERR_FORMAT),
        "col_zero": ("%%MatrixMarket matrix coordinate real general\n3 3 1\n1 0 1.0\n", capi.ERR_FORMAT),
        "truncated": ("%%MatrixMarket matrix coordinate real general\n3 3 3\n1 1 1.0\n2 2\n", capi.ERR_FORMAT),
        "garbage_value": ("%%MatrixMarket matrix coordinate real general\n3 3 1\n1 1 abc\n", capi.ERR_FORMAT),
        "array_file": ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", capi.ERR_UNSUPPORTED),
        "symmetric_rectangular": ("%%MatrixMarket matrix coordinate real symmetric\n2 4 1\n1 4 1.0\n",
                                  capi.ERR_FORMAT),
    }
    for name, (text, status) in cases.items():
        path = write(tmp_path, name + ".mtx", text)
        with pytest.raises(capi.SwiftError) as e:
            read_mtx(path)
        assert e.value.status == status, name
        assert compat.mmio_allinone(path)[0] in (-2, -5), name


def test_large_file_round_trip(tmp_path):
    """A 20,000 x 20,000 file of 400,000 entries, written with numpy, reads back exactly."""
    rng = np.random.default_rng(7)
    M = 20000
    r = rng.integers(1, M + 1, 400000)
    c = rng.integers(1, M + 1, 400000)
    v = rng.uniform(-1, 1, 400000)
    path = str(tmp_path / "big.mtx")
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{M} {M} {r.size}\n")
        np.savetxt(f, np.column_stack([r, c, v]), fmt=["%d", "%d", "%.17g"])
    got = read_mtx(path)
    order = np.argsort(r, kind="stable")
    assert np.array_equal(got.rowptr, np.concatenate([[0], np.cumsum(np.bincount(r - 1, minlength=M))]))
    assert np.array_equal(got.colidx, (c - 1)[order])
    assert np.array_equal(got.val, v[order])


@pytest.mark.gpu
@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_plan_from_mtx(dt, tmp_path):
    import torch

    from swift_b200 import Plan, gen
    path = write(tmp_path, "sym.mtx", CASES["random_symmetric"]())
    mm = read_mtx(path, dt)
    plan = Plan.from_mtx(path, dt)
    B = gen.dense_uniform(mm.cols, 64, 3, dt)
    ref = oracle.csr_spmm_f64(mm.rows, mm.cols, mm.rowptr, mm.colidx, mm.val, B)
    for engine in ("tiled", "rowwise"):
        C = plan.spmm(torch.from_numpy(B).cuda(), engine=engine).cpu().numpy()
        err = np.abs(C - ref).max() / np.abs(ref).max()
        assert err <= (1e-5 if dt == np.float32 else 1e-12), engine
    plan.close()
    assert os.path.exists(path)
