"""The reference's own driver programs, unmodified, on this library.

oracle/Makefile (target refdrv) compiles test/k-32/FP32/main.cu (FP32, N = 32) and src/main.cu
(FP64, N = 32) against include/swift_compat.h: the stand-ins in tests/refdrop take the place
of every reference header the drivers include except Swift_cpu.h and gpu_cusparse_spmm.h,
which stay the reference's own.  Each driver reads a MatrixMarket file with the library's
reader, checks the library's CSR-to-CSC (its own test against the CSR product), runs the
library's format build (col_sort, formattransation, block_catgory, balance, row_idx_sort),
checks the reference's Swift_cpu over the library's format arrays against its golden product,
then runs the five GPU wrappers, each against that golden (|C - golden| <= 1e-2,
src/auxiliary.h:156-165), and prints the best time (src/main.cu:207-441,
test/k-32/FP32/main.cu:217-455).

The binaries are built where the reference checkout is present (they travel with
oracle/_ref); without them these tests skip.
"""
import os
import subprocess

import numpy as np
import pytest

from swift_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVERS = {"f32": os.path.join(ROOT, "oracle", "_ref", "refdrv_f32"),
           "f64": os.path.join(ROOT, "oracle", "_ref", "refdrv_f64")}


def write_mtx(path, M, K, rowptr, colidx, symmetric=False):
    rows = np.repeat(np.arange(M), np.diff(rowptr))
    kind = "symmetric" if symmetric else "general"
    if symmetric:
        keep = rows >= colidx
        rows, cols = rows[keep], colidx[keep]
    else:
        cols = colidx
    vals = gen.uniform_values(rows.size, 5, np.float64)
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real {kind}\n% written by the test\n")
        f.write(f"{M} {K} {rows.size}\n")
        for r, c, v in zip(rows, cols, vals):
            f.write(f"{r + 1} {c + 1} {v:.17g}\n")


def matrices(tmp_path):
    out = []
    rp, ci = gen.rmat(12, 16 << 12, seed=1)
    write_mtx(tmp_path / "rmat12.mtx", 4096, 4096, rp, ci)
    out.append(tmp_path / "rmat12.mtx")
    rp, ci = gen.poisson_uniform(3000, 2500, 12.0, seed=2)
    write_mtx(tmp_path / "poisson_rect.mtx", 3000, 2500, rp, ci)
    out.append(tmp_path / "poisson_rect.mtx")
    rp, ci = gen.rmat(11, 8 << 11, seed=3, symmetric=True)
    write_mtx(tmp_path / "rmat11_sym.mtx", 2048, 2048, rp, ci, symmetric=True)
    out.append(tmp_path / "rmat11_sym.mtx")
    return out


@pytest.mark.parametrize("flavour", ["f32", "f64"])
def test_reference_driver_is_built_against_the_library(flavour):
    drv = DRIVERS[flavour]
    if not os.path.exists(drv):
        pytest.skip("reference drivers not built (needs the reference checkout at build time)")
    r = subprocess.run(["ldd", drv], capture_output=True, text=True)
    assert r.returncode == 0
    assert "libswiftb200.so" in r.stdout and "not found" not in r.stdout.split("libswiftb200.so")[1].split("\n")[0]


@pytest.mark.gpu
@pytest.mark.parametrize("flavour", ["f32", "f64"])
def test_reference_driver_runs_on_the_library(flavour, tmp_path):
    drv = DRIVERS[flavour]
    if not os.path.exists(drv):
        pytest.skip("reference drivers not built (needs the reference checkout at build time)")
    (tmp_path / "data").mkdir()  # the drivers append their result line to ./data/
    for path in matrices(tmp_path):
        r = subprocess.run([drv, "-d", "0", str(path)], capture_output=True, text=True, timeout=600,
                           cwd=str(tmp_path))
        log = f"{path.name}:\n{r.stdout}\n{r.stderr}"
        assert r.returncode == 0, log
        assert "NO PASS" not in r.stdout, log
        assert "failed" not in r.stderr, log
        # the library's csr_to_csc against the driver's own CSR product: the FP32 driver prints
        # a success line (test/k-32/FP32/main.cu), the FP64 one only an error line
        # (src/main.cu:226-232)
        if flavour == "f32":
            assert "success format csc" in r.stdout, log
        assert "error format csc" not in r.stdout, log
        assert "success Swift CPU" in r.stdout, log   # the reference's Swift_cpu on the library's format
        # best of the five wrappers, all checked (src/main.cu:451 prints "Swift GPU SpMM time")
        assert ("Swift GPU time:" if flavour == "f32" else "Swift GPU SpMM time") in r.stdout, log
    lines = (tmp_path / "data" / ("results_Swift_FP32_32.txt" if flavour == "f32" else "results_Swift_32.txt")).read_text()
    assert len(lines.strip().splitlines()) == 3  # one result line per matrix, none marked failed
