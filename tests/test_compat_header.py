"""include/swift_compat.h: the reference's C++ signatures over the C ABI.

CPU: the header compiles in both flavours and a driver program written like the reference's
main links against libswiftb200.so.  GPU: that driver runs the whole reference chain and every
SpMM wrapper passes the reference's own check (|C - golden| <= 1e-2, src/auxiliary.h:156-165).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
DRIVER = os.path.join(ROOT, "tests", "compat_driver.cpp")
LIBDIR = os.path.join(ROOT, "swift-high-performance-sparse-dense-matrix-multiplication-on-gpus_b200", "swift_b200")

CXX = shutil.which("g++") or shutil.which("c++")
pytestmark = pytest.mark.skipif(CXX is None, reason="no C++ compiler")


def build_driver(out, fp32):
    cmd = [CXX, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", INCLUDE, DRIVER, "-o", out,
           "-L", LIBDIR, "-lswiftb200", "-Wl,-rpath," + LIBDIR]
    if fp32:
        cmd.insert(1, "-DSWIFT_COMPAT_FP32")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("fp32", [False, True])
def test_header_compiles(fp32, tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "swift_compat.h"\nint main() { slide_matrix m{}; Tile_destroy(&m); return 0; }\n')
    cmd = [CXX, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-I", INCLUDE, str(src)]
    if fp32:
        cmd.insert(1, "-DSWIFT_COMPAT_FP32")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("fp32", [False, True])
def test_driver_links(fp32, tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libswiftb200.so")):
        pytest.skip("library not built")
    build_driver(str(tmp_path / "drv"), fp32)


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("shape", [(2000, 1500, 0.01, 32, 1), (700, 300, 0.05, 64, 2), (64, 20, 0.2, 8, 3)])
def test_driver_runs_reference_chain(fp32, shape, tmp_path):
    drv = build_driver(str(tmp_path / "drv"), fp32)
    r = subprocess.run([drv] + [str(x) for x in shape], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "NO PASS" not in r.stdout
    assert r.stdout.count("GFLOP/s") == 5


HELPERS = r'''
#include <cstdio>
#include "swift_compat.h"
int main() {
  float t = 7.f;
  result_check(3.f, 2.f, 5.f, t); if (t != 2.f) return 1;
  result_check(-1.f, 2.f, 5.f, t); if (t != 2.f) return 2;
  result_check(4.f, -1.f, 3.f, t); if (t != 3.f) return 3;
  result_check(-1.f, -1.f, -1.f, t); if (t != -1.f) return 4;
  t = 9.f; result_check(-1.f, -1.f, 5.f, t); if (t != 9.f) return 5;  // one valid: unchanged
  double a[6] = {1, 2, 3, 4, 5, 6}, b[6];
  dense_mtx2dense_mtx_spmm(2, 3, a, b);  // 2 x 3 -> 3 x 2
  const double want[6] = {1, 4, 2, 5, 3, 6};
  for (int i = 0; i < 6; ++i) if (b[i] != want[i]) return 6;
  float x[3] = {0.f, 1.f, 2.f}, y[3] = {0.f, 1.005f, 2.5f};
  int err = 1;
  ResultVerify(x, y, 3, err); if (err != 2) return 7;
  return 0;
}
'''


def test_driver_helpers_match_the_reference_semantics(tmp_path):
    src = tmp_path / "h.cpp"
    src.write_text(HELPERS)
    exe = str(tmp_path / "h")
    r = subprocess.run([CXX, "-std=c++17", "-Wall", "-Werror", "-I", INCLUDE, str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([exe]).returncode == 0


MMIO = r"""
#include <cstdio>
#include <cstdlib>
#include "swift_compat.h"
int main(int argc, char **argv) {
  int m, n, nnz, sym, *rp, *ci;
  double *v;
  if (mmio_allinone(&m, &n, &nnz, &sym, &rp, &ci, &v, argv[1]) != 0) return 1;
  // 3 x 3 symmetric: (1,1)=2, (3,1)=-1 -> row 0: [0]=2, [2]=-1; row 2: [0]=-1
  if (m != 3 || n != 3 || nnz != 3 || sym != 1) return 2;
  if (rp[0] != 0 || rp[1] != 2 || rp[2] != 2 || rp[3] != 3) return 3;
  if (ci[0] != 0 || ci[1] != 2 || ci[2] != 0 || v[0] != 2.0 || v[1] != -1.0 || v[2] != -1.0) return 4;
  free(rp); free(ci); free(v);
  float *f;
  if (mmio_allinone(&m, &n, &nnz, &sym, &rp, &ci, &f, argv[1]) != 0 || f[1] != -1.0f) return 5;
  free(rp); free(ci); free(f);
  if (mmio_allinone(&m, &n, &nnz, &sym, &rp, &ci, &v, argv[2]) != -1) return 6;   // missing file
  return 0;
}
"""


def test_mmio_allinone_shim(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libswiftb200.so")):
        pytest.skip("library not built")
    mtx = tmp_path / "a.mtx"
    mtx.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n1 1 2.0\n3 1 -1.0\n")
    src = tmp_path / "m.cpp"
    src.write_text(MMIO)
    exe = str(tmp_path / "m")
    r = subprocess.run([CXX, "-std=c++17", "-Wall", "-Werror", "-I", INCLUDE, str(src), "-o", exe, "-L", LIBDIR,
                        "-lswiftb200", "-Wl,-rpath," + LIBDIR], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([exe, str(mtx), str(tmp_path / "absent.mtx")]).returncode == 0
