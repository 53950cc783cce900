"""The C-ABI library loads without a GPU and exports every function include/swift_b200.h
declares (no compute call is made here)."""
import ctypes
import os
import re

import pytest

from swift_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "swift_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", text)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(swift_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("library not built")
    return ctypes.CDLL(capi.LIB_PATH)


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    assert len(names) >= 40
    for n in ("swift_plan_create", "swift_spmm", "swift_spmm_noalloc", "swift_ref_spmm_f32",
              "swift_ref_formattransation_f64", "swift_ref_row_idx_sort_f32", "swift_batch_run_graph"):
        assert n in names, n


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_matches_exports(lib):
    missing = [name for name, _, _ in capi._SIGS if not hasattr(lib, name)]
    assert not missing, missing
    capi.lib()  # sets every restype/argtypes


def test_status_strings_without_gpu(lib):
    L = capi.lib()
    assert L.swift_status_string(capi.OK).decode()
    assert L.swift_version().decode()
