"""Swift SpMM on B200: Python layer over libswiftb200.so (the C ABI in include/swift_b200.h).

The compute path is the CUDA library; this package only binds it (ctypes), provides the
torch.autograd.Function for the backward pass, and the seeded input generators.
"""
from . import _capi as capi  # noqa: F401
from .plan import Batch, Plan  # noqa: F401

__all__ = ["Plan", "Batch", "capi", "lib_path"]
# torch.autograd binding: swift_b200.autograd (swift_spmm, SwiftSpMMFunction, SwiftSparseLinear)


def lib_path() -> str:
    return capi.LIB_PATH
