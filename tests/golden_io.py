"""Loads the fixtures made by tests/golden/make_golden.py (reference outputs)."""
import os

import numpy as np

import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

SCALARS = ["tilenum", "regular_nnz", "reside_col", "reside_nnz", "segsum", "numblk", "nsteps"]
ARRAYS = ["tile_ptr", "tile_len", "tile_colidx", "tile_tall", "sortrowidx", "sortval",
          "reside_cscptr", "reside_cscrowidx", "reside_val", "tile_format", "segmentoffset",
          "sortrowindex", "colorblk", "blkstart", "blkstop", "blkptr", "rowsorted_rowidx",
          "val_position", "val_offset"]


def _split(npz, prefix):
    d = {k[len(prefix):]: npz[k] for k in npz.files if k.startswith(prefix) and "/" not in k[len(prefix):]}
    for k in ("M", "K") + tuple(SCALARS):
        if k in d:
            d[k] = int(d[k])
    return d


def load(name: str, dtype=np.float32):
    """Fixture for 'poisson4096' or one of cases.SMALL, FP32 inputs; with dtype float64 the
    inputs are widened and C is the reference's FP64 result."""
    if name == "poisson4096":
        d = _split(np.load(os.path.join(GOLDEN, "poisson4096_n32_f32.npz")), "")
        c64 = np.load(os.path.join(GOLDEN, "poisson4096_n32_f64.npz"))["C"]
    else:
        assert name in cases.SMALL, name
        d = _split(np.load(os.path.join(GOLDEN, "small_f32.npz")), name + "/")
        c64 = np.load(os.path.join(GOLDEN, "small_f64.npz"))[name + "/C"]
    if dtype == np.float64:
        for k in ("val", "B", "sortval", "reside_val"):
            d[k] = d[k].astype(np.float64)
        d["C"] = c64
    return d


ALL = ["poisson4096"] + cases.SMALL
