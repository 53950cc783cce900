"""The oracle reproduces the committed reference fixtures bit for bit (runs without the
reference checkout, so it also pins the oracle on the GPU box)."""
import numpy as np
import pytest

import golden_io
import oracle
from test_oracle import check_val_position


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", golden_io.ALL)
def test_oracle_reproduces_fixture(name, dt):
    g = golden_io.load(name, dt)
    out = oracle.pipeline(g["M"], g["K"], g["rowptr"], g["colidx"], g["val"], g["B"], impl="oracle")
    assert np.array_equal(out["perm"], g["perm"])
    assert np.array_equal(out["nnzpercol"], g["nnzpercol"])
    assert np.array_equal(out["csccolptr"], g["csccolptr"])
    s = out["slide"]
    for k in golden_io.SCALARS:
        assert getattr(s, k) == g[k], k
    for k in golden_io.ARRAYS:
        if k == "val_position":
            continue
        a = s[k]
        assert np.array_equal(a, g[k].astype(a.dtype)), k
    check_val_position(s["sortrowidx"], g["rowsorted_rowidx"], g["val_position"], s.tilenum)
    assert out["C"].dtype == dt
    assert np.array_equal(out["C"], g["C"])


def test_fixture_is_the_parity_workload():
    g = golden_io.load("poisson4096")
    assert g["M"] == g["K"] == 4096 and g["B"].shape == (4096, 32)
    lens = np.diff(g["rowptr"])
    assert 15.5 < lens.mean() < 16.5 and g["regular_nnz"] + g["reside_nnz"] == g["rowptr"][-1]
    assert np.abs(g["val"]).max() <= 1.0 and np.abs(g["B"]).max() <= 1.0
