"""Operand checks of the Python layer (swift_b200.plan._dense / _vec), run on CPU: every dense
operand and vector is checked for shape, dtype and CUDA residence before its pointer reaches
the C ABI, so a wrong shape or a host tensor is an error on the host instead of an out-of-bounds
access on the GPU."""
import pytest

from swift_b200 import plan as P

torch = pytest.importorskip("torch")


def test_dense_operand_shape_dtype_and_device():
    with pytest.raises(ValueError, match="2-D"):
        P._dense(torch.zeros(6), 2, 3, "B")
    with pytest.raises(ValueError, match=r"shape \(3, 2\), expected \(2, 3\)"):
        P._dense(torch.zeros(3, 2), 2, 3, "B")
    with pytest.raises(ValueError, match="dtype"):
        P._dense(torch.zeros(2, 3, dtype=torch.float64), 2, 3, "C_out", torch.float32)
    # right shape and dtype, but in host memory
    with pytest.raises(ValueError, match="CUDA tensor"):
        P._dense(torch.zeros(2, 3), 2, 3, "B", torch.float32)
    with pytest.raises(ValueError, match="CUDA tensor"):
        P._dense(torch.zeros(0, 3), 0, 3, "B")


def test_vector_operand_checks():
    with pytest.raises(ValueError, match="5 elements"):
        P._vec(torch.zeros(4), 5, "c_scale", torch.float32)
    with pytest.raises(ValueError, match="contiguous"):
        P._vec(torch.zeros(10)[::2], 5, "b_scale", torch.float32)
    with pytest.raises(ValueError, match="float32"):
        P._vec(torch.zeros(5, dtype=torch.float16), 5, "b_scale", torch.float32)
    with pytest.raises(ValueError, match="CUDA tensor"):
        P._vec(torch.zeros(5), 5, "dA", torch.float32)
