"""Gram build A = X X^T on the tensor cores (split BF16, FP32 accumulation)
against an FP64 torch reference of the same product."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402


def check_gram(rows, cols, seed, fp64=True):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    X = torch.rand(rows, cols, dtype=torch.float32, device="cuda", generator=g)
    A, A64 = B.gram_build(X, fp64=fp64)
    torch.cuda.synchronize()
    Xd = X.double()
    ref = Xd @ Xd.T
    bound = Xd.abs() @ Xd.abs().T
    err = (A.double() - ref).abs()
    # split BF16 keeps ~16 mantissa bits of each factor: relative 1e-4 of
    # sum |x_ik x_jk| per entry bounds the worst case
    assert (err <= 1e-4 * bound).all(), float((err / bound).max())
    # the FP32 accumulation of the tensor cores dominates for long sums
    assert float((err / bound).mean()) < 5e-5
    assert torch.equal(A, A.T)
    if fp64:
        assert torch.equal(A64, A.double())


@pytest.mark.parametrize("rows,cols", [(256, 256), (128, 64), (300, 1000), (512, 4096)])
def test_gram_tensor_cores(rows, cols):
    check_gram(rows, cols, seed=rows + cols)
