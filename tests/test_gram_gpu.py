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


@pytest.mark.parametrize("rows,cols", [(256, 256), (128, 64), (300, 1000), (512, 4096), (1, 5), (129, 31)])
def test_gram_tensor_cores(rows, cols):
    check_gram(rows, cols, seed=rows + cols)


@pytest.mark.parametrize("rows,cols", [(3000, 1000), (4096, 160)])
def test_gram_stream_k_split_tiles(rows, cols):
    # more upper-triangle tiles than SMs (156 and 272): the stream-K shares
    # split tiles between two CTAs, whose partials the finishing kernel adds
    check_gram(rows, cols, seed=7 * rows + cols)


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols", [(600, 3000), (513, 1027)])
def test_implicit_gram_operator_matches_explicit(rows, cols):
    # w = X (X^T v) never forming A; eigenpairs vs the solve on the FP64 Gram
    # of the same FP32 images (the implicit operator is that Gram exactly)
    g = torch.Generator(device="cuda")
    g.manual_seed(rows)
    # images = 8 separated components + noise: well-separated top spectrum
    U = torch.randn(rows, 8, generator=g, device="cuda", dtype=torch.float64)
    V = torch.randn(8, cols, generator=g, device="cuda", dtype=torch.float64)
    S = torch.tensor([10.0, 8.0, 6.5, 5.0, 4.0, 3.0, 2.4, 2.0], device="cuda", dtype=torch.float64)
    X = ((U * S) @ V / cols ** 0.5 + 0.05 * torch.randn(rows, cols, generator=g, device="cuda",
                                                         dtype=torch.float64)).float().contiguous()
    A64 = X.double() @ X.double().T
    ref = B.Arnoldi(rows, 24, 6, seed=3)
    ref.set_operator(A64.contiguous())
    ev_ref, res_ref, st = ref.solve()
    assert st == B.OK
    imp = B.Arnoldi(rows, 24, 6, seed=3)
    imp.set_gram_operator(X)
    ev, res, st = imp.solve()
    assert st == B.OK and max(res) <= 1e-10
    assert np.allclose(np.array(ev).real, np.array(ev_ref).real, rtol=1e-11, atol=0)


@pytest.mark.gpu
def test_images_to_matrix_matches_reference_conversion():
    # (r << 16 | g << 8 | b) / 0xFFFFFF per pixel (Image::convertRgbToFloatt),
    # from host and from device buffers, one image per row of X
    rng = np.random.default_rng(8)
    rgb = rng.integers(0, 256, size=(7, 1000, 3), dtype=np.uint8)
    expect = ((rgb[..., 0].astype(np.int64) << 16) | (rgb[..., 1].astype(np.int64) << 8) | rgb[..., 2]) / 16777215.0
    X = B.images_to_matrix(rgb)
    assert np.array_equal(X.cpu().numpy(), expect.astype(np.float32))
    Xd = B.images_to_matrix(torch.from_numpy(rgb).cuda())
    assert torch.equal(Xd, X)
