"""Gram build A = X X^T on the tensor cores (split BF16, FP32 accumulation)
against an FP64 torch reference of the same product; the implicit Gram
operator (X on the device, or in host memory streamed by column blocks)
against the CPU oracle's FP64 IRAM on the exact Gram."""
import numpy as np
import pytest

import oracle as O

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


def test_gram_workspace_pool_reuse_and_trim():
    # the build's workspace comes from a library-owned pool that keeps it for
    # the next build: repeated builds give identical results; trimming the
    # pool returns its memory and the next build still runs
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    X = torch.rand(700, 2500, dtype=torch.float32, device="cuda", generator=g)
    A1, _ = B.gram_build(X)
    A2, _ = B.gram_build(X)
    assert torch.equal(A1, A2)
    assert B.lib().oapb_gram_trim() == B.OK
    A3, _ = B.gram_build(X)
    assert torch.equal(A1, A3)


@pytest.mark.parametrize("rows,cols", [(3000, 1000), (4096, 160)])
def test_gram_more_tiles_than_sms(rows, cols):
    # more upper-triangle tiles than SMs (156 and 272): a second wave of
    # CTAs, ragged edge tiles, one partial per tile through the finishing
    # kernel
    check_gram(rows, cols, seed=7 * rows + cols)


def separated_images(rows, cols, seed):
    """images = 8 separated components + noise: a well-separated top spectrum"""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    U = torch.randn(rows, 8, generator=g, device="cuda", dtype=torch.float64)
    V = torch.randn(8, cols, generator=g, device="cuda", dtype=torch.float64)
    S = torch.tensor([10.0, 8.0, 6.5, 5.0, 4.0, 3.0, 2.4, 2.0], device="cuda", dtype=torch.float64)
    return ((U * S) @ V / cols ** 0.5 + 0.05 * torch.randn(rows, cols, generator=g, device="cuda",
                                                           dtype=torch.float64)).float().contiguous()


def oracle_gram_eigenvalues(X, k, m):
    """The CPU oracle's FP64 IRAM on the exact Gram of the FP32 images."""
    Xd = X.double().cpu().numpy()
    A = Xd @ Xd.T
    o = O.iram(A, k, m, which="LM", tol=1e-12, seed=3)
    assert o["rc"] == 0
    return np.sort(o["eigenvalues"].real)[::-1]


@pytest.mark.gpu
@pytest.mark.parametrize("rows,cols", [(600, 3000), (513, 1027)])
def test_implicit_gram_operator_matches_oracle(rows, cols):
    # w = X (X^T v) never forming A: the eigenpairs of the exact Gram of the
    # FP32 images, against the CPU oracle's FP64 IRAM on that Gram
    X = separated_images(rows, cols, rows)
    imp = B.Arnoldi(rows, 24, 6, seed=3)
    imp.set_gram_operator(X)
    ev, res, st = imp.solve()
    assert st == B.OK and max(res) <= 1e-10
    ref = oracle_gram_eigenvalues(X, 6, 24)
    assert np.allclose(np.sort(np.array(ev).real)[::-1], ref, rtol=1e-11, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("cols,block_cols,resident", [(3000, 1000, 0), (1027, 256, 2), (2048, 4096, 0),
                                                      (1027, 100, 10 ** 9)])
def test_host_streamed_gram_operator_matches_oracle(cols, block_cols, resident):
    # X in pinned host memory, applied by column blocks (some resident, the
    # rest streamed on every application, ragged last blocks): the same
    # eigenvalues as the CPU oracle's FP64 IRAM on the exact Gram, and the
    # bytes streamed per application equal the non-resident blocks
    rows = 600
    X = separated_images(rows, cols, cols + block_cols)
    Xh = X.cpu().pin_memory()
    s = B.Arnoldi(rows, 24, 6, seed=3)
    s.set_gram_operator_host(Xh, block_cols, resident_bytes=resident * 4 * rows * ((block_cols + 3) // 4 * 4))
    nb, nres, by0 = s.gram_stream_info()
    bc = min(cols, (block_cols + 3) // 4 * 4)
    assert nb == -(-cols // bc) and nres == min(nb, resident) and by0 == 0
    ev, res, st = s.solve()
    assert st == B.OK and max(res) <= 1e-10
    ref = oracle_gram_eigenvalues(X, 6, 24)
    assert np.allclose(np.sort(np.array(ev).real)[::-1], ref, rtol=1e-11, atol=0)
    nb, nres, by = s.gram_stream_info()
    per_application = 4 * rows * (cols - min(cols, nres * bc))
    if per_application == 0:
        assert by == 0
    else:  # every application (Arnoldi steps and residual checks) streams the same bytes
        assert by % per_application == 0 and by // per_application >= s.stats()["matvecs"]


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
