"""The CPU network oracle itself: its output-layer gradient and loss agree with
a direct restatement (parameters and inputs exact in BF16)."""
import numpy as np

from oracle import mlp as M


def test_oracle_output_layer_gradient():
    rng = np.random.default_rng(0)
    sizes = [3, 5, 4]
    npar = 3 * 5 + 5 * 4 + 5 + 4
    # BF16-exact parameters and inputs: multiples of 1/64 in [-1, 1]
    p = (rng.integers(-64, 65, size=npar) / 64.0).astype(np.float32)
    x = (rng.integers(-64, 65, size=(6, 3)) / 64.0).astype(np.float32)
    t = rng.normal(size=(6, 4))
    loss, g = M.loss_and_grads(p, sizes, x, t)
    # compare only the output layer (no BF16 rounding of intermediate values
    # enters its gradient) with central differences in float64
    W, b = M.unpack(p.astype(np.float64), sizes)
    hf, hb = M.forward(p, sizes, x)
    h = hb[1]
    y = h @ W[1].T + b[1]
    # the device rounds dY to BF16 before the weight-gradient product
    dy = M.bf16(((y - t) / 6.0).astype(np.float32)).astype(np.float64)
    gW = dy.T @ h
    assert np.allclose(g[15:35].reshape(4, 5), gW, rtol=1e-6, atol=1e-9)
    # and the loss is the plain mean squared error / 2
    assert np.isclose(loss, 0.5 * np.sum((y - t) ** 2) / 6.0, rtol=1e-6)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] - (-3.140625)) < 1e-6
