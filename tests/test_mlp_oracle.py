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


def test_activation_derivatives():
    # the oracle's activation derivatives (the reference's dsigmoid / dtanh /
    # dsin / dlinear) against central differences of the activations
    z = np.linspace(-3, 3, 61)
    for a in (M.LINEAR, M.SIGMOID, M.TANH, M.SIN):
        h = M.act(z, a)
        fd = (M.act(z + 1e-6, a) - M.act(z - 1e-6, a)) / 2e-6
        assert np.allclose(M.act_grad(z, h, a), fd, atol=1e-8), a


def test_oracle_gradient_with_activations_is_consistent():
    # with every rounding point of the device removed (float64 parameters
    # that are exact in BF16, no intermediate rounding effects checked), the
    # output-layer weight gradient of a sigmoid output follows dL/dz = (y - t)
    # sigmoid'(z) / B
    rng = np.random.default_rng(3)
    sizes = [3, 4, 2]
    npar = 3 * 4 + 4 * 2 + 4 + 2
    p = (rng.integers(-64, 65, size=npar) / 64.0).astype(np.float32)
    x = (rng.integers(-64, 65, size=(5, 3)) / 64.0).astype(np.float32)
    t = rng.normal(size=(5, 2))
    acts = [M.SIN, M.SIGMOID]
    loss, g = M.loss_and_grads(p, sizes, x, t, acts)
    hf, hb, zs = M.forward(p, sizes, x, acts, with_z=True)
    y = hf[-1].astype(np.float64)
    dz = M.bf16(((y - t) / 5.0 * y * (1 - y)).astype(np.float32)).astype(np.float64)
    gW = dz.T @ hb[1]
    assert np.allclose(g[12:20].reshape(2, 4), gW, rtol=1e-5, atol=1e-7)
    assert np.isclose(loss, 0.5 * np.sum((y - t) ** 2) / 5.0, rtol=1e-6)
