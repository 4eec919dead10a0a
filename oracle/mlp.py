"""CPU oracle of the warm-start network (test infrastructure only).

Restates, in numpy, the arithmetic of oap_b200/csrc/mlp.cu: weights and
activations rounded to BF16 (round to nearest even) where the device rounds
them, products accumulated in float64 (the device accumulates in FP32),
per-layer activations (default tanh hidden layers, linear output), loss
1/(2B) sum (y - t)^2.  Parameter packing: weight matrices [out x in] in layer
order, then the biases.

The activations are the reference's (oapNeuralHost/oapLayerStructure.h:32-38,
in its order: LINEAR 0, SIGMOID 1, TANH 2, SIN 3) with the derivatives its
derivativeFunc applies (oapNeuralHost/oapGenericNeuralApi.h:102-120; element
bodies oapMatrixCuda/CuProcedures/CuSigmoidProcedures.h:27-37,
CuTanhProcedures.h:27-37, CuSinProcedures.h:27-35): sigmoid' = h (1 - h),
tanh' = 1 - h^2, sin' = cos z, for h the activation of z.
"""
import numpy as np

LINEAR, SIGMOID, TANH, SIN = 0, 1, 2, 3


def default_acts(nlayers):
    return [TANH] * (nlayers - 1) + [LINEAR]


def act(z, a):
    if a == SIGMOID:
        return 1.0 / (1.0 + np.exp(-z))
    if a == TANH:
        return np.tanh(z)
    if a == SIN:
        return np.sin(z)
    return z


def act_grad(z, h, a):
    if a == SIGMOID:
        return h * (1.0 - h)
    if a == TANH:
        return 1.0 - h * h
    if a == SIN:
        return np.cos(z)
    return np.ones_like(h)


def bf16(x):
    """Round float32 values to BF16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(params, sizes):
    W, b, off = [], [], 0
    for l in range(len(sizes) - 1):
        n = sizes[l] * sizes[l + 1]
        W.append(params[off:off + n].reshape(sizes[l + 1], sizes[l]))
        off += n
    for l in range(len(sizes) - 1):
        b.append(params[off:off + sizes[l + 1]])
        off += sizes[l + 1]
    return W, b


def forward(params, sizes, x, acts=None, with_z=False):
    W, b = unpack(params, sizes)
    L = len(W)
    acts = default_acts(L) if acts is None else list(acts)
    hb = [bf16(x).astype(np.float64)]
    hf, zs = [], []
    for l in range(L):
        z = (hb[-1] @ bf16(W[l]).astype(np.float64).T + b[l]).astype(np.float32)
        h = act(z.astype(np.float64), acts[l]).astype(np.float32)
        zs.append(z)
        hf.append(h)
        hb.append(bf16(h).astype(np.float64))
    return (hf, hb, zs) if with_z else (hf, hb)


def loss_and_grads(params, sizes, x, t, acts=None):
    """(loss, gradient vector) with the device's rounding points."""
    W, b = unpack(params, sizes)
    L = len(W)
    acts = default_acts(L) if acts is None else list(acts)
    B = x.shape[0]
    hf, hb, zs = forward(params, sizes, x, acts, with_z=True)
    y = hf[-1].astype(np.float64)
    d = y - t
    loss = 0.5 * np.sum(d * d) / B
    g = (d / B).astype(np.float32)
    if acts[-1] != LINEAR:
        g = (g.astype(np.float64) * act_grad(zs[-1].astype(np.float64), y, acts[-1])).astype(np.float32)
    gW, gb = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        gbf = bf16(g).astype(np.float64)
        gW[l] = gbf.T @ hb[l]
        gb[l] = g.astype(np.float64).sum(axis=0)
        if l == 0:
            break
        dx = (gbf @ bf16(W[l]).astype(np.float64)).astype(np.float32).astype(np.float64)
        h = hf[l - 1].astype(np.float64)
        g = (dx * act_grad(zs[l - 1].astype(np.float64), h, acts[l - 1])).astype(np.float32)
    vec = np.concatenate([w.ravel() for w in gW] + [v.ravel() for v in gb])
    return loss, vec
