"""CPU oracle of the warm-start network (test infrastructure only).

Restates, in numpy, the arithmetic of oap_b200/csrc/mlp.cu: weights and
activations rounded to BF16 (round to nearest even) where the device rounds
them, products accumulated in float64 (the device accumulates in FP32),
tanh hidden layers, linear output, loss 1/(2B) sum (y - t)^2.  Parameter
packing: weight matrices [out x in] in layer order, then the biases.
"""
import numpy as np


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


def forward(params, sizes, x):
    W, b = unpack(params, sizes)
    hb = [bf16(x).astype(np.float64)]
    hf = []
    L = len(W)
    for l in range(L):
        z = hb[-1] @ bf16(W[l]).astype(np.float64).T + b[l]
        if l + 1 < L:
            h = np.tanh(z).astype(np.float32)
            hf.append(h)
            hb.append(bf16(h).astype(np.float64))
        else:
            hf.append(z.astype(np.float32))
    return hf, hb


def loss_and_grads(params, sizes, x, t):
    """(loss, gradient vector) with the device's rounding points."""
    W, b = unpack(params, sizes)
    L = len(W)
    B = x.shape[0]
    hf, hb = forward(params, sizes, x)
    y = hf[-1].astype(np.float64)
    d = y - t
    loss = 0.5 * np.sum(d * d) / B
    g = (d / B).astype(np.float32)
    gW, gb = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        gbf = bf16(g).astype(np.float64)
        gW[l] = gbf.T @ hb[l]
        gb[l] = g.astype(np.float64).sum(axis=0)
        if l == 0:
            break
        dx = gbf @ bf16(W[l]).astype(np.float64)
        h = hf[l - 1].astype(np.float64)
        g = (dx * (1.0 - h * h)).astype(np.float32)
    vec = np.concatenate([w.ravel() for w in gW] + [v.ravel() for v in gb])
    return loss, vec
