"""The int8-slice arithmetic of the FP64-class block pass, restated in numpy
(CPU): operator rows cut into 6 signed 7-bit digits below a power-of-two row
scale, vectors into 7 below a per-vector scale, slice products of order
i + j <= 8 summed exactly in integers and scaled by 2^-7(i+j).  Checks the
digit ranges, that |acc_o| grows by at most 32640 per K column (so a
16384-column segment fits int32), and the error bound the GPU test asserts
for the pass (2^-40 of the row maximum times |x|_1 plus 2^-45 n of row
maximum times vector maximum)."""
import numpy as np
import pytest

SA, SX = 6, 7


def scale_exponent(m):
    """e with m 2^-e <= 127/128 (0 for m = 0)."""
    m = np.asarray(m, dtype=np.float64)
    f, e = np.frexp(m)
    e = np.where(f > 127.0 / 128.0, e + 1, e)
    return np.where(m > 0, e, 0).astype(np.int64)


def slices(v, ns):
    """digits d_i (int64) with v = sum_i d_i 2^-7(i+1) + remainder."""
    out = []
    v = v.astype(np.float64).copy()
    for _ in range(ns):
        v *= 128.0
        t = np.rint(v)
        out.append(t.astype(np.int64))
        v -= t
    return out, v


def i8_product(A, X):
    """W = A X^T by the pass's slice arithmetic (A: rows x n, X: b x n, real)."""
    ea = scale_exponent(np.abs(A).max(axis=1))
    ex = scale_exponent(np.abs(X).max(axis=1))
    a, _ = slices(A * np.ldexp(1.0, -ea)[:, None], SA)
    x, _ = slices(X * np.ldexp(1.0, -ex)[:, None], SX)
    acc = {}
    for i in range(SA):
        for j in range(SX - i):
            o = i + j
            acc[o] = acc.get(o, 0) + a[i] @ x[j].T  # exact in int64
    W = np.zeros((A.shape[0], X.shape[0]))
    for o in sorted(acc):
        W += acc[o].astype(np.float64) * 2.0 ** (-7 * (o + 2))
    return W * np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, ex)[None, :], acc, a, x


def test_digit_ranges_and_remainder():
    rng = np.random.default_rng(5)
    v = rng.uniform(-127 / 128, 127 / 128, 20000)
    d, rem = slices(v, SX)
    assert np.abs(d[0]).max() <= 127
    assert all(np.abs(di).max() <= 64 for di in d[1:])
    assert np.abs(rem).max() <= 0.5
    back = sum(di * 2.0 ** (-7 * (i + 1)) for i, di in enumerate(d)) + rem * 2.0 ** (-7 * SX)
    assert np.array_equal(back, v)


def test_scale_exponent_keeps_first_digit_in_int8():
    for m in [1.0, 0.5, 127 / 128, 0.999, 3.0, 4.0, 1e-300, 7e10]:
        e = int(scale_exponent(m))
        assert m * 2.0 ** -e <= 127 / 128
        assert m * 2.0 ** -e > 127 / 512  # at most two bits of headroom lost
    assert int(scale_exponent(0.0)) == 0


def test_order_accumulators_grow_at_most_32640_per_column():
    # worst case digits: |d_0| = 127, |d_i| = 64 after it, all of one sign
    a = [127] + [64] * (SA - 1)
    x = [127] + [64] * (SX - 1)
    per_col = max(sum(a[i] * x[o - i] for i in range(SA) if 0 <= o - i < SX) for o in range(SX))
    assert per_col == 32640
    assert per_col * 16384 < 2 ** 31


@pytest.mark.parametrize("n,b", [(96, 5), (257, 16), (64, 32)])
def test_slice_product_error_bound(n, b):
    rng = np.random.default_rng(n + b)
    rs = 10.0 ** rng.uniform(-6, 6, n)
    A = rng.standard_normal((n, n)) / n ** 0.5 * rs[:, None]
    A[np.arange(0, n, 17), np.arange(0, n, 17)] += 4.0 * rs[::17]
    X = rng.standard_normal((b, n)) * 10.0 ** rng.uniform(-3, 3, b)[:, None]
    X[:, ::5] *= 1e-9
    W, acc, a, x = i8_product(A, X)
    ref = A @ X.T
    bound = (2.0 ** -40 * np.abs(A).max(axis=1)[:, None] * np.abs(X).sum(axis=1)[None, :]
             + 2.0 ** -45 * n * np.abs(A).max(axis=1)[:, None] * np.abs(X).max(axis=1)[None, :])
    err = np.abs(W - ref)
    assert (err <= bound).all(), (err / bound).max()
    # the integer sums stay far inside int32 at this size
    assert max(int(np.abs(v).max()) for v in acc.values()) < 2 ** 31


def test_dropped_orders_are_below_the_bound():
    # keeping every order (i + j up to 11) changes W by less than the bound
    rng = np.random.default_rng(11)
    n, b = 200, 8
    A = rng.standard_normal((n, n))
    X = rng.standard_normal((b, n))
    W, _, a, x = i8_product(A, X)
    ea = scale_exponent(np.abs(A).max(axis=1))
    ex = scale_exponent(np.abs(X).max(axis=1))
    full = np.zeros_like(W)
    for i in range(SA):
        for j in range(SX):
            full += (a[i] @ x[j].T).astype(np.float64) * 2.0 ** (-7 * (i + j + 2))
    full *= np.ldexp(1.0, ea)[:, None] * np.ldexp(1.0, ex)[None, :]
    bound = 2.0 ** -45 * n * np.abs(A).max(axis=1)[:, None] * np.abs(X).max(axis=1)[None, :]
    assert (np.abs(full - W) <= bound).all()
