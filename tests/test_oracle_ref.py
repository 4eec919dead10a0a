"""The oracle checked against the reference's own host code.

oracle/_ref/libref.so is the reference's operator surface (oapMatrixCpu's
HostProcedures over oapMatrix / oapMath / oapUtils) compiled from the
reference sources by oracle/ref/build_ref.sh; these CPU tests run the same
seeded inputs through it and through the oracle's restatement.  They are
skipped where the reference build is absent."""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref/libref.so not built")


def rnd(rng, shape, cplx):
    a = rng.normal(size=shape)
    return a + 1j * rng.normal(size=shape) if cplx else a


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("M,K,N", [(4, 4, 4), (7, 5, 3), (16, 16, 1), (1, 9, 6)])
def test_dot_product_matches_reference(cplx, M, K, N):
    rng = np.random.default_rng(M * 100 + K * 10 + N)
    a, b = rnd(rng, (M, K), cplx), rnd(rng, (K, N), cplx)
    ref = O.ref_dot_product(a, b)
    mine = O.dot_product(a, b)
    assert np.allclose(mine, ref, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("rows,cols", [(3, 5), (8, 8), (1, 7)])
def test_transpose_matches_reference(cplx, rows, cols):
    rng = np.random.default_rng(rows * 10 + cols)
    a = rnd(rng, (rows, cols), cplx)
    assert np.array_equal(O.transpose(a), O.ref_transpose(a))


@pytest.mark.parametrize("cplx", [False, True])
def test_sum_and_substract_match_reference(cplx):
    rng = np.random.default_rng(5)
    a, b = rnd(rng, (6, 9), cplx), rnd(rng, (6, 9), cplx)
    sre, sim = O.ref_sum(a)
    mre, mim = O.matsum(a)
    assert abs(complex(mre, mim) - complex(sre, sim)) <= 1e-12 * np.abs(a).sum()
    assert np.array_equal(O.ref_substract(a, b), a - b)


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32])
def test_householder_qr_matches_reference(n):
    # the reference's reflector norms use sqrtf (CuQRProcedures_HT.h:97), the
    # oracle FP64 sqrt: same reflectors, factors equal to FP32 rounding
    rng = np.random.default_rng(n)
    a = rng.normal(size=(n, n))
    q_ref, r_ref = O.ref_qr_householder(a)
    q, r = O.qr_householder(a)
    assert np.allclose(q @ r, a, atol=1e-12)
    assert np.abs(q - q_ref).max() <= 1e-6
    assert np.abs(r - r_ref).max() <= 1e-6 * np.abs(r).max()


def test_set_vector_matches_reference():
    rng = np.random.default_rng(9)
    V = rng.normal(size=(10, 4))
    x = rng.normal(size=10)
    out = O.ref_set_vector(V, 2, x, 7)
    exp = V.copy()
    exp[:7, 2] = x[:7]
    assert np.array_equal(out, exp)
