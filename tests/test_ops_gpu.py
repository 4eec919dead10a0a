"""Operator surface (oap::CuProceduresApi) on the GPU through the C ABI,
against the CPU oracle and the reference's fixtures."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402
from gpu_util import dev, host, planes, zeros  # noqa: E402

L = B.lib()
S = None  # legacy default stream
rng = np.random.default_rng(1234)


def cm(shape):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def M(x):
    return np.array(x["re"]).reshape(x["rows"], x["columns"])


def run(fn, *args):
    st = fn(*args)
    assert st == B.OK, B.status_string(st)
    torch.cuda.synchronize()


@pytest.mark.parametrize("shape", [(37, 29, 13), (5, 300, 1), (512, 512, 1), (64, 64, 64)])
@pytest.mark.parametrize("cplx", [False, True])
def test_dot_product(shape, cplx):
    mr, k, nc = shape
    A = cm((mr, k)) if cplx else rng.normal(size=(mr, k))
    Bm = cm((k, nc)) if cplx else rng.normal(size=(k, nc))
    a, b = planes(A), planes(Bm)
    o = zeros((mr, nc), cplx)
    run(L.oapb_dot_product, C.byref(B.mat(*o)), C.byref(B.mat(*a)), C.byref(B.mat(*b)), S)
    ref = O.dot_product(A, Bm)
    assert np.abs(host(*o) - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * k


@pytest.mark.parametrize("cplx", [False, True])
def test_transpose_and_conjugate(cplx):
    A = cm((70, 45)) if cplx else rng.normal(size=(70, 45))
    a = planes(A)
    for conj, fn in ((False, L.oapb_transpose), (True, L.oapb_conjugate_transpose)):
        o = zeros((45, 70), cplx)
        run(fn, C.byref(B.mat(*o)), C.byref(B.mat(*a)), S)
        assert np.array_equal(host(*o), O.transpose(A, conj=conj))


def test_magnitude_and_sum():
    for A in (cm((3000, 7)), rng.normal(size=(1, 100000))):
        a = planes(A)
        out = C.c_double()
        run(L.oapb_magnitude, C.byref(out), C.byref(B.mat(*a)), S)
        assert abs(out.value - O.magnitude(A)) <= 1e-12 * O.magnitude(A)
        sr, si = C.c_double(), C.c_double()
        run(L.oapb_sum, C.byref(sr), C.byref(si), C.byref(B.mat(*a)), S)
        er, ei = O.matsum(A)
        # summation-order rounding: within 1e-14 of sum |a| (the sums
        # themselves can be near zero)
        sa_re = float(np.abs(np.real(A)).sum())
        sa_im = float(np.abs(np.imag(A)).sum())
        assert abs(sr.value - er) <= 1e-14 * sa_re and abs(si.value - ei) <= 1e-14 * max(sa_im, 1e-300)


def test_tensor_product():
    P0, P1 = rng.normal(size=(3, 4)), rng.normal(size=(5, 2))
    o = zeros((15, 8), False)
    p0, p1 = planes(P0), planes(P1)   # keep the device buffers alive
    run(L.oapb_tensor_product, C.byref(B.mat(*o)), C.byref(B.mat(*p0)), C.byref(B.mat(*p1)), S)
    assert np.array_equal(host(*o), O.tensor_product(P0, P1))


def test_elementwise_beyond_one_block():
    # the reference's add indexes threadIdx only (wrong past one block)
    X, Y = cm((4096, 3)), cm((4096, 3))
    x, y = planes(X), planes(Y)
    for fn, ref in ((L.oapb_add, X + Y), (L.oapb_substract, X - Y)):
        o = zeros((4096, 3), True)
        run(fn, C.byref(B.mat(*o)), C.byref(B.mat(*x)), C.byref(B.mat(*y)), S)
        assert np.array_equal(host(*o), ref)
    o = zeros((4096, 3), True)
    run(L.oapb_multiply_constant, C.byref(B.mat(*o)), C.byref(B.mat(*x)), 0.5, -2.0, S)
    assert np.allclose(host(*o), O.dot_product(X.reshape(-1, 1), np.array([[0.5 - 2.0j]])).reshape(4096, 3))
    run(L.oapb_multiply_re_constant, C.byref(B.mat(*o)), C.byref(B.mat(*x)), 3.0, S)
    assert np.allclose(host(*o), 3.0 * X)


def test_set_get_vector_identity_diagonal():
    V = zeros((50, 8), True)
    v = planes(cm(50))
    run(L.oapb_set_vector, C.byref(B.mat(*V)), 3, C.byref(B.mat(*v)), 40, S)
    ref = np.zeros((50, 8), complex)
    hv = host(*v)
    ref[:40, 3] = hv[:40]
    assert np.array_equal(host(*V), ref)
    w = zeros(50, True)
    run(L.oapb_get_vector, C.byref(B.mat(*w)), 50, C.byref(B.mat(*V)), 3, S)
    assert np.array_equal(host(*w), ref[:, 3])
    Mx = zeros((6, 6), True)
    run(L.oapb_set_identity, C.byref(B.mat(*Mx)), S)
    assert np.array_equal(host(*Mx), np.eye(6))
    run(L.oapb_set_diagonal, C.byref(B.mat(*Mx)), 2.0, -1.0, S)
    assert np.array_equal(host(*Mx), (2 - 1j) * np.eye(6))
    run(L.oapb_set_zero_matrix, C.byref(B.mat(*Mx)), S)
    assert not host(*Mx).any()


def _qr(fn, A, cplx):
    n = A.shape[0]
    a = planes(A, cplx)
    q, r = zeros((n, n), cplx), zeros((n, n), cplx)
    run(fn, C.byref(B.mat(*q)), C.byref(B.mat(*r)), C.byref(B.mat(*a)), S)
    return host(*q), host(*r)


def test_qr_givens_reference_samples(golden):
    for s in golden["qr_samples"] + golden["host_qr_samples"]:
        A = M(s["matrix"])
        Q, R = _qr(L.oapb_qr_givens, A, False)
        Qo, Ro = O.qr_givens(A)
        assert np.abs(Q - Qo).max() < 1e-12 and np.abs(R - Ro).max() < 1e-12 * np.abs(Ro).max()
        assert np.abs(np.abs(Q) - np.abs(M(s["q"]))).max() < 1e-4


@pytest.mark.parametrize("n", [3, 17, 64, 100])
def test_qr_givens_complex(n):
    A = cm((n, n))
    Q, R = _qr(L.oapb_qr_givens, A, True)
    Qo, Ro = O.qr_givens(A)
    assert np.abs(Q - Qo).max() < 1e-10
    assert np.abs(R - Ro).max() < 1e-10 * np.abs(Ro).max()
    assert np.abs(Q @ R - A).max() < 1e-12 * n * np.abs(A).max()


def test_qr_householder(golden):
    c = golden["small_qr"]["hessenberg4"]
    cases = [np.array(c["h"]).reshape(4, 4) - c["shift"] * np.eye(4),
             np.array(golden["small_qr"]["sym3"]["a"], float).reshape(3, 3),
             rng.normal(size=(40, 40))]
    for A in cases:
        Q, R = _qr(L.oapb_qr_householder, A, False)
        Qo, Ro = O.qr_householder(A)
        assert np.abs(Q - Qo).max() < 1e-12 and np.abs(R - Ro).max() < 1e-11 * np.abs(Ro).max()
    Q, R = _qr(L.oapb_qr_householder, cases[0], False)
    assert np.abs(np.abs(Q) - np.abs(np.array(c["q_expected"]).reshape(4, 4))).max() < 1e-3


def test_is_upper_triangular():
    T = np.triu(rng.normal(size=(9, 9)))
    T[4, 3] = 5e-4
    out = C.c_int()
    t = planes(T)
    run(L.oapb_is_upper_triangular, C.byref(out), C.byref(B.mat(*t)), 1e-3, S)
    assert out.value == 1 == int(O.is_upper_triangular(T))
    T[4, 3] = 2e-3
    t = planes(T)
    run(L.oapb_is_upper_triangular, C.byref(out), C.byref(B.mat(*t)), 1e-3, S)
    assert out.value == 0 == int(O.is_upper_triangular(T))


def test_calc_triangular_h_schur_fixtures(golden):
    for s in golden["schur"][:2]:
        A = M(s["matrix"])
        h = planes(A, False)
        q = zeros(A.shape, False)
        it = C.c_uint32()
        run(L.oapb_calc_triangular_h, C.byref(B.mat(*h)), C.byref(B.mat(*q)), 600, C.byref(it), S)
        To, Qo, ito = O.calc_triangular_h(A)
        assert it.value == ito
        assert np.abs(host(*h) - To).max() < 1e-8 * np.abs(To).max()
        assert np.abs(host(*q) - Qo).max() < 1e-8
