"""CPU FP64 oracle for the oap Arnoldi hot path (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package; the shipped library never does.  The
numerical code is ``oracle.c`` (built into ``liboracle.so`` by the Makefile
next to it); this module is a thin numpy/ctypes front end whose functions use
the reference's matrix convention: row-major, element (column c, row r) at
``c + r * columns``, complex values as numpy complex128 arrays.
"""

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

WHICH = {"LM": 0, "LR": 1, "LI": 2, "SM": 3, "SR": 4, "SI": 5}


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_magnitude.restype = C.c_double
        _LIB.orc_num_threads.restype = C.c_int
    return _LIB


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _split(a):
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return (np.ascontiguousarray(a.real, dtype=np.float64),
                np.ascontiguousarray(a.imag, dtype=np.float64))
    return np.ascontiguousarray(a, dtype=np.float64), None


def _join(re, im):
    return re if im is None else re + 1j * im


def dot_product(a, b):
    """C = A B (CuProceduresApi::dotProduct)."""
    a = np.asarray(a)
    b = np.asarray(b)
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    ar, ai = _split(a.astype(np.complex128) if cplx else a)
    br, bi = _split(b.astype(np.complex128) if cplx else b)
    orows, inner = a.shape
    ocols = b.shape[1]
    ore = np.zeros((orows, ocols))
    oim = np.zeros((orows, ocols)) if cplx else None
    lib().orc_dot_product(_p(ore), _p(oim), _p(ar), _p(ai), _p(br), _p(bi),
                          ocols, orows, inner)
    return _join(ore, oim)


def transpose(a, conj=False):
    a = np.asarray(a)
    ar, ai = _split(a)
    rows, cols = a.shape
    ore = np.zeros((cols, rows))
    oim = np.zeros((cols, rows)) if ai is not None else None
    lib().orc_transpose(_p(ore), _p(oim), _p(ar), _p(ai), cols, rows, int(conj))
    return _join(ore, oim)


def magnitude(x):
    xr, xi = _split(np.ravel(x))
    return lib().orc_magnitude(_p(xr), _p(xi), C.c_long(xr.size))


def matsum(x):
    xr, xi = _split(np.ravel(x))
    sre, sim = C.c_double(), C.c_double()
    lib().orc_sum(_p(xr), _p(xi), C.c_long(xr.size), C.byref(sre), C.byref(sim))
    return sre.value, sim.value


def tensor_product(p0, p1):
    p0 = np.asarray(p0)
    p1 = np.asarray(p1)
    cplx = np.iscomplexobj(p0) or np.iscomplexobj(p1)
    r0, c0 = p0.shape
    r1, c1 = p1.shape
    a_r, a_i = _split(p0.astype(np.complex128) if cplx else p0)
    b_r, b_i = _split(p1.astype(np.complex128) if cplx else p1)
    ore = np.zeros((r0 * r1, c0 * c1))
    oim = np.zeros_like(ore) if cplx else None
    lib().orc_tensor_product(_p(ore), _p(oim), _p(a_r), _p(a_i), c0, r0,
                             _p(b_r), _p(b_i), c1, r1)
    return _join(ore, oim)


def is_upper_triangular(a, tol=1e-3):
    a = np.asarray(a)
    ar, ai = _split(a)
    return bool(lib().orc_is_upper_triangular(_p(ar), _p(ai), a.shape[0],
                                              C.c_double(tol)))


def qr_givens(a):
    a = np.asarray(a)
    n = a.shape[0]
    ar, ai = _split(a)
    cplx = ai is not None
    qr, rr = np.zeros((n, n)), np.zeros((n, n))
    qi = np.zeros((n, n)) if cplx else None
    ri = np.zeros((n, n)) if cplx else None
    lib().orc_qr_givens(_p(qr), _p(qi), _p(rr), _p(ri), _p(ar), _p(ai), n)
    return _join(qr, qi), _join(rr, ri)


def qr_householder(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    q, r = np.zeros((n, n)), np.zeros((n, n))
    lib().orc_qr_householder(_p(q), _p(r), _p(a), n)
    return q, r


def calc_triangular_h(h, count=600, tol=1e-3):
    h = np.array(h)
    n = h.shape[0]
    hr, hi = _split(h)
    hr, hi = hr.copy(), (hi.copy() if hi is not None else None)
    qr = np.zeros((n, n))
    qi = np.zeros((n, n)) if hi is not None else None
    it = lib().orc_calc_triangular_h(_p(hr), _p(hi), _p(qr), _p(qi), n, count,
                                     C.c_double(tol))
    return _join(hr, hi), _join(qr, qi), it


def eigvals_dense(a):
    a = np.asarray(a)
    n = a.shape[0]
    ar, ai = _split(a)
    wr, wi = np.zeros(n), np.zeros(n)
    rc = lib().orc_eigvals_dense(_p(ar), _p(ai), n, _p(wr), _p(wi))
    assert rc == 0
    return wr + 1j * wi


def schur_hessenberg(h):
    """Complex Schur form T = Z^H H Z of a Hessenberg matrix (numpy layout)."""
    h = np.asarray(h, dtype=np.complex128)
    m = h.shape[0]
    hc = np.asfortranarray(h)
    hr = np.ascontiguousarray(hc.real.ravel(order="F"))
    hi = np.ascontiguousarray(hc.imag.ravel(order="F"))
    tr, ti, zr, zi = (np.zeros(m * m) for _ in range(4))
    rc = lib().orc_schur_split(_p(hr), _p(hi), m, _p(tr), _p(ti), _p(zr), _p(zi))
    assert rc == 0
    t = (tr + 1j * ti).reshape(m, m, order="F")
    z = (zr + 1j * zi).reshape(m, m, order="F")
    return t, z


def matvec(a, x):
    a = np.asarray(a)
    n = a.shape[0]
    ar, ai = _split(a)
    xc = np.asarray(x, dtype=np.complex128)
    xr, xi = _split(xc)
    yr, yi = np.zeros(n), np.zeros(n)
    lib().orc_matvec(n, _p(ar), _p(ai), _p(xr), _p(xi), _p(yr), _p(yi))
    return yr + 1j * yi


def iram(a, k, m, which="LM", tol=1e-10, maxit=300, rho=1.0 / 3.14,
         v0=None, seed=0):
    """Textbook FP64 IRAM on a dense operator (see oracle.c: orc_iram).

    Returns dict(eigenvalues, vectors (k x n), residuals, restarts, matvecs,
    converged, dgks, rc)."""
    ar, ai = _split(np.asarray(a))
    return iram_planes(ar, ai, k, m, which, tol, maxit, rho, v0, seed)


def iram_planes(are, aim, k, m, which="LM", tol=1e-10, maxit=300, rho=1.0 / 3.14, v0=None, seed=0):
    """iram() on an operator given as its split FP64 planes (C-contiguous
    numpy arrays, aim None for a real operator), without forming the complex
    matrix: the form for large n (one n = 16384 complex operator is 4 GiB)."""
    n = are.shape[0]
    assert are.dtype == np.float64 and are.flags.c_contiguous
    assert aim is None or (aim.dtype == np.float64 and aim.flags.c_contiguous)
    if v0 is None:
        v0 = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    v0r, v0i = _split(np.asarray(v0))
    evr, evi = np.zeros(k), np.zeros(k)
    xr, xi = np.zeros(k * n), np.zeros(k * n)
    res = np.zeros(k)
    stats = (C.c_int * 4)()
    rc = lib().orc_iram(n, _p(are), _p(aim), m, k, WHICH[which], C.c_double(tol),
                        maxit, C.c_double(rho), _p(v0r), _p(v0i), _p(evr),
                        _p(evi), _p(xr), _p(xi), _p(res), stats)
    return {"eigenvalues": evr + 1j * evi,
            "vectors": (xr + 1j * xi).reshape(k, n),
            "residuals": res, "restarts": stats[0], "matvecs": stats[1],
            "converged": bool(stats[2]), "dgks": stats[3], "rc": rc}


def iram_reference(a, k, m, which="LM", maxit=300, rho=1.0 / 3.14, blimit=1e-5, v0=None, seed=0):
    """The reference's CuHArnoldi::execute restated as written, for a real
    operator (see oracle.c: orc_iram_reference): V^T projections over all m
    basis columns, the 1e-3 triangular gate of the unshifted QR, the
    reference's shift accumulation and residual-update indices, CHECK_INTERNAL
    stopping, Krylov-column eigenvectors.

    Returns dict(eigenvalues, vectors (k x n), residuals, restarts, matvecs,
    stopped (1: CHECK_INTERNAL ended it, 0: maxit), triangular_steps, rc)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    if v0 is None:
        v0 = np.random.default_rng(seed).uniform(-1.0, 1.0, n)
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    evr, evi = np.zeros(k), np.zeros(k)
    x = np.zeros(k * n)
    res = np.zeros(k)
    stats = (C.c_int * 4)()
    rc = lib().orc_iram_reference(n, _p(a), m, k, WHICH[which], maxit, C.c_double(rho), C.c_double(blimit),
                                  _p(v0), _p(evr), _p(evi), _p(x), _p(res), stats)
    return {"eigenvalues": evr + 1j * evi, "vectors": x.reshape(k, n), "residuals": res,
            "restarts": stats[0], "matvecs": stats[1], "stopped": stats[2], "triangular_steps": stats[3],
            "rc": rc}


def qr_givens_reference(a):
    """The reference's Givens QR as the reference-faithful IRAM restates it
    (oracle.c: orc_qrgr_ref): rotations only where the input entry is
    outside (-1e-5, 1e-5), r = sqrtf(c^2 + s^2), the output buffers as the
    reference's pointer ping-pong leaves them."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    q, r = np.zeros((n, n)), np.zeros((n, n))
    lib().orc_qrgr_ref(_p(a), _p(q), _p(r), n)
    return q, r


def match_eigenvalues(ev, ref):
    """Largest |ev_i - ref_j| / max|ref| over a one-to-one matching of two
    eigenvalue lists (each value of `ev` to the nearest unused one of `ref`,
    taken in `ref`'s order: the wanted-set order of SortLargestValues,
    ArnoldiPackage/ArnoldiUtils.cpp:24-28, when both lists are sorted so)."""
    ev = list(np.asarray(ev, dtype=np.complex128))
    ref = np.asarray(ref, dtype=np.complex128)
    scale = np.abs(ref).max() if ref.size else 1.0
    worst = 0.0
    for r in ref:
        j = int(np.argmin([abs(e - r) for e in ev]))
        worst = max(worst, abs(ev[j] - r) / scale)
        ev.pop(j)
    return worst


def num_threads():
    return lib().orc_num_threads()


# --------------------------------------------------------------------------
# The reference's own host implementation (oracle/_ref/libref.so, built from
# the reference sources by oracle/ref/build_ref.sh where they are present):
# used only to check this oracle against the reference's code.
_REF = None


def ref():
    """ctypes handle of oracle/_ref/libref.so, or None when it is not built."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref.so")
        if not os.path.exists(path):
            return None
        _REF = C.CDLL(path)
    return _REF


def _planes(a):
    a = np.asarray(a)
    re = np.ascontiguousarray(a.real, dtype=np.float64)
    im = np.ascontiguousarray(a.imag, dtype=np.float64) if np.iscomplexobj(a) else None
    return re, im


def ref_dot_product(a, b):
    """output = a b by HostProcedures::dotProduct (a: M x K, b: K x N as numpy (rows, cols))."""
    M, K = a.shape
    N = b.shape[1]
    ar, ai = _planes(a)
    br, bi = _planes(b)
    cplx = ai is not None or bi is not None
    if cplx:
        ai = ai if ai is not None else np.zeros_like(ar)
        bi = bi if bi is not None else np.zeros_like(br)
    o_re = np.zeros((M, N))
    o_im = np.zeros((M, N)) if cplx else None
    ref().ref_dot_product(M, K, N, _p(ar), _p(ai), _p(br), _p(bi), _p(o_re), _p(o_im))
    return o_re + 1j * o_im if cplx else o_re


def ref_transpose(a):
    rows, cols = a.shape
    ar, ai = _planes(a)
    o_re = np.zeros((cols, rows))
    o_im = np.zeros((cols, rows)) if ai is not None else None
    ref().ref_transpose(cols, rows, _p(ar), _p(ai), _p(o_re), _p(o_im))
    return o_re + 1j * o_im if ai is not None else o_re


def ref_substract(a, b):
    rows, cols = a.shape
    ar, ai = _planes(a)
    br, bi = _planes(b)
    o_re = np.zeros((rows, cols))
    o_im = np.zeros((rows, cols)) if ai is not None else None
    ref().ref_substract(cols, rows, _p(ar), _p(ai), _p(br), _p(bi), _p(o_re), _p(o_im))
    return o_re + 1j * o_im if ai is not None else o_re


def ref_sum(a):
    rows, cols = a.shape
    ar, ai = _planes(a)
    sre, sim = C.c_double(), C.c_double()
    ref().ref_sum(cols, rows, _p(ar), _p(ai), C.byref(sre), C.byref(sim))
    return sre.value, sim.value


def ref_qr_householder(a):
    n = a.shape[0]
    q, r = np.zeros((n, n)), np.zeros((n, n))
    rc = ref().ref_qr_householder(n, _p(np.ascontiguousarray(a, dtype=np.float64)), _p(q), _p(r))
    if rc:
        raise ValueError("n * n > 1024")
    return q, r


def ref_set_vector(V, column, x, length):
    V = np.ascontiguousarray(V, dtype=np.float64).copy()
    rows, cols = V.shape
    ref().ref_set_vector(cols, rows, _p(V), column, _p(np.ascontiguousarray(x, dtype=np.float64)), length)
    return V


def ref_write_matrix(path, a):
    """The reference's oap::host::WriteMatrix of a numpy matrix (rows, columns)."""
    rows, cols = a.shape
    ar, ai = _planes(a)
    rc = ref().ref_write_matrix(str(path).encode(), cols, rows, _p(ar), _p(ai))
    if rc:
        raise OSError("WriteMatrix failed")

