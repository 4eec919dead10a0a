"""The allocation-free Givens QR entry point (oapb_qr_givens_noalloc).

Callers that cannot allocate device memory (a stream capture that forbids
allocations, allocator hooks, fixed memory budgets) use this variant; its
workspace is a static device array of the library (n <= 128).  The test
calls it through the C ABI and checks it against oapb_qr_givens on two calls
in a row with different inputs: the shared workspace keeps the previous
call's contents, and the results must not depend on them.  This file is
collected last so that a run stopping at the first failure has run every
other test first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def qr(fn, A):
    n = A.shape[0]
    a = (dev(A.real), dev(A.imag))
    q = (torch.zeros(n, n, dtype=torch.float64, device="cuda"),
         torch.zeros(n, n, dtype=torch.float64, device="cuda"))
    r = (torch.zeros(n, n, dtype=torch.float64, device="cuda"),
         torch.zeros(n, n, dtype=torch.float64, device="cuda"))
    st = fn(C.byref(B.mat(*q)), C.byref(B.mat(*r)), C.byref(B.mat(*a)), None)
    assert st == B.OK, B.status_string(st)
    torch.cuda.synchronize()
    return (q[0].cpu().numpy() + 1j * q[1].cpu().numpy(),
            r[0].cpu().numpy() + 1j * r[1].cpu().numpy())


def test_noalloc_qr_matches_allocating_entry_point_twice():
    L = B.lib()
    rng = np.random.default_rng(2024)
    # two different sizes in a row: the second call reuses the workspace
    for n in (120, 37):
        A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        Qn, Rn = qr(L.oapb_qr_givens_noalloc, A)
        Qa, Ra = qr(L.oapb_qr_givens, A)
        tol = 1e-12 * max(1.0, np.abs(Ra).max())
        assert np.abs(Qn - Qa).max() <= tol
        assert np.abs(Rn - Ra).max() <= tol
        assert np.abs(Qn @ Rn - A).max() <= 1e-12 * n * np.abs(A).max()


def test_noalloc_qr_rejects_sizes_beyond_its_workspace():
    L = B.lib()
    n = 129
    z = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    m = B.mat(z)
    assert L.oapb_qr_givens_noalloc(C.byref(m), C.byref(m), C.byref(m), None) == B.ERR_ARG
