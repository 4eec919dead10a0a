"""Failure paths of the solver on the GPU, made on the host or by a bounded
device wait that nothing releases: a user callback that fails, a callback
that writes NaN, a restart budget that runs out, and the bounded mbarrier
wait of the tensor-core kernels running out.  The reference aborts the
process on every CUDA error (oapCuda/KernelExecutor.h:34-41); here each case
ends in a status code and the handle (and the CUDA context) stay usable.
Nothing in these tests faults, traps or hangs the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402
from gpu_util import planes, planted_symmetric  # noqa: E402

TOL = 1e-10


def ptr_tensor(ptr, n):
    """A torch view of n FP64 values at a raw device pointer."""
    class _A:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                    "version": 3, "strides": None}
    return torch.as_tensor(_A(), device="cuda")


def callback(a, n, fail_after=None, rc=7, nan_after=None):
    """w = A v on the solver's stream; from call `fail_after` on return `rc`,
    from call `nan_after` on write NaN into w."""
    calls = []

    def mv(w, v, typ, stream):
        calls.append(typ)
        if fail_after is not None and len(calls) > fail_after:
            return rc
        st = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
        with torch.cuda.stream(st):
            out = ptr_tensor(w.re, n)
            torch.mv(a, ptr_tensor(v.re, n), out=out)
            if nan_after is not None and len(calls) > nan_after:
                out[n // 2] = float("nan")
        return 0
    return mv, calls


def good_solve(s, a, n, lam, k):
    mv, _ = callback(a, n)
    s.set_callback(mv)
    ev, res, st = s.solve()
    assert st == B.OK and max(res) <= TOL
    assert np.allclose(np.sort(np.array(ev).real)[::-1], lam[:k], rtol=1e-10)


@pytest.mark.parametrize("fail_after", [0, 20])
def test_callback_error_returns_status(fail_after):
    # CuHArnoldiCallback's MultiplyFunc returning non-zero ends the solve with
    # OAPB_ERR_CALLBACK (first call, and in the middle of the factorization);
    # the same handle then solves with a working callback
    n, k = 300, 5
    A, lam = planted_symmetric(n, seed=4)
    a = planes(A, False)[0]
    s = B.Arnoldi(n, 32, k, seed=3)
    mv, calls = callback(a, n, fail_after=fail_after)
    s.set_callback(mv)
    with pytest.raises(B.OapbError) as e:
        s.solve()
    assert e.value.status == B.ERR_CALLBACK
    assert len(calls) == fail_after + 1  # the solve stopped at the failing call
    torch.cuda.synchronize()
    good_solve(s, a, n, lam, k)
    s.close()


def test_callback_exception_is_reported():
    # a Python exception inside the callback becomes OAPB_ERR_CALLBACK and is
    # chained to the raised error
    n, k = 200, 3
    A, lam = planted_symmetric(n, seed=5)
    a = planes(A, False)[0]
    s = B.Arnoldi(n, 20, k, seed=3)

    def bad(w, v, typ, stream):
        raise ValueError("operator unavailable")

    s.set_callback(bad)
    with pytest.raises(B.OapbError) as e:
        s.solve()
    assert e.value.status == B.ERR_CALLBACK
    assert isinstance(e.value.__cause__, ValueError)
    good_solve(s, a, n, lam, k)
    s.close()


@pytest.mark.parametrize("nan_after", [0, 10])
def test_callback_nan_is_not_converged(nan_after):
    # a callback that writes NaN into w: the solve ends with
    # OAPB_ERR_NONFINITE (never OK, never a hang: every device loop is
    # bounded) and the handle solves again afterwards
    n, k = 300, 5
    A, lam = planted_symmetric(n, seed=4)
    a = planes(A, False)[0]
    s = B.Arnoldi(n, 32, k, seed=3)
    mv, calls = callback(a, n, nan_after=nan_after)
    s.set_callback(mv)
    with pytest.raises(B.OapbError) as e:
        s.solve()
    assert e.value.status == B.ERR_NONFINITE, B.status_string(e.value.status)
    torch.cuda.synchronize()
    good_solve(s, a, n, lam, k)
    s.close()


def test_nan_operator_is_not_converged():
    # a dense operator holding a NaN: the same status, on the library's own
    # matvec
    n, k = 256, 4
    A, lam = planted_symmetric(n, seed=7)
    A[17, 40] = np.nan
    s = B.Arnoldi(n, 24, k, seed=1)
    s.set_operator(*planes(A, False))
    with pytest.raises(B.OapbError) as e:
        s.solve()
    assert e.value.status == B.ERR_NONFINITE
    s.close()


def test_restart_budget_runs_out():
    # a restart budget too small for a clustered spectrum: OAPB_NOT_CONVERGED
    # with the best pairs in the outputs (finite, residuals above the goal);
    # the well-separated spectrum reaches the goal within the default budget
    n, k = 256, 4
    A, lam = planted_symmetric(n, seed=6, lo_exp=-0.05)
    for budget in (0, 2):
        s = B.Arnoldi(n, 12, k, max_restarts=budget, seed=1)
        s.set_operator(*planes(A, False))
        ev, res, st = s.solve(allow_not_converged=True)
        assert st == B.NOT_CONVERGED, (budget, st)
        assert np.all(np.isfinite(res)) and np.all(np.isfinite(np.array(ev)))
        assert s.stats()["restarts"] <= budget and max(res) > TOL
        s.close()
    A, lam = planted_symmetric(n, seed=6)
    s = B.Arnoldi(n, 12, k, seed=1)
    s.set_operator(*planes(A, False))
    ev, res, st = s.solve()
    assert st == B.OK and max(res) <= TOL
    s.close()


@pytest.mark.parametrize("limit_us", [1000, 50000])
def test_bounded_wait_runs_out(limit_us):
    # the bounded mbarrier wait of the tensor-core kernels: with no arrival
    # it gives up after its limit, the kernel returns, the call reports
    # OAPB_ERR_TIMEOUT, and the context keeps working (a second self-test
    # whose barrier is released completes)
    torch.cuda.synchronize()
    st, timed_out = B.selftest_bounded_wait(limit_us, arrive=False)
    assert st == B.ERR_TIMEOUT and timed_out == 1
    st, timed_out = B.selftest_bounded_wait(limit_us, arrive=True)
    assert st == B.OK and timed_out == 0
    x = torch.arange(10, dtype=torch.float64, device="cuda")
    assert float(x.sum()) == 45.0


def test_bounded_wait_rejects_bad_limits():
    for lim in (0, 2000000):
        st, _ = B.selftest_bounded_wait(lim)
        assert st == B.ERR_ARG
