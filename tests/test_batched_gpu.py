"""Batched persistent solver (oapb_arnoldi_solve_batched) against numpy /
the oracle and against the single-problem solver."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402
from gpu_util import planes, zeros, host  # noqa: E402

TOL = 1e-10


def complex_problem(n, rng, nplant=4):
    s = 1.0 / np.sqrt(2.0 * n)
    A = rng.normal(scale=s, size=(n, n)) + 1j * rng.normal(scale=s, size=(n, n))
    pos = rng.choice(n, nplant, replace=False)
    A[pos, pos] += 4.0
    return A


def top_lm(A, k):
    w = np.linalg.eigvals(A)
    return w[np.argsort(-np.abs(w))][:k]


def test_batched_uneven_complex():
    rng = np.random.default_rng(77)
    sizes = list(rng.integers(32, 257, size=40)) + [20, 25, 512]
    As = [complex_problem(int(n), rng) for n in sizes]
    mats = [planes(A) for A in As]
    vecs = [zeros((A.shape[0], 4), True) for A in As]
    ev, res, st, stats, rc = B.solve_batched(mats, 4, hdim=24, vectors=vecs)
    assert rc == B.OK, (st, res.max())
    assert (st == B.OK).all()
    assert res.max() <= TOL
    assert stats["converged"] == len(As) and stats["ctas"] >= 1
    for i, A in enumerate(As):
        want = top_lm(A, 4)
        for lam in want:
            assert np.min(np.abs(ev[i] - lam)) < 1e-9 * abs(lam), (i, A.shape[0])
        X = host(*vecs[i])
        for q in range(4):
            x = X[:, q]
            assert np.linalg.norm(A @ x - ev[i, q] * x) <= TOL * np.abs(ev[i]).max() * 1.01


def test_batched_real_symmetric_matches_single_solver():
    rng = np.random.default_rng(5)
    As = []
    for n in (64, 100, 150):
        Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
        lam = np.linspace(1.0, 0.01, n)
        lam[:3] = [5.0, 4.0, 3.0]
        As.append((Q * lam) @ Q.T)
    mats = [planes(A, False) for A in As]
    ev, res, st, stats, rc = B.solve_batched(mats, 3, hdim=16, sort="LR")
    assert rc == B.OK and res.max() <= TOL
    for i, A in enumerate(As):
        assert np.allclose(ev[i].real, [5.0, 4.0, 3.0], rtol=1e-10)
        assert np.abs(ev[i].imag).max() == 0
        s = B.Arnoldi(A.shape[0], 16, 3, sort="LR")
        s.set_operator(*planes(A, False))
        e1, r1, _ = s.solve()
        assert np.allclose(np.sort(np.array(e1).real), np.sort(ev[i].real), rtol=1e-12)


def test_batched_against_oracle_iram():
    rng = np.random.default_rng(9)
    As = [complex_problem(n, rng) for n in (48, 96, 130)]
    ev, res, st, stats, rc = B.solve_batched([planes(A) for A in As], 4, hdim=20)
    assert rc == B.OK
    for i, A in enumerate(As):
        o = O.iram(A, 4, 20, which="LM", tol=TOL, seed=i)
        for lam in o["eigenvalues"]:
            assert np.min(np.abs(ev[i] - lam)) < 1e-9 * abs(lam)


def test_batched_rejects_bad_arguments():
    A = complex_problem(40, np.random.default_rng(1))
    with pytest.raises(B.OapbError):
        B.solve_batched([planes(A)], 4, hdim=40)     # hdim > 32
    with pytest.raises(B.OapbError):
        B.solve_batched([planes(A)], 8, hdim=8)      # wanted >= hdim


def test_batched_launch_variants_agree():
    # the autotuner's launch variants (threads per CTA x CTAs per SM: 256 x 1,
    # 128 x 2, 256 x 2, 128 x 4, 64 x 8; forced with autotune = 2 + v) solve
    # every problem to the default variant's eigenvalues; the tuned call
    # reports the variant it chose
    rng = np.random.default_rng(5)
    sizes = list(rng.integers(24, 300, size=60))
    As = [complex_problem(int(n), rng) for n in sizes]
    mats = [planes(A) for A in As]
    ev0, res0, st0, stats0, rc0 = B.solve_batched(mats, 4, hdim=20, autotune=False)
    assert rc0 == B.OK and stats0["variant"] == 0 and stats0["threads"] == 256
    for v, threads in enumerate((256, 128, 256, 128, 64)):
        ev, res, st, stats, rc = B.solve_batched(mats, 4, hdim=20, autotune=2 + v)
        assert rc == B.OK and stats["variant"] == v and stats["threads"] == threads
        assert res.max() <= TOL
        scale = np.abs(ev0).max(axis=1, keepdims=True)
        assert (np.abs(ev - ev0) <= 1e-10 * scale).all(), v
    ev, res, st, stats, rc = B.solve_batched(mats, 4, hdim=20, autotune=True)
    assert rc == B.OK and 0 <= stats["variant"] < 5 and res.max() <= TOL
    ev2, _, _, stats2, _ = B.solve_batched(mats, 4, hdim=20, autotune=True)
    assert stats2["variant"] == stats["variant"]  # cached per shape
    assert (np.abs(ev2 - ev0) <= 1e-10 * np.abs(ev0).max(axis=1, keepdims=True)).all()
