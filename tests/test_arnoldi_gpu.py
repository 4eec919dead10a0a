"""The implicitly restarted Arnoldi solver on the GPU through the C ABI,
against the CPU oracle, known spectra and the reference's fixtures."""
import ctypes as C

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402
from gpu_util import planes, planted_complex, planted_symmetric, zeros, host  # noqa: E402

TOL = 1e-10


def solve(A, k, m, sort="LM", precision=B.PREC_FP64, seed=1, vectors=False, **kw):
    n = A.shape[0]
    cplx = np.iscomplexobj(A)
    s = B.Arnoldi(n, m, k, is_complex=cplx, sort=sort, precision=precision, seed=seed, **kw)
    a = planes(A, cplx)
    s.set_operator(*a)
    vec = zeros((n, k), cplx) if vectors else None
    ev, res, st = s.solve(vectors=vec)
    out = {"ev": np.array(ev), "res": np.array(res), "stats": s.stats(), "solver": s}
    if vectors:
        out["x"] = host(*vec)
    return out


def test_planted_symmetric_n256():
    # the reference's CPU-sized case: n=256 float64, lambda 1 .. 1e-3, top-5 LM, m=32
    A, lam = planted_symmetric(256, seed=0)
    r = solve(A, 5, 32, vectors=True)
    assert np.allclose(np.sort(r["ev"].real)[::-1], lam[:5], rtol=1e-10, atol=0)
    assert np.abs(r["ev"].imag).max() == 0
    assert r["res"].max() <= TOL
    # eigenvectors: residual recomputed on the host in FP64
    X = r["x"]
    for q in range(5):
        x = X[:, q]
        assert abs(np.linalg.norm(x) - 1) < 1e-12
        assert np.linalg.norm(A @ x - r["ev"][q] * x) <= TOL
    # against the oracle on the same start vector
    o = O.iram(A, 5, 32, which="LM", tol=TOL, v0=B.start_vector(256, 1))
    assert np.allclose(np.sort(o["eigenvalues"].real), np.sort(r["ev"].real), rtol=1e-12)


@pytest.mark.parametrize("m", [24, 40])
def test_real_symmetric_takes_tridiagonal_path(m):
    # a real symmetric operator: the restart loop's small eigensolves take the
    # symmetric tridiagonal QR (four warps for m <= 32, one above); eigenpairs
    # against the known spectrum and the host FP64 residuals
    A, lam = planted_symmetric(512, seed=4)
    r = solve(A, 6, m, vectors=True)
    assert r["stats"]["symtri"] > 0
    assert np.allclose(np.sort(r["ev"].real)[::-1], lam[:6], rtol=1e-10, atol=0)
    assert r["res"].max() <= TOL
    X = r["x"]
    for q in range(6):
        assert np.linalg.norm(A @ X[:, q] - r["ev"][q] * X[:, q]) <= TOL * lam[0]
    # a small non-symmetric perturbation keeps the general Schur path, and
    # its eigenvalues agree with numpy's for the perturbed operator
    rng = np.random.default_rng(9)
    P = A + 1e-6 * rng.normal(size=A.shape) / np.sqrt(512)
    rp = solve(P, 6, m)
    assert rp["stats"]["symtri"] == 0
    ref = np.linalg.eigvals(P)
    ref = ref[np.argsort(-np.abs(ref))][:6]
    assert np.allclose(np.sort(rp["ev"].real), np.sort(ref.real), rtol=1e-9, atol=1e-12)
    assert rp["res"].max() <= TOL


def test_complex_hermitian_takes_tridiagonal_path():
    # A = Q diag(lambda) Q^H with a complex unitary Q: the Arnoldi matrix is
    # Hermitian tridiagonal to rounding, reduced to a real symmetric one by
    # phases; eigenvalues against the known spectrum, host FP64 residuals
    n, k, m = 400, 6, 24
    rng = np.random.default_rng(21)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    lam = 10.0 ** (-2.0 * np.arange(n) / (n - 1))
    A = (Q * lam) @ Q.conj().T
    A = (A + A.conj().T) / 2
    r = solve(A, k, m, vectors=True)
    assert r["stats"]["symtri"] > 0
    assert np.allclose(np.sort(r["ev"].real)[::-1], lam[:k], rtol=1e-10, atol=0)
    assert np.abs(r["ev"].imag).max() <= 1e-12
    assert r["res"].max() <= TOL
    X = r["x"]
    for q in range(k):
        assert np.linalg.norm(A @ X[:, q] - r["ev"][q] * X[:, q]) <= TOL * lam[0]


@pytest.mark.parametrize("idx", range(4))
def test_reference_known_spectrum(golden, idx):
    # oapArnoldiPackageMatricesTests.cpp:244-266 (SortLargestReValues)
    c = golden["cmatrix"][idx]
    n = c["n"]
    A = np.array(c["re"]).reshape(n, n)
    r = solve(A, c["wanted"], c["hdim"], sort="LR")
    want = np.sort(c["eigenvalues"])[::-1][: c["wanted"]]
    assert np.allclose(r["ev"].real, want, rtol=1e-10)
    assert r["res"].max() <= TOL  # reference gate: 0.02 - 0.047 absolute
    for q in range(c["wanted"]):
        assert r["solver"].test_outcome(q) <= TOL


@pytest.mark.parametrize("n,k,m", [(512, 6, 30), (1024, 16, 64)])
def test_complex_nonhermitian(n, k, m):
    A = planted_complex(n, seed=n, nplant=k)
    r = solve(A, k, m, vectors=True)
    assert r["res"].max() <= TOL
    w = np.linalg.eigvals(A)
    w = w[np.argsort(-np.abs(w))][:k]
    for lam in w:
        assert np.min(np.abs(r["ev"] - lam)) < 1e-9 * abs(lam)
    o = O.iram(A, k, m, which="LM", tol=TOL, v0=B.start_vector(n, 1, True))
    for lam in o["eigenvalues"]:
        assert np.min(np.abs(r["ev"] - lam)) < 1e-9 * abs(lam)
    X = r["x"]
    for q in range(k):
        assert np.linalg.norm(A @ X[:, q] - r["ev"][q] * X[:, q]) <= TOL * np.abs(r["ev"]).max()


def test_callback_operator_matches_dense():
    # CuHArnoldiCallback::setCallback: the matvec is user code on the device
    A, lam = planted_symmetric(300, seed=4)
    a = planes(A, False)[0]
    calls = []

    def mv(w, v, typ, stream):
        # run on the solver's stream so the ordering with its kernels holds
        st = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
        with torch.cuda.stream(st):
            torch.mv(a, ptr_tensor(v.re, 300), out=ptr_tensor(w.re, 300))
        calls.append(typ)
        return 0

    s = B.Arnoldi(300, 32, 5, seed=3)
    s.set_callback(mv)
    ev, res, st = s.solve()
    assert st == B.OK
    assert B.TYPE_WV in calls and B.TYPE_EIGENVECTOR in calls
    assert np.allclose(np.sort(np.array(ev).real)[::-1], lam[:5], rtol=1e-10)
    d = solve(A, 5, 32, seed=3)
    assert np.allclose(np.sort(np.array(ev).real), np.sort(d["ev"].real), rtol=1e-12)


def ptr_tensor(ptr, n):
    """A torch view of n FP64 values at a raw device pointer."""
    class _A:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                    "version": 3, "strides": None}
    return torch.as_tensor(_A(), device="cuda")


def test_solve_from_host_buffers():
    A = planted_complex(400, seed=9, nplant=5)
    s = B.Arnoldi(400, 24, 5, is_complex=True, seed=2)
    ev, res, st, X = s.solve_host(np.ascontiguousarray(A.real), np.ascontiguousarray(A.imag), vectors=True)
    assert st == B.OK and max(res) <= TOL
    for q in range(5):
        assert np.linalg.norm(A @ X[:, q] - ev[q] * X[:, q]) <= TOL * max(abs(e) for e in ev)


@pytest.mark.parametrize("n", [8192, 1000])
def test_mixed_solve_from_host_buffers(n):
    # the mixed form's host-input solve copies the operator in row blocks and
    # splits each block while the next one is copied: the same pairs as the
    # solve on the device-resident operator (n = 1000: ragged last block,
    # the plain path solving on the same handle)
    A = planted_complex(n, seed=21, nplant=6)
    s = B.Arnoldi(n, 32, 6, is_complex=True, precision=B.PREC_MIXED, seed=4)
    ev, res, st, X = s.solve_host(np.ascontiguousarray(A.real), np.ascontiguousarray(A.imag), vectors=True)
    assert st == B.OK and max(res) <= TOL
    scale = max(abs(e) for e in ev)
    for q in range(6):
        assert np.linalg.norm(A @ X[:, q] - ev[q] * X[:, q]) <= TOL * scale * 1.01
    d = solve(A, 6, 32, precision=B.PREC_MIXED, seed=4)
    for lam in d["ev"]:
        assert np.min(np.abs(np.array(ev) - lam)) < 1e-9 * abs(lam)
    if n >= 8192:  # the BF16 planes built block by block equal the ones built at once
        xr = torch.randn(4, n, dtype=torch.float64, device="cuda")
        xi = torch.randn(4, n, dtype=torch.float64, device="cuda")
        w1 = s.apply_block(xr, xi, precision=B.PREC_MIXED)
        w2 = d["solver"].apply_block(xr, xi, precision=B.PREC_MIXED)
        assert torch.equal(w1[0], w2[0]) and torch.equal(w1[1], w2[1])


def test_mixed_solve_on_a_user_stream():
    # the mixed form on a caller's non-default stream: its overlapped checks
    # (second stream, events) order against that stream; same pairs as on the
    # default stream, and the caller's stream sees the results in order
    n = 8192
    A = planted_complex(n, seed=31, nplant=6)
    are, aim = planes(A, True)
    d = solve(A, 6, 32, precision=B.PREC_MIXED, seed=5)
    user = torch.cuda.Stream()
    user.wait_stream(torch.cuda.current_stream())  # the operator planes were written on the default stream
    with torch.cuda.stream(user):
        s = B.Arnoldi(n, 32, 6, is_complex=True, precision=B.PREC_MIXED, seed=5, stream=user.cuda_stream)
        s.set_operator(are, aim)
        ev, res, st = s.solve()
    user.synchronize()
    assert st == B.OK and max(res) <= TOL
    assert s.stats()["refine_iterations"] >= 2
    assert np.allclose(np.array(ev), d["ev"], rtol=0, atol=1e-12 * np.abs(d["ev"]).max())


def test_first_value_is_one_start():
    A, lam = planted_symmetric(200, seed=5)
    r = solve(A, 3, 20, init=B.INIT_FIRST_VALUE_IS_ONE)
    assert np.allclose(np.sort(r["ev"].real)[::-1], lam[:3], rtol=1e-10)


def test_not_converged_is_reported():
    A, lam = planted_symmetric(256, seed=6, lo_exp=-0.01)   # tiny gaps
    s = B.Arnoldi(256, 12, 4, max_restarts=1)
    s.set_operator(*planes(A, False))
    ev, res, st = s.solve(allow_not_converged=True)
    assert st == B.NOT_CONVERGED


@pytest.mark.parametrize("n,refine", [(8192, True), (8192, False)])
def test_mixed_precision_reaches_fp64_residual(n, refine):
    # FP32-class phase, then the FP64-anchored Sylvester refinement (refine)
    # or FP64 subspace iteration to 1e-10
    A = planted_complex(n, seed=n + 1, nplant=8)
    r = solve(A, 8, 40, precision=B.PREC_MIXED, vectors=True, refine=refine)
    st = r["stats"]
    assert st["converged"] == 1 and r["res"].max() <= TOL
    assert st["matvec_fp32"] == 0 or st["refine_iterations"] >= 1
    if refine:  # FP64 operator: about two passes (no fallback to FP64 subspace iteration)
        assert st["fallbacks"] == 0 and st["block_matvecs"] - st["refine_iterations"] >= 1
    p = solve(A, 8, 40, precision=B.PREC_FP64)
    for lam in p["ev"]:
        assert np.min(np.abs(r["ev"] - lam)) < 1e-9 * abs(lam)
    X = r["x"]
    for q in range(8):
        assert np.linalg.norm(A @ X[:, q] - r["ev"][q] * X[:, q]) <= TOL * np.abs(r["ev"]).max() * 1.01


def test_mixed_trace_and_bf16_passes():
    # the convergence trace of a mixed solve: FP32-class checks with falling
    # residuals, then the refinement's outer steps down to the goal; the
    # leading powers run on the BF16 planes, and the FP32-class passes before
    # each check keep the measured residuals on the FP32-class operator
    A = planted_complex(8192, seed=11, nplant=8)
    r = solve(A, 8, 40, precision=B.PREC_MIXED)
    tr = r["solver"].trace()
    st = r["stats"]
    assert st["converged"] == 1 and r["res"].max() <= TOL
    assert [t[0] for t in tr if t[0] != 1] and all(t[0] in (1, 3) for t in tr)
    p1 = [t for t in tr if t[0] == 1]
    assert p1 and p1[0][3] >= 1 and st["block_bf16"] >= p1[0][3]
    assert all(a[4] > b[4] for a, b in zip(p1, p1[1:3]))
    assert tr[-1][0] == 3 and tr[-1][4] <= TOL
    # the refinement's Rayleigh-Ritz matrix is nearly triangular: inverse
    # iteration delivered its eigenpairs
    assert st["eig_fast"] >= 1
    assert all(a[2] < b[2] for a, b in zip(tr, tr[1:]))
    # CUDA-core passes (tensor_cores = 0) take no BF16 pass
    r0 = solve(A, 8, 40, precision=B.PREC_MIXED, tensor_cores=False)
    assert r0["stats"]["block_bf16"] == 0 and r0["res"].max() <= TOL


@pytest.mark.parametrize("gap", ["separated", "clustered"])
def test_mixed_precision_real_symmetric(gap):
    # separated: 4 eigenvalues well above the rest; clustered: the geometric
    # 1 .. 1e-3 spectrum, where the refinement must hand over to the FP64
    # Krylov restarts
    n = 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(8)
    Q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g))
    lam = 10.0 ** (-3.0 * torch.arange(n, dtype=torch.float64, device="cuda") / (n - 1))
    if gap == "separated":
        lam[:4] = torch.tensor([8.0, 7.0, 6.0, 5.0], dtype=torch.float64, device="cuda")
    A = ((Q * lam) @ Q.T).contiguous()
    s = B.Arnoldi(n, 32, 4, precision=B.PREC_MIXED, seed=1)
    s.set_operator(A)
    ev, res, st = s.solve()
    assert st == B.OK and max(res) <= TOL
    want = torch.sort(lam, descending=True).values[:4].cpu().numpy()
    assert np.allclose(np.sort(np.array(ev).real)[::-1], want, rtol=1e-10)


@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n,b", [(1024, 20), (1000, 7), (8192, 18), (999, 5), (130, 32), (2, 1)])
def test_block_pass_precisions(cplx, n, b):
    # FP64 block passes (DMMA tensor cores and CUDA cores; odd n takes the
    # CUDA-core pass) vs the FP64 torch product, the FP32 (CUDA-core) and
    # split-BF16 tensor-core passes within their precision
    g = torch.Generator(device="cuda")
    g.manual_seed(n + b)
    are = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    aim = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5 if cplx else None
    xr = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g)
    xi = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g) if cplx else None
    A = are if not cplx else torch.complex(are, aim)
    X = xr if not cplx else torch.complex(xr, xi)
    ref = (A @ X.T).T
    scale = (A.abs() @ X.abs().T).T
    # (the BF16 pass: operator rounded to BF16, unit roundoff 2^-8 = 3.9e-3, X split;
    # its coarse form rounds X to BF16 too: each product within 2^-7 = 7.8e-3;
    # FP64 passes through a mixed-form handle and through an FP64 handle)
    # (the FP64 pass of a mixed-form handle takes the int8-slice pass for b <= 16
    # complex / 32 real vectors: 2^-43 of the row scale per element)
    for prec, tc, tol, hp in ((B.PREC_FP64, True, 1e-12, B.PREC_MIXED), (B.PREC_FP64, True, 1e-13, B.PREC_FP64),
                              (B.PREC_FP64, False, 1e-13, B.PREC_MIXED), (B.PREC_MIXED, False, 2e-6, B.PREC_MIXED),
                              (B.PREC_MIXED, True, 1e-4, B.PREC_MIXED), (B.PASS_BF16, True, 4e-3, B.PREC_MIXED),
                              (B.PASS_BF16_COARSE, True, 8e-3, B.PREC_MIXED)):
        s = B.Arnoldi(n, min(16, n), min(4, n - 1), is_complex=cplx, precision=hp, tensor_cores=tc)
        s.set_operator(are, aim)
        wr, wi = s.apply_block(xr, xi, precision=prec)
        W = wr if not cplx else torch.complex(wr, wi)
        err = ((W - ref).abs() / scale).max().item()
        assert err <= tol, (prec, tc, hp, err)
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n,b", [(1000, 7), (4096, 16), (130, 3), (2, 1), (8192, 16), (999, 32), (4096, 24)])
def test_i8_block_pass(cplx, n, b):
    # the FP64-class pass on the integer tensor cores (6 int8 slices of each
    # operator row below its power-of-two scale, 7 of each vector, slice
    # products of order <= 8) against the FP64 torch product, on rows and
    # columns of widely different magnitude and a planted diagonal: the
    # error stays below 2^-40 of the row maximum times |x|_1 plus the
    # truncated slice products, 2^-45 n of row maximum times vector maximum
    if cplx and b > 16:
        pytest.skip("complex operators take the int8 pass for b <= 16")
    g = torch.Generator(device="cuda")
    g.manual_seed(7 * n + b)
    rs = torch.logspace(-6, 6, n, dtype=torch.float64, device="cuda")[torch.randperm(n, generator=g, device="cuda")]
    are = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    are += torch.diag(4.0 * (torch.arange(n, device="cuda") % 17 == 0).double())
    are *= rs[:, None]
    aim = (torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5 * rs[:, None]
           if cplx else None)
    cs = torch.logspace(-3, 3, b, dtype=torch.float64, device="cuda")
    xr = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g) * cs[:, None]
    xr[:, ::5] *= 1e-9  # entries far below their vector's maximum
    xi = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g) * cs[:, None] if cplx else None
    A = are if not cplx else torch.complex(are, aim)
    X = xr if not cplx else torch.complex(xr, xi)
    ref = (A @ X.T).T
    rowmax = are.abs().amax(1) if not cplx else torch.maximum(are.abs().amax(1), aim.abs().amax(1))
    xmax = xr.abs().amax(1) if not cplx else torch.maximum(xr.abs().amax(1), xi.abs().amax(1))
    x1 = xr.abs().sum(1) + (xi.abs().sum(1) if cplx else 0)
    bound = 2.0 ** -40 * rowmax[None, :] * x1[:, None] + 2.0 ** -45 * n * rowmax[None, :] * xmax[:, None]
    s = B.Arnoldi(n, min(16, n), min(4, n - 1), is_complex=cplx, precision=B.PREC_MIXED, tensor_cores=True)
    s.set_operator(are, aim)
    before = s.stats()["block_i8"]
    for _ in range(2):  # the vector-slice scratch is reused
        wr, wi = s.apply_block(xr, xi, precision=B.PREC_FP64)
        W = wr if not cplx else torch.complex(wr, wi)
        err = (W - ref).abs()
        assert bool((err <= bound).all()), (err / bound).max().item()
    assert s.stats()["block_i8"] == before + 2
    s.close()


@pytest.mark.gpu
def test_i8_pass_gated_by_tolerance():
    # residual goals below 1e-12 keep the exact FP64 (DMMA) pass on a
    # mixed-form handle; 1e-12 and above take the int8-slice pass
    n, b = 1024, 8
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    are = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    aim = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    xr = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g)
    xi = torch.randn(b, n, dtype=torch.float64, device="cuda", generator=g)
    ref = (torch.complex(are, aim) @ torch.complex(xr, xi).T).T
    scale = (torch.complex(are, aim).abs() @ torch.complex(xr, xi).abs().T).T
    for tol, i8 in ((1e-13, False), (1e-12, True), (1e-10, True)):
        s = B.Arnoldi(n, 16, 4, is_complex=True, precision=B.PREC_MIXED, tensor_cores=True, tolerance=tol)
        s.set_operator(are, aim)
        wr, wi = s.apply_block(xr, xi, precision=B.PREC_FP64)
        assert s.stats()["block_i8"] == (1 if i8 else 0), tol
        err = ((torch.complex(wr, wi) - ref).abs() / scale).max().item()
        assert err <= (1e-12 if i8 else 1e-13), (tol, err)
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [True, False])
def test_matvec_autotune_variants(cplx):
    # every launch variant of the single-vector pass (forced: autotune = 2 + v)
    # and the autotuned one solve to the pairs of the default variant
    n = 2048
    A = planted_complex(n, seed=21, nplant=5) if cplx else planted_symmetric(n, seed=21)[0]
    r0 = solve(A, 5, 24, autotune=False)
    assert r0["stats"]["matvec_variant"] == 0 and r0["res"].max() <= TOL
    for autotune in [True] + [2 + v for v in range(6)]:
        r = solve(A, 5, 24, autotune=autotune)
        v = r["stats"]["matvec_variant"]
        assert 0 <= v < 6 and (autotune is True or v == autotune - 2)
        assert r["res"].max() <= TOL
        assert np.allclose(np.sort_complex(r0["ev"]), np.sort_complex(r["ev"]), rtol=1e-11, atol=0)


@pytest.mark.parametrize("cplx,n,k,m", [(False, 256, 5, 32), (True, 300, 6, 24), (True, 2048, 4, 32),
                                        (False, 64, 4, 12)])
def test_onchip_chosen_form_small_operators(cplx, n, k, m):
    # the chosen form below the tensor-core sizes: the whole restart loop of
    # one problem on one CTA; the same eigenpairs as the multi-kernel FP64
    # restart loop and the oracle, eigenvectors and test_outcome as usual
    A = planted_complex(n, seed=n + k, nplant=k) if cplx else planted_symmetric(n, seed=n)[0]
    r = solve(A, k, m, precision=B.PREC_MIXED, vectors=True)
    assert r["stats"]["onchip"] == 1 and r["stats"]["converged"] == 1
    assert r["res"].max() <= TOL
    p = solve(A, k, m, precision=B.PREC_FP64)
    assert p["stats"]["onchip"] == 0
    scale = np.abs(p["ev"]).max()
    for lam in p["ev"]:
        assert np.min(np.abs(r["ev"] - lam)) <= 1e-10 * scale
    o = O.iram(A, k, m, which="LM", tol=TOL, seed=1)
    for lam in o["eigenvalues"]:
        assert np.min(np.abs(r["ev"] - lam)) <= 1e-10 * scale
    X = r["x"]
    for q in range(k):
        assert np.linalg.norm(A @ X[:, q] - r["ev"][q] * X[:, q]) <= TOL * scale * 1.01
        assert r["solver"].test_outcome(q) <= TOL
