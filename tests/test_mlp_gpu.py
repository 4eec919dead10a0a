"""Warm-start network kernels (BF16, FP32 accumulation) against the CPU
oracle, training, and the learned warm start on a parameterised operator."""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oap_b200 as B  # noqa: E402
from oap_b200 import warmstart as W  # noqa: E402


@pytest.mark.parametrize("acts", [None, [M.SIGMOID, M.SIN, M.TANH], [M.SIN, M.TANH, M.SIGMOID],
                                  [M.LINEAR, M.SIGMOID, M.SIN]])
def test_forward_and_gradients_match_oracle(acts):
    # every activation of the reference (LINEAR, SIGMOID, TANH, SIN) in hidden
    # and output layers: forward output and all gradients against the oracle
    sizes = [16, 64, 48, 40]
    net = W.Net(sizes, seed=3, acts=acts)
    if acts is not None:
        assert net.activations() == acts
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, size=(24, 16)).astype(np.float32)
    t = rng.normal(size=(24, 40)).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = net.forward(xd).cpu().numpy()
    p = net.params()
    hf, _ = M.forward(p, sizes, x, acts)
    assert np.abs(y - hf[-1]).max() <= 1e-3 * max(1.0, np.abs(hf[-1]).max())
    loss = net.backward(xd, td)
    g = net.grads()
    lo, go = M.loss_and_grads(p, sizes, x, t, acts)
    assert abs(loss - lo) <= 1e-4 * lo
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel < 1e-3, rel
    assert np.allclose(g, go, rtol=2e-2, atol=2e-3 * np.abs(go).max())


def test_training_reduces_loss():
    sizes = [16, 64, 64, 8]
    net = W.Net(sizes, seed=5)
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, size=(2048, 16)).astype(np.float32)
    A = rng.normal(size=(16, 8)) / 4
    T = np.sin(X @ A).astype(np.float32)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    losses = net.train(Xd, Td, epochs=20, batch=128, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0]


def test_param_operators_match_definition():
    fam = W.ParamFamily(n=96, nparams=5, seed=2)
    theta = torch.rand(7, 5, dtype=torch.float64, device="cuda") * 2 - 1
    ops = fam.operators(theta)
    for p in range(7):
        ref = fam.A0 + sum(theta[p, i] * fam.B[i] for i in range(5))
        assert torch.allclose(ops[p], ref, rtol=0, atol=1e-14)


@pytest.mark.parametrize("scale,max_ratio", [(0.01, 0.85), (1.0, 1.10)])
def test_learned_warm_start_on_parametric_family(scale, max_ratio):
    # A(theta) = A0 + scale sum theta_i B_i (n = 256, 16 parameters, top-8):
    # the network is trained on the plain method's own eigenvectors, and the
    # held-out solves from its prediction are judged by the plain method
    # (every pair at 1e-10, the same eigenvalues as the random start).  With
    # scale 0.01 the wanted subspace is a smooth function of theta and the
    # prediction saves operator applications (at most 0.85x of the random
    # start's); with scale 1 (the family's specified form) it is not, the
    # prediction is about as far from the subspace as a random vector, and
    # the learned start costs at most 10 % more
    n, k = 256, 8
    fam = W.ParamFamily(n=n, nparams=16, seed=4, scale=scale)
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    th_train = torch.rand(3072, 16, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    th_test = torch.rand(16, 16, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    T, evs, st = W.make_targets(fam, th_train, wanted=k, nshift=8, chunk=512)
    # the targets come from the plain method's converged solves only
    ok = st == B.OK
    assert ok.mean() >= 0.9, ok.mean()
    net = W.Net([16, 256, 256, n + 8], seed=1)
    keep = torch.from_numpy(np.nonzero(ok)[0]).cuda()
    X = th_train[keep].float().contiguous()
    Td = torch.from_numpy(T[ok]).cuda()
    losses = net.train(X, Td, epochs=60, batch=128, lr=2e-3)
    assert losses[-1] < losses[0]
    pred = net.forward(th_test.float().contiguous())
    ops = fam.operators(th_test)
    mv_warm = mv_rand = 0
    eps = []
    for i in range(th_test.shape[0]):
        A = ops[i].contiguous()
        ev_w, res_w, st_w, s_w = W.solve_from_prediction(A, pred[i], n, wanted=k, hdim=24)
        ev_r, res_r, st_r, s_r, Xr = W.solve_random(A, n, wanted=k, hdim=24, vectors=True)
        assert st_w == B.OK and max(res_w) <= 1e-10
        assert st_r == B.OK and max(res_r) <= 1e-10
        assert np.allclose(np.sort(np.array(ev_w).real), np.sort(np.array(ev_r).real), rtol=1e-9)
        mv_warm += s_w["matvecs"]
        mv_rand += s_r["matvecs"]
        eps.append(W.start_error(pred[i, :n], Xr))
    print("scale", scale, "warm-start matvecs", mv_warm, "random-start matvecs", mv_rand,
          "median eps of the prediction", float(np.median(eps)))
    assert mv_warm <= max_ratio * mv_rand


@pytest.mark.gpu
def test_network_save_load_round_trip(tmp_path):
    # Network::save / load in the reference's matrix format: same outputs
    from oap_b200 import warmstart as W
    net = W.Net([5, 16, 3], seed=4)
    x = torch.randn(64, 5, device="cuda")
    y1 = net.forward(x)
    p = tmp_path / "net.bin"
    net.save(p)
    back = W.Net.load(p)
    assert back.sizes == [5, 16, 3]
    assert torch.equal(back.forward(x), y1)
    assert B.mat_read_info(p) == (1, 3, True, False)   # first record: the layer sizes
    # the activations travel with the file (the last record)
    net2 = W.Net([5, 16, 16, 3], seed=5, acts=[B.ACT_SIN, B.ACT_SIGMOID, B.ACT_TANH])
    y2 = net2.forward(x)
    p2 = tmp_path / "net2.bin"
    net2.save(p2)
    back2 = W.Net.load(p2)
    assert back2.activations() == [B.ACT_SIN, B.ACT_SIGMOID, B.ACT_TANH]
    assert torch.equal(back2.forward(x), y2)
