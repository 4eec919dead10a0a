"""Learned warm start for parameterised operators A(theta) = A0 + sum_i theta_i B_i.

The network (oapb_mlp: BF16 weights and activations, FP32 accumulation,
trained on the GPU by the library's own forward / backward / Adam kernels)
maps theta to
  * a start vector: the projection P(theta) u of a fixed seeded vector u on
    the wanted invariant subspace (sign-free, unlike single eigenvectors),
  * a shift set: the next eigenvalues after the wanted ones (the unwanted
    values closest to the wanted set, i.e. the final exact shifts of the
    plain method).
A solve from the prediction filters the predicted vector with the predicted
shifts (oapb_arnoldi_set_start_shifts) and runs the plain FP64 restarted
Arnoldi, which accepts the result only at its residual goal; if the goal is
not met within the restart budget the same call solves again from the seeded
random start (fallback_random).

The training targets come from the plain method itself: batched FP64 IRAM
solves (oapb_arnoldi_solve_batched) of A(theta) for random theta.
"""

import ctypes as C

import numpy as np

from . import (INIT_USER, OK, Arnoldi, check, lib, solve_batched, _stream)


class ParamFamily:
    """A0 and B_1..B_p: seeded symmetric Gaussian (G + G^T) / (2 sqrt(n)),
    FP64 on the device; the B_i multiplied by `scale` (1: the family as
    specified; a smaller scale makes the wanted subspace a smooth function of
    theta, see solve_from_prediction)."""

    def __init__(self, n=2048, nparams=16, seed=0, device="cuda", scale=1.0):
        import torch
        self.n, self.nparams = n, nparams
        g = torch.Generator(device=device)
        g.manual_seed(seed)

        def sym():
            G = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
            return ((G + G.T) / (2.0 * n ** 0.5)).contiguous()

        self.A0 = sym()
        self.B = [sym().mul_(scale) for _ in range(nparams)]
        self.scale = scale
        self._ptrs = (C.c_void_p * nparams)(*[b.data_ptr() for b in self.B])

    def operators(self, theta, out=None, stream=None):
        """A(theta_p) for theta (P x nparams, float64, device) -> (P, n, n)."""
        import torch
        P = theta.shape[0]
        theta = theta.to(dtype=torch.float64).contiguous()
        if out is None:
            out = torch.empty(P, self.n, self.n, dtype=torch.float64, device=theta.device)
        check(lib().oapb_param_operators(C.c_void_p(self.A0.data_ptr()), self._ptrs, self.nparams,
                                         C.c_void_p(theta.data_ptr()), P, self.n,
                                         C.c_void_p(out.data_ptr()), _stream(stream)),
              "oapb_param_operators")
        return out


def probe_vector(n, seed=12345):
    """The fixed vector u whose projections are the start-vector targets."""
    rng = np.random.default_rng(seed)
    u = rng.normal(size=n)
    return u / np.linalg.norm(u)


def make_targets(fam, theta, wanted=8, nshift=8, chunk=256, hdim=32, tol=1e-10, sort="LR"):
    """Plain-method solves of A(theta) (batched FP64 IRAM, top wanted + nshift
    values) -> (targets P x (n + nshift) float32, eigenvalues, status)."""
    import torch
    n = fam.n
    kk = wanted + nshift
    u = torch.from_numpy(probe_vector(n)).cuda()
    T = np.zeros((theta.shape[0], n + nshift), dtype=np.float32)
    evs = np.zeros((theta.shape[0], kk))
    sts = np.zeros(theta.shape[0], dtype=np.int32)
    for c0 in range(0, theta.shape[0], chunk):
        c1 = min(theta.shape[0], c0 + chunk)
        ops = fam.operators(theta[c0:c1])
        mats = [(ops[i], None) for i in range(c1 - c0)]
        vecs = [(torch.empty(n, kk, dtype=torch.float64, device="cuda"), None) for _ in range(c1 - c0)]
        ev, res, st, stats, rc = solve_batched(mats, kk, hdim=hdim, sort=sort, tolerance=tol, vectors=vecs)
        for i in range(c1 - c0):
            X = vecs[i][0][:, :wanted]
            v = X @ (X.T @ u)
            v = v / torch.linalg.norm(v)
            T[c0 + i, :n] = (v * n ** 0.5).float().cpu().numpy()
            T[c0 + i, n:] = ev[i, wanted:kk].real
        evs[c0:c1] = ev.real
        sts[c0:c1] = st
        del ops, mats, vecs
    return T, evs, sts


class Net:
    """oapb_mlp over the C ABI."""

    def __init__(self, sizes, seed=1, acts=None):
        """acts: one oapb_activation per layer (len(sizes) - 1), default tanh
        hidden layers and a linear output."""
        self.sizes = list(sizes)
        self.h = C.c_void_p()
        arr = (C.c_uint32 * len(sizes))(*sizes)
        check(lib().oapb_mlp_create(C.byref(self.h), arr, len(sizes) - 1, seed), "oapb_mlp_create")
        self.nparam = int(lib().oapb_mlp_num_params(self.h))
        if acts is not None:
            self.set_activations(acts)

    def set_activations(self, acts):
        arr = (C.c_int32 * len(acts))(*[int(a) for a in acts])
        check(lib().oapb_mlp_set_activations(self.h, arr, len(acts)), "oapb_mlp_set_activations")

    def activations(self):
        arr = (C.c_int32 * (len(self.sizes) - 1))()
        check(lib().oapb_mlp_get_activations(self.h, arr, len(self.sizes) - 1), "oapb_mlp_get_activations")
        return list(arr)

    def close(self):
        if self.h:
            lib().oapb_mlp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, x):
        import torch
        B = x.shape[0]
        y = torch.empty(B, self.sizes[-1], dtype=torch.float32, device="cuda")
        check(lib().oapb_mlp_forward(self.h, C.c_void_p(x.data_ptr()), B, C.c_void_p(y.data_ptr()), None),
              "oapb_mlp_forward")
        return y

    def backward(self, x, target):
        loss = C.c_double()
        check(lib().oapb_mlp_backward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(target.data_ptr()),
                                      x.shape[0], C.byref(loss), None), "oapb_mlp_backward")
        return loss.value

    def adam(self, lr):
        check(lib().oapb_mlp_adam_step(self.h, C.c_float(lr), None), "oapb_mlp_adam_step")

    def params(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        check(lib().oapb_mlp_copy(self.h, 0, C.c_void_p(out.ctypes.data), None), "oapb_mlp_copy")
        return out

    def grads(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        check(lib().oapb_mlp_copy(self.h, 1, C.c_void_p(out.ctypes.data), None), "oapb_mlp_copy")
        return out

    def save(self, path):
        """Network::save in the reference's matrix file format (oapb_mlp_save)."""
        check(lib().oapb_mlp_save(self.h, str(path).encode()), "oapb_mlp_save")

    @classmethod
    def load(cls, path, seed=1):
        """Network::load (oapb_mlp_load)."""
        net = cls.__new__(cls)
        net.h = C.c_void_p()
        check(lib().oapb_mlp_load(C.byref(net.h), str(path).encode(), seed), "oapb_mlp_load")
        n = lib().oapb_mlp_num_layers(net.h, None)
        sizes = (C.c_uint32 * (n + 1))()
        lib().oapb_mlp_num_layers(net.h, sizes)
        net.sizes = list(sizes)
        net.nparam = int(lib().oapb_mlp_num_params(net.h))
        return net

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().oapb_mlp_set_params(self.h, C.c_void_p(p.ctypes.data), None), "oapb_mlp_set_params")

    def train(self, X, T, epochs=30, batch=256, lr=1e-3, seed=0, lr_decay=0.97):
        """Mini-batch Adam on device tensors X (P x in), T (P x out)."""
        import torch
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        losses = []
        P = X.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(P, generator=g, device="cuda")
            tot = 0.0
            nb = 0
            for b0 in range(0, P - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xb = X[idx].contiguous()
                tb = T[idx].contiguous()
                tot += self.backward(xb, tb)
                self.adam(lr)
                nb += 1
            losses.append(tot / max(1, nb))
            lr *= lr_decay
        return losses


def solve_from_prediction(A, pred, n, wanted=8, hdim=24, tol=1e-10, max_restarts=300, seed=7,
                          use_shifts=False):
    """Solve A (device FP64 n x n) from a network prediction (n + shifts).

    The predicted vector starts the plain FP64 restarted Arnoldi, which judges
    the result at its residual goal and restarts from the seeded random
    vector when the goal is not met (fallback_random).  How much the start
    saves depends on its distance eps from the wanted subspace (the norm of
    its component outside the subspace over the norm inside): on the
    specified family (n = 2048, scale 1) measured plain-IRAM costs were 616
    operator applications from a random start and 568 / 520 / 472 / 376 / 56
    from starts with eps = 1 / 0.1 / 0.01 / 0.001 / 0 (hdim 24, 8 wanted):
    only starts far closer than a theta -> vector regression reaches on that
    family pay.  With use_shifts the predicted shifts (the unwanted values
    next to the wanted set) also filter the start vector; with predictions at
    the family's eigenvalue-fluctuation level this filter damps nothing and
    is off by default."""
    import torch
    v0 = pred[:n].double().contiguous()
    s = Arnoldi(n, hdim, wanted, sort="LR", tolerance=tol, max_restarts=max_restarts, seed=seed,
                init=INIT_USER, fallback_random=True)
    s.set_operator(A)
    s.set_start_vector(v0)
    if use_shifts:
        s.set_start_shifts([float(x) for x in pred[n:].cpu().numpy()])
    ev, res, st = s.solve(allow_not_converged=True)
    stats = s.stats()
    s.close()
    return ev, res, st, stats


def solve_random(A, n, wanted=8, hdim=24, tol=1e-10, max_restarts=300, seed=7, vectors=False):
    """The method without the network: the plain FP64 restarted Arnoldi from
    its seeded random start (with vectors: also the (n, wanted) eigenvectors)."""
    import torch
    s = Arnoldi(n, hdim, wanted, sort="LR", tolerance=tol, max_restarts=max_restarts, seed=seed)
    s.set_operator(A)
    X = torch.zeros(n, wanted, dtype=torch.float64, device="cuda") if vectors else None
    ev, res, st = s.solve(vectors=(X, None) if vectors else None, allow_not_converged=True)
    stats = s.stats()
    s.close()
    return (ev, res, st, stats, X) if vectors else (ev, res, st, stats)


def start_error(v, X):
    """eps of a start vector v against the wanted subspace span(X) (X: n x k
    orthonormal columns): the norm of v's component outside the subspace
    over the norm of its component inside."""
    import torch
    v = v.double()
    inside = X @ (X.T @ v)
    return float(torch.linalg.norm(v - inside) / torch.linalg.norm(inside).clamp_min(1e-300))
