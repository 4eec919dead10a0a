"""Helpers for the GPU tests: numpy <-> device planes in the reference layout."""
import numpy as np


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def planes(a, complex_=None):
    """(re, im) device tensors of a numpy matrix / vector; im None if real."""
    a = np.asarray(a)
    cplx = np.iscomplexobj(a) if complex_ is None else complex_
    re = dev(a.real)
    im = dev(a.imag) if cplx else None
    return re, im


def host(re, im=None):
    r = re.cpu().numpy()
    return r if im is None else r + 1j * im.cpu().numpy()


def zeros(shape, cplx):
    import torch
    re = torch.zeros(shape, dtype=torch.float64, device="cuda")
    im = torch.zeros(shape, dtype=torch.float64, device="cuda") if cplx else None
    return re, im


def planted_symmetric(n, seed, lo_exp=-3.0):
    """A = Q diag(lambda) Q^T, Q from QR of a seeded N(0,1) matrix,
    lambda_i = 10^(lo_exp * i / (n-1)) (1 down to 10^lo_exp)."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    lam = 10.0 ** (lo_exp * np.arange(n) / (n - 1))
    return (Q * lam) @ Q.T, lam


def planted_complex(n, seed, nplant, shift=4.0):
    """Complex A with entries N(0, 1/n) (re, im each variance 1/(2n)) plus
    `shift` on `nplant` seeded diagonal positions."""
    rng = np.random.default_rng(seed)
    s = 1.0 / np.sqrt(2.0 * n)
    A = rng.normal(scale=s, size=(n, n)) + 1j * rng.normal(scale=s, size=(n, n))
    pos = rng.choice(n, nplant, replace=False)
    A[pos, pos] += shift
    return A
