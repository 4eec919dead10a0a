"""Matrix files in the reference's format (oap::host::WriteMatrix /
ReadMatrix: one utils::ByteBuffer holding SaveMatrix's packed record) and
the solver checkpoint built on them.  CPU: the header parser against files
written by the reference's own writer (oracle/_ref) and by a byte-level
restatement of the format; GPU: device round trips, files of the reference's
writer read into device planes, and save / load / resume of an interrupted
solve.  (The reference's own reader cannot run here: utils::Buffer::
increaseReadIdx, oapUtils/Buffer.h:324-327, falls off the end of a
value-returning function, which g++ compiles to a trap.)"""

import ctypes as C
import struct

import numpy as np
import pytest

import oap_b200 as B
import oracle as O

HAVE_REF = O.ref() is not None


def write_bytes(path, a, header_slack=0):
    """The format restated byte by byte: size_t 1, size_t length, payload
    (bool present, bool isRe, bool isIm, uint32 columns, uint32 rows, re, im)."""
    rows, cols = a.shape
    cplx = np.iscomplexobj(a)
    payload = struct.pack("<???II", True, True, cplx, cols, rows)
    payload += np.ascontiguousarray(a.real, dtype="<f8").tobytes()
    if cplx:
        payload += np.ascontiguousarray(a.imag, dtype="<f8").tobytes()
    with open(path, "wb") as f:
        f.write(struct.pack("<QQ", 1, len(payload) + header_slack))
        f.write(payload)


@pytest.mark.parametrize("cplx", [False, True])
def test_read_info_of_restated_format(tmp_path, cplx):
    rng = np.random.default_rng(1)
    a = rng.normal(size=(5, 3)) + (1j * rng.normal(size=(5, 3)) if cplx else 0)
    p = tmp_path / "m.bin"
    write_bytes(p, a, header_slack=37)  # the reference announces its allocated length
    assert B.mat_read_info(p) == (3, 5, True, cplx)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref/libref.so not built")
@pytest.mark.parametrize("cplx", [False, True])
def test_read_info_of_reference_writer(tmp_path, cplx):
    rng = np.random.default_rng(2)
    a = rng.normal(size=(7, 4)) + (1j * rng.normal(size=(7, 4)) if cplx else 0)
    p = tmp_path / "ref.bin"
    O.ref_write_matrix(p, a)
    assert B.mat_read_info(p) == (4, 7, True, cplx)
    # the reference's own writer produces exactly the restated payload
    q = tmp_path / "mine.bin"
    write_bytes(q, a)
    assert open(p, "rb").read()[16:] == open(q, "rb").read()[16:]


def test_bad_file_is_an_argument_error(tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(b"\x02" + b"\x00" * 20)
    c = C.c_uint32()
    assert B.lib().oapb_mat_read_info(str(p).encode(), C.byref(c), None, None, None) == B.ERR_ARG
    assert B.lib().oapb_mat_read_info(str(tmp_path / "missing.bin").encode(), None, None, None, None) == B.ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [False, True])
def test_device_round_trip_and_reference_interchange(tmp_path, cplx):
    import torch
    rng = np.random.default_rng(3)
    a = rng.normal(size=(33, 17)) + (1j * rng.normal(size=(33, 17)) if cplx else 0)
    re = torch.from_numpy(np.ascontiguousarray(a.real)).cuda()
    im = torch.from_numpy(np.ascontiguousarray(a.imag)).cuda() if cplx else None
    p = tmp_path / "dev.bin"
    B.mat_write(p, re, im)
    r2, i2 = B.mat_read(p)
    assert torch.equal(r2, re) and (not cplx or torch.equal(i2, im))
    q0 = tmp_path / "restated.bin"
    write_bytes(q0, a)
    assert open(p, "rb").read() == open(q0, "rb").read()
    if HAVE_REF:  # a file of the reference's writer read into device planes
        q = tmp_path / "ref.bin"
        O.ref_write_matrix(q, a)
        r3, i3 = B.mat_read(q)
        back = r3.cpu().numpy() + (1j * i3.cpu().numpy() if cplx else 0)
        assert np.array_equal(back, a)


def planted(n, seed):
    rng = np.random.default_rng(seed)
    A = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) / np.sqrt(2 * n)
    A[np.arange(6), np.arange(6)] += np.array([3.0, 2.9, 2.8, 2.7, 2.6, 2.5])
    return A


@pytest.mark.gpu
def test_checkpoint_resume_equals_uninterrupted(tmp_path):
    import torch
    n, m, k = 600, 12, 4
    A = planted(n, 7)
    re = torch.from_numpy(np.ascontiguousarray(A.real)).cuda()
    im = torch.from_numpy(np.ascontiguousarray(A.imag)).cuda()
    full = B.Arnoldi(n, m, k, is_complex=True, seed=5)
    full.set_operator(re, im)
    ev_full, res_full, st = full.solve()
    restarts_full = full.stats()["restarts"]
    assert st == B.OK and restarts_full >= 3
    # interrupted after one restart, saved, loaded into a fresh handle, resumed
    part = B.Arnoldi(n, m, k, is_complex=True, seed=5, max_restarts=1)
    part.set_operator(re, im)
    _, _, st = part.solve(allow_not_converged=True)
    assert st == B.NOT_CONVERGED
    p = tmp_path / "ckpt.bin"
    part.save(p)
    c, r, hr, hi = B.mat_read_info(p)          # first record: the 1 x 8 header
    assert (c, r, hr) == (1, 8, True)
    fresh = B.Arnoldi(n, m, k, is_complex=True, seed=99)
    fresh.set_operator(re, im)
    fresh.load(p)
    ev, res, st = fresh.resume()
    assert st == B.OK and max(res) <= 1e-10
    assert fresh.stats()["restarts"] == restarts_full
    assert np.allclose(np.array(ev), np.array(ev_full), rtol=1e-12, atol=0)
    # a handle of another shape refuses the file; an unsolved handle has nothing to save
    other = B.Arnoldi(n, m + 2, k, is_complex=True)
    other.set_operator(re, im)
    assert B.lib().oapb_arnoldi_load(other.h, str(p).encode()) == B.ERR_ARG
    assert B.lib().oapb_arnoldi_save(other.h, str(tmp_path / "x.bin").encode()) == B.ERR_ARG
