"""CPU-side checks of the C ABI: the library builds, loads and exports every
function declared in include/oapb200.h.  No compute calls (no GPU here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"OAPB_EXPORT\s+[\w\s\*]+?\b(oapb_\w+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def libpath():
    from oap_b200 import build
    return build.build()


def test_header_declares_surface():
    names = declared()
    for must in ("oapb_dot_product", "oapb_transpose", "oapb_magnitude", "oapb_sum",
                 "oapb_tensor_product", "oapb_qr_givens", "oapb_qr_householder",
                 "oapb_arnoldi_create", "oapb_arnoldi_solve"):
        assert must in names


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version(libpath):
    import oap_b200
    L = oap_b200.lib()
    assert L.oapb_api_version() == 1
    assert oap_b200.status_string(oap_b200.NOT_CONVERGED) == "not converged"


def test_argument_validation_without_gpu(libpath):
    # Argument checks happen on the host before any CUDA call.
    import oap_b200
    L = oap_b200.lib()
    cfg = oap_b200.Config()
    L.oapb_arnoldi_config_default(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    cfg.n, cfg.hdim, cfg.wanted = 10, 4, 4   # wanted must be < hdim
    assert L.oapb_arnoldi_create(ctypes.byref(h), ctypes.byref(cfg), None) == oap_b200.ERR_ARG
    bad = oap_b200.Mat(0, 0, None, None, 0)
    assert L.oapb_transpose(ctypes.byref(bad), ctypes.byref(bad), None) == oap_b200.ERR_ARG


def test_start_vector_restatement():
    import numpy as np
    import oap_b200
    v = oap_b200.start_vector(1000, 7)
    assert v.min() >= -1 and v.max() < 1 and abs(v.mean()) < 0.1
    assert np.array_equal(v, oap_b200.start_vector(1000, 7))
