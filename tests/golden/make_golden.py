"""Extract the numeric fixtures that the reference's own tests use into
``fixtures.json`` (data only, no code).

Run in a checkout that has the oap sources next to it:

    python tests/golden/make_golden.py /root/reference

Sources read (paths relative to the oap project root):

* ``oapQRTestSamples/qrtest1..9.h``  - 32x32 Hessenberg matrices produced by
  the Arnoldi package at step 3 with their Q and R (used by
  ``oapDeviceTests/oapQRTests.cpp:51-195``).
* ``oapHostTests/host_qrtest1..4.h`` - small QR samples
  (``oapHostTests/oapQRTests.cpp:152-176``).
* ``oapHostTests/oapQRHTTests.cpp:38-76`` and
  ``oapDeviceTests/oapGenericArnoldiApiTests.cpp:53-333`` - the 4x4
  Hessenberg with its shift, and the 3x3 / 2x2 QR cases with expected Q, R and
  R*Q.
* ``oapArnoldiDeviceTests/schur1..3.h`` - matrices and the diagonal of their
  triangular form (``oapSchurDecompositionTests.cpp:61-130``).
* ``oapCMatrixDataTests/CMatrixData1..4.h`` - real matrices with their listed
  eigenvalues, and the solver settings / tolerances of
  ``oapArnoldiDeviceTests/oapArnoldiPackageMatricesTests.cpp:244-266``.

Matrices are stored the way the reference stores them: row-major, element
(column c, row r) at ``c + r * columns``.
"""

import json
import math
import os
import re
import sys

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def _strings(text, name):
    """Concatenate the C string literal(s) assigned to ``const char* name``."""
    m = re.search(r"const\s+char\s*\*\s*" + name + r"\s*=\s*(.*?);", text, re.S)
    if not m:
        raise KeyError(name)
    body = m.group(1)
    parts = re.findall(r'"((?:[^"\\]|\\.)*)"', body, re.S)
    return "".join(parts).replace("\\\n", " ").replace("\\", " ")


def _parse_matrix(s):
    """Parse the reference's text matrix format ``[a, b, ... | c, ...]``."""
    s = s.strip()
    inner = s[s.index("[") + 1: s.rindex("]")]
    # gdb-style run-length form: "0 <repeats 30 times>"
    inner = re.sub(r"(" + NUM + r")\s*<repeats\s+(\d+)\s+times>",
                   lambda m: ", ".join([m.group(1)] * int(m.group(2))), inner)
    rows = [r for r in inner.split("|")]
    vals = [float(x) for x in re.findall(NUM, inner)]
    if len(rows) > 1:
        ncols = len(re.findall(NUM, rows[0]))
        nrows = len(rows)
    else:
        side = int(round(math.sqrt(len(vals))))
        assert side * side == len(vals), (len(vals), s[:80])
        ncols = nrows = side
    assert ncols * nrows == len(vals)
    return {"columns": ncols, "rows": nrows, "re": vals}


def _c_array(text, name):
    m = re.search(r"\b" + name + r"\s*\[\s*\]\s*=\s*\{(.*?)\}\s*;", text, re.S)
    if not m:
        raise KeyError(name)
    return [float(x) for x in re.findall(NUM, m.group(1))]


def main(root):
    out = {"source": "oap reference test fixtures", "qr_samples": [],
           "host_qr_samples": [], "schur": [], "cmatrix": [], "small_qr": {}}

    for i in range(1, 10):
        path = os.path.join(root, "oapQRTestSamples", "qrtest%d.h" % i)
        t = open(path).read()
        out["qr_samples"].append({
            "name": "qrtest%d" % i,
            "matrix": _parse_matrix(_strings(t, "matrix")),
            "q": _parse_matrix(_strings(t, "qref")),
            "r": _parse_matrix(_strings(t, "rref")),
        })

    for i in range(1, 5):
        path = os.path.join(root, "oapHostTests", "host_qrtest%d.h" % i)
        t = open(path).read()
        item = {"name": "host_qrtest%d" % i,
                "matrix": _parse_matrix(_strings(t, "matrix"))}
        for key, name in (("q", "qref"), ("r", "rref")):
            try:
                item[key] = _parse_matrix(_strings(t, name))
            except KeyError:
                pass
        out["host_qr_samples"].append(item)

    for i in range(1, 4):
        path = os.path.join(root, "oapArnoldiDeviceTests", "schur%d.h" % i)
        t = open(path).read()
        out["schur"].append({
            "name": "schur%d" % i,
            "matrix": _parse_matrix(_strings(t, "matrix")),
            "triangular": _parse_matrix(_strings(t, "eq_matrix")),
        })

    # Solver settings of oapArnoldiPackageMatricesTests.cpp:244-266:
    # (wanted, hdim, tolerance on ||A x - lambda x||), sort = largest Re.
    settings = {1: (2, 6, 0.02), 2: (3, 6, 0.047), 3: (6, 12, 0.047),
                4: (6, 12, 0.047)}
    for i in range(1, 5):
        path = os.path.join(root, "oapCMatrixDataTests", "CMatrixData%d.h" % i)
        t = open(path).read()
        mat = _c_array(t, "matrix")
        ev = _c_array(t, "eigenvalues")
        n = len(ev)
        assert len(mat) == n * n
        wanted, hdim, tol = settings[i]
        out["cmatrix"].append({
            "name": "CMatrixData%d" % i, "n": n, "re": mat,
            "eigenvalues": ev, "wanted": wanted, "hdim": hdim,
            "tolerance": tol, "sort": "SortLargestReValues",
        })

    # 4x4 Hessenberg + shift (oapQRHTTests.cpp:38-76,
    # oapGenericArnoldiApiTests.cpp:53-100).
    h_init = [-4.4529e-01, -1.8641e+00, -2.8109e+00, 7.2941e+00,
              8.0124e+00, 6.2898e+00, 1.2058e+01, -1.6088e+01,
              0.0, 4.0087e-01, 1.1545e+00, -3.3722e-01,
              0.0, 0.0, -1.5744e-01, 3.0010e+00]
    out["small_qr"]["hessenberg4"] = {
        "h": h_init, "shift": h_init[15],
        "r_expected": [8.7221, 3.7577, 12.1875, -17.6610,
                       0.0, 0.5755, -2.8519, -0.4816,
                       0.0, 0.0, -0.2507, 0.0019,
                       0.0, 0.0, 0.0, -0.0015],
        "q_expected": [-0.3951, -0.6591, -0.4979, 0.4019,
                       0.9186, -0.2835, -0.2142, 0.1728,
                       0.0, 0.6965, -0.5584, 0.4506,
                       0.0, 0.0, 0.6280, 0.7782],
        "h1_expected": [3.0067e+00, 1.6742e+00, -2.3047e+01, -4.0863e+00,
                        5.2870e-01, 8.5146e-01, 1.1660e+00, -1.5609e+00,
                        0.0, -1.7450e-01, 3.1421e+00, -1.1140e-01,
                        0.0, 0.0, -1.0210e-03, 2.9998e+00],
        "tolerance": 0.001,
    }
    out["small_qr"]["sym3"] = {
        "a": [6, 5, 0, 5, 1, 4, 0, 4, 3],
        "q_expected": [0.7682, 0.3327, 0.547, 0.6402, -0.3992, -0.6564,
                       0, 0.8544, -0.5196],
        "r_expected": [7.8102, 4.4813, 2.5607, 0, 4.6817, 0.9664, 0, 0,
                       -4.1843],
        "tolerance": 0.01,
    }
    out["small_qr"]["sym2"] = {
        "a": [7, 2, 2, 4],
        "q_expected": [0.962, -.275, .275, .962],
        "r_expected": [7.28, 3.02, 0, 3.3],
        "rq_expected": [7.83, 0.906, 0.906, 3.17],
        "tolerance": 0.01,
    }

    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                       "fixtures.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
