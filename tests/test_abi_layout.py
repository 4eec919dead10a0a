"""The ctypes mirrors in oap_b200 against the C structs of include/oapb200.h:
a C program compiled here prints each field's offset and each struct's size,
and they must equal the ctypes layout (a field added on one side only would
shift every field after it)."""
import ctypes as C
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oap_b200 as B  # noqa: E402

STRUCTS = [("oapb_mat", B.Mat), ("oapb_arnoldi_config", B.Config), ("oapb_arnoldi_stats", B.Stats),
           ("oapb_trace_rec", B.TraceRec), ("oapb_batch_problem", B.BatchProblem),
           ("oapb_batch_stats", B.BatchStats)]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "oapb200.h"', "int main(void) {"]
    for cname, py in STRUCTS:
        lines.append('  printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, py in STRUCTS:
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
