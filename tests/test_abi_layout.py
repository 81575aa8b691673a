"""The ctypes mirrors in grapher_b200/_native.py have the C layout of the
structs include/gvizcuda.h declares: a small C program compiled with the
system compiler against the header prints each struct's size and every
field's offset, and the Python side must agree field for field (no GPU)."""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> ctypes class name in grapher_b200._native
STRUCTS = {
    "gvizCudaForceParams": "ForceParams",
    "gvizCudaGraphDesc": "GraphDesc",
    "gvizCudaCsr": "Csr",
    "gvizCudaStepStats": "StepStats",
    "gvizCudaGripRoundStats": "GripRoundStats",
}


@pytest.fixture(scope="module")
def c_layout():
    from grapher_b200 import _native as N
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gvizcuda.h"',
             "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(N, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                       check=True, capture_output=True, text=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, key, value = line.split()
        layout[(cname, key)] = int(value)
    return N, layout


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_mirror_matches_the_header(c_layout, cname):
    N, layout = c_layout
    cls = getattr(N, STRUCTS[cname])
    assert C.sizeof(cls) == layout[(cname, "size")]
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == layout[(cname, field)], field
