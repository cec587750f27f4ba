"""The ctypes mirrors of the C-ABI structs (revsim/_lib.py) against the headers: every field's
offset and each struct's size, as the C compiler lays them out.  A mismatch would hand the
library shifted fields; this runs on CPU with gcc."""

import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

STRUCTS = {
    "revsim_system_desc": "SystemDesc",
    "revsim_rdf_term": "RdfTermC",
    "revsim_barostat_desc": "BarostatDesc",
    "revsim_sw_desc": "SwDesc",
    "revsim_sw_loss": "SwLossC",
    "revsim_gas_desc": "GasDesc",
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_headers(tmp_path):
    from revsim import _lib
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "revsim.h"',
             '#include "revsim_sw.h"', '#include "revsim_gas.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        py = getattr(_lib, pyname)
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            name, field, val = line.split()
            got[(name, field)] = int(val)
    for cname, pyname in STRUCTS.items():
        py = getattr(_lib, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])
