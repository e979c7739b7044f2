"""The ctypes structures of `_lib.py` against the C layout of
`include/sgpar_b200.h`: a small C program, compiled here with gcc against the
header, prints the size of every public struct and the offset of every field,
and each must equal ctypes' own.  A field added to one side only (the options
struct has grown twice) would otherwise pass values into the wrong fields or
write past a caller's stack copy.  CPU only: nothing runs on a device."""
import ctypes
import os
import shutil
import subprocess

import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "sgpar_b200.h")

# ctypes names that differ from the C field (Python keywords)
C_NAME = {"lambda_": "lambda"}

STRUCTS = [L.sgp_pcg32_random_t, L.sgp_graph_t, L.config_t, L.sgp_b200_graph_t, L.sgp_b200_options_t,
           L.sgp_b200_result_t, L.sgp_b200_mtx_info_t]


def c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for s in STRUCTS:
        name = s.__name__
        lines.append(f'    printf("{name} size %zu\\n", sizeof({name}));')
        for f in s._fields_:
            field = f[0]
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {C_NAME.get(field, field)}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return dict((" ".join(l.split()[:2]), int(l.split()[2])) for l in out.splitlines())


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_header(tmp_path):
    got = c_layout(tmp_path)
    for s in STRUCTS:
        name = s.__name__
        assert got[f"{name} size"] == ctypes.sizeof(s), name
        for f in s._fields_:
            assert got[f"{name} {f[0]}"] == getattr(s, f[0]).offset, (name, f[0])
