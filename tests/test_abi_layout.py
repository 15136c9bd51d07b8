"""The Python mirrors of the C structs have the header's layout.

A small C program built against include/mfcfd.h prints sizeof and the
offset of every field of each struct the Python package passes across the
boundary; each must equal the ctypes mirror's.  A field added on one side
only (or in a different place) fails here instead of shifting the fields
after it in silence.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [("Params", "mfcfd_params"), ("Info", "mfcfd_info"), ("ServerConfig", "mfcfd_server_config"),
         ("Request", "mfcfd_request"), ("Result", "mfcfd_result"), ("ServerStats", "mfcfd_server_stats")]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    from mfcfd import _lib
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "mfcfd.h"', "int main(void) {"]
    expect = []
    for py, c in PAIRS:
        cls = getattr(_lib, py)
        lines.append(f'    printf("{c} %zu\\n", sizeof({c}));')
        expect.append(f"{c} {ctypes_sizeof(cls)}")
        for f, _ in cls._fields_:
            lines.append(f'    printf("{c}.{f} %zu\\n", offsetof({c}, {f}));')
            expect.append(f"{c}.{f} {getattr(cls, f).offset}")
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")[:-1]
    assert got == expect


def ctypes_sizeof(cls):
    import ctypes
    return ctypes.sizeof(cls)
